// Launchers of the spline model's kernels (separate translation unit for parallel builds).
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_spline(int G, int, int) { return generic_fit_table<SplineModel>(G); }

EvalLaunch eval_launcher_spline(int G) { return eval_table<SplineModel>(G); }

AdjointLaunch adjoint_launcher_spline() { return launch_adjoint<SplineModel, 8>; }

}  // namespace pb200
