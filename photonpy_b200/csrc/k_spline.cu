// Launchers of the spline models' kernels (separate translation unit for parallel builds):
// flat background, tilted background and background image.
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_spline(int G, int, int) { return generic_fit_table<SplineModel>(G); }

EvalLaunch eval_launcher_spline(int G) { return eval_table<SplineModel>(G); }

AdjointLaunch adjoint_launcher_spline() { return launch_adjoint<SplineModel, 8>; }

FitLaunch fit_launcher_spline_tilted(int G) { return generic_fit_table<SplineModelT<1>>(G); }

FitLaunch fit_launcher_spline_bgimage(int G) { return generic_fit_table<SplineModelT<2>>(G); }

EvalLaunch eval_launcher_spline_tilted(int G) { return eval_table<SplineModelT<1>>(G); }

EvalLaunch eval_launcher_spline_bgimage(int G) { return eval_table<SplineModelT<2>>(G); }

}  // namespace pb200
