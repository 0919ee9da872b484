// Launchers of the spline models' kernels (separate translation unit for parallel builds):
// flat background, tilted background and background image.
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_spline(int G, int, int) { return spline_fit_table<0>(G); }

StreamLaunch stream_launcher_spline(int, int) { return nullptr; }  // spline host calls use the slot pipeline

EvalLaunch eval_launcher_spline(int G) { return spline_eval_table<0>(G); }

static void launch_adjoint_spline(const ModelDesc& d, AdjointArgs a, cudaStream_t s) {
    if (d.spline_q == 1.0f) launch_adjoint<SplineModelT<0, false>, 8>(d, a, s);
    else launch_adjoint<SplineModelT<0, true>, 8>(d, a, s);
}

AdjointLaunch adjoint_launcher_spline() { return launch_adjoint_spline; }

FitLaunch fit_launcher_spline_tilted(int G) { return spline_fit_table<1>(G); }

FitLaunch fit_launcher_spline_bgimage(int G) { return generic_fit_table<SplineModelT<2>>(G); }

EvalLaunch eval_launcher_spline_tilted(int G) { return spline_eval_table<1>(G); }

EvalLaunch eval_launcher_spline_bgimage(int G) { return eval_table<SplineModelT<2>>(G); }

}  // namespace pb200
