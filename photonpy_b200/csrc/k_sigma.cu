// Launchers of the sigma model's kernels (separate translation unit for parallel builds).
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_sigma(int G, int CPL, int variant) {
    if (variant == 0) return gauss_fit_table<GaussModel<MODEL_XYIBG_SIGMA>>(G, CPL);
    return generic_fit_table<GaussModel<MODEL_XYIBG_SIGMA>>(G);
}

StreamLaunch stream_launcher_sigma(int G, int CPL) { return gauss_stream_table<GaussModel<MODEL_XYIBG_SIGMA>>(G, CPL); }

EvalLaunch eval_launcher_sigma(int G) { return eval_table<GaussModel<MODEL_XYIBG_SIGMA>>(G); }

AdjointLaunch adjoint_launcher_sigma() { return launch_adjoint<GaussModel<MODEL_XYIBG_SIGMA>, 8>; }

}  // namespace pb200
