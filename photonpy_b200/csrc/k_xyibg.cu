// Launchers of the xyibg model's kernels (separate translation unit for parallel builds).
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_xyibg(int G, int CPL, int variant) {
    if (variant == 0) return gauss_fit_table<GaussModel<MODEL_XYIBG>>(G, CPL);
    return generic_fit_table<GaussModel<MODEL_XYIBG>>(G);
}

StreamLaunch stream_launcher_xyibg(int G, int CPL) { return gauss_stream_table<GaussModel<MODEL_XYIBG>>(G, CPL); }

EvalLaunch eval_launcher_xyibg(int G) { return eval_table<GaussModel<MODEL_XYIBG>>(G); }

AdjointLaunch adjoint_launcher_xyibg() { return launch_adjoint<GaussModel<MODEL_XYIBG>, 8>; }

}  // namespace pb200
