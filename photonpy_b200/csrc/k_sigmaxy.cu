// Launchers of the sigmaxy model's kernels (separate translation unit for parallel builds).
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_sigmaxy(int G, int CPL, int variant) {
    if (variant == 0) return gauss_fit_table<GaussModel<MODEL_XYIBG_SIGMAXY>>(G, CPL);
    return generic_fit_table<GaussModel<MODEL_XYIBG_SIGMAXY>>(G);
}

StreamLaunch stream_launcher_sigmaxy(int G, int CPL) { return gauss_stream_table<GaussModel<MODEL_XYIBG_SIGMAXY>>(G, CPL); }

EvalLaunch eval_launcher_sigmaxy(int G) { return eval_table<GaussModel<MODEL_XYIBG_SIGMAXY>>(G); }

AdjointLaunch adjoint_launcher_sigmaxy() { return launch_adjoint<GaussModel<MODEL_XYIBG_SIGMAXY>, 8>; }

}  // namespace pb200
