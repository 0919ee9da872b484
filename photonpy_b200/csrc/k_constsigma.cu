// Launchers of the constsigma model's kernels (separate translation unit for parallel builds).
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_constsigma(int G, int CPL, int variant) {
    if (variant == 0) return gauss_fit_table<GaussModel<MODEL_XYIBG_CONSTSIGMA>>(G, CPL);
    return generic_fit_table<GaussModel<MODEL_XYIBG_CONSTSIGMA>>(G);
}

StreamLaunch stream_launcher_constsigma(int G, int CPL) { return gauss_stream_table<GaussModel<MODEL_XYIBG_CONSTSIGMA>>(G, CPL); }

EvalLaunch eval_launcher_constsigma(int G) { return eval_table<GaussModel<MODEL_XYIBG_CONSTSIGMA>>(G); }

AdjointLaunch adjoint_launcher_constsigma() { return launch_adjoint<GaussModel<MODEL_XYIBG_CONSTSIGMA>, 8>; }

}  // namespace pb200
