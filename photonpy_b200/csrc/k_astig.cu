// Launchers of the astig model's kernels (separate translation unit for parallel builds).
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_astig(int G, int CPL, int variant) {
    if (variant == 0) return gauss_fit_table<GaussModel<MODEL_XYZIBG>>(G, CPL);
    return generic_fit_table<GaussModel<MODEL_XYZIBG>>(G);
}

StreamLaunch stream_launcher_astig(int G, int CPL) { return gauss_stream_table<GaussModel<MODEL_XYZIBG>>(G, CPL); }

EvalLaunch eval_launcher_astig(int G) { return eval_table<GaussModel<MODEL_XYZIBG>>(G); }

AdjointLaunch adjoint_launcher_astig() { return launch_adjoint<GaussModel<MODEL_XYZIBG>, 8>; }

}  // namespace pb200
