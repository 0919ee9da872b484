// Launchers of the tilted-background Gaussian models' kernels and of the intensity/background
// fit (generic table kernel; the column-blocked kernel covers the flat-background Gaussians).
#include "launch.cuh"

namespace pb200 {

FitLaunch fit_launcher_tilted(int G, int CPL, int variant) {
    (void)CPL;
    (void)variant;
    return generic_fit_table<TiltedGaussModel<MODEL_XYITILTEDBG>>(G);
}

FitLaunch fit_launcher_tilted_sxy(int G, int CPL, int variant) {
    (void)CPL;
    (void)variant;
    return generic_fit_table<TiltedGaussModel<MODEL_XYITILTEDBG_SIGMAXY>>(G);
}

EvalLaunch eval_launcher_tilted(int G) { return eval_table<TiltedGaussModel<MODEL_XYITILTEDBG>>(G); }

EvalLaunch eval_launcher_tilted_sxy(int G) { return eval_table<TiltedGaussModel<MODEL_XYITILTEDBG_SIGMAXY>>(G); }

FitLaunch fit_launcher_intensity_bg(int G) { return generic_fit_table<IntensityBgModel>(G); }

}  // namespace pb200
