// Device services of the spot detector and the camera calibration shared by the host
// translation units (spot_detect.cu, spot_queue.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/photonpy_b200.h"

namespace pb200 {

// Applies the calibration (CameraCalibration.cu semantics) to n frames [n][h][w] on stream s:
// out = f(in). The per-pixel calibrations need w x h equal to their image size (checked).
void camera_calib_apply_f32(const CameraCalibration* c, const float* d_in, float* d_out, int w, int h, int n,
                            cudaStream_t s);
// The same from raw 16-bit frames (converted exactly to float first); c may be null.
void camera_calib_apply_u16(const CameraCalibration* c, const uint16_t* d_in, float* d_out, int w, int h, int n,
                            cudaStream_t s);

// Spot detection and ordered compaction of n device frames with the factory's configuration:
// found[n], and the first maxSpots spots of each frame as pixel indices y*w+x (index[n][maxSpots])
// and scores (score[n][maxSpots]). No ROI cut-out.
void spot_detect_indices(SpotDetectorFactory* sdf, const float* d_frames, const float* d_bg, int n, int w, int h,
                         int maxSpots, int* d_found, int* d_index, float* d_score, cudaStream_t s);

// The configuration a factory was made with (its backgroundImage is the caller's host pointer).
const SpotDetectorConfig* spot_factory_config(const SpotDetectorFactory* sdf);

}  // namespace pb200
