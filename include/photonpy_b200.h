/* photonpy_b200 — C ABI of the B200 (sm_100a) batched Poisson-MLE PSF estimator.
 *
 * Drop-in for photonpy's estimator ABI: every function below that carries a
 * reference citation has the same name, argument order, argument meaning and
 * error behaviour as the photonpy export it replaces, so photonpy's ctypes
 * bindings (photonpy/cpp/estimator.py, gaussian.py, cspline.py, context.py) can
 * bind libphotonpy_b200.so unchanged. Unless stated otherwise all pointers are
 * HOST memory and the caller allocates every output. Errors never propagate as
 * C++ exceptions: like the reference, functions return void (factories return
 * NULL) and report through the debug-print callback; in addition the message is
 * kept for PB200_GetLastError().
 *
 * Citations are paths inside photonpy's cpp/SMLMLib.
 */
#ifndef PHOTONPY_B200_H
#define PHOTONPY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#else
#include <stdbool.h>
#endif

typedef struct Estimator Estimator; /* opaque */
typedef struct Context Context;     /* opaque */
typedef struct MixedPlan MixedPlan; /* opaque */

/* LMParams, Estimators/Estimator.h:18-26. `factor` is accepted and unused, as in the reference. */
typedef struct LMParams {
    int iterations;
    float lambda;
    float factor;
} LMParams;

/* ParamLimit, Estimators/Estimator.h:28-31. */
typedef struct ParamLimit {
    float min, max;
} ParamLimit;

/* EstimatorProperties, Estimators/Estimator.h:151-154. */
typedef struct EstimatorProperties {
    int numParams, sampleCount, numDiag, numConst, sampleIndexDims;
} EstimatorProperties;

/* Gauss3D_Calibration, Estimators/Gaussian/GaussianPSF.h:27-33:
 * sigma(z) = s0*sqrt(1 + tz^2/d^2 + A*tz^3/d^2), tz = z - gamma; x/y = {s0, gamma, d, A}. */
typedef struct Gauss3D_Calibration {
    float x[4];
    float y[4];
    float minz, maxz;
} Gauss3D_Calibration;

/* Extension (no reference counterpart): astigmatic calibration with a quartic term,
 * x/y = {s0, gamma, d, A, B}: sigma(z) = s0*sqrt(1 + tz^2/d^2 + A tz^3/d^2 + B tz^4/d^4).
 * B = 0 gives results identical to Gauss3D_Calibration. */
typedef struct Gauss3D_CalibrationB {
    float x[5];
    float y[5];
    float minz, maxz;
} Gauss3D_CalibrationB;

/* CSpline_Calibration, Estimators/CSpline/CubicSplinePSF.h:12-23 (shape = z, y, x). */
typedef struct CSpline_Calibration {
    int shape[3];
    float z_min;
    float z_max;
    const float* coefs; /* [shape0][shape1][shape2][64] */
} CSpline_Calibration;

/* ---- Context (Context.h:43-44) ------------------------------------------------------ */
Context* Context_Create(void);  /* replaces Context.cpp Context_Create */
void Context_Destroy(Context* ctx); /* replaces Context_Destroy; deletes every estimator it owns */

/* ---- Estimator factories -------------------------------------------------------------
 * `cuda` is accepted for ABI compatibility; every estimator of this library runs on the
 * current CUDA device (there is no CPU path). */
/* Estimators/Gaussian/GaussianPSF.cu:87-108 */
Estimator* Gauss2D_CreatePSF_XYIBg(int roisize, float sigmaX, float sigmaY, bool cuda, Context* ctx);
/* Estimators/Gaussian/GaussianPSF.cu:110-132 (sigma x/y per spot as 2 constants) */
Estimator* Gauss2D_CreatePSF_XYIBgConstSigma(int roisize, bool cuda, Context* ctx);
/* Estimators/Gaussian/GaussianPSF.cu:136-158 */
Estimator* Gauss2D_CreatePSF_XYIBgSigma(int roisize, float initialSigma, bool cuda, Context* ctx);
/* Estimators/Gaussian/GaussianPSF.cu:162-185 */
Estimator* Gauss2D_CreatePSF_XYIBgSigmaXY(int roisize, float initialSigmaX, float initialSigmaY, bool cuda,
                                          Context* ctx);
/* Estimators/Gaussian/GaussianPSF.cu:36-59 (the calibration is passed by reference in C++,
 * i.e. as a pointer in the ABI) */
Estimator* Gauss2D_CreatePSF_XYZIBg(int roisize, const Gauss3D_Calibration* calib, bool cuda, Context* ctx);
/* Estimators/Gaussian/GaussianPSF.cu:62-85: theta = (x, y, I, bg, bgx, bgy), sigma_x/sigma_y as
 * 2 per-spot constants, mu = bg + bgx (x - W/2) + bgy (y - H/2) + I PSF. */
Estimator* Gauss2D_CreatePSF_XYITiltedBg(int roisize, bool cuda, Context* ctx);
/* Estimators/Gaussian/GaussianPSF.cu:187-212: theta = (x, y, I, bg, bgx, bgy, sx, sy). As in the
 * reference, the tilt is in the Jacobian but not in mu (GaussianPSFModels.h:542 vs 549). */
Estimator* Gauss2D_CreatePSF_XYITiltedBgSigmaXY(int roisize, float initialSigmaX, float initialSigmaY, bool cuda,
                                                Context* ctx);
/* Estimators/Gaussian/GaussianPSF.cu:216-240: intensity and background of numspots ROIs
 * imageData[n][imgw][imgw] with the spot at xy[n][2]: LM fit of mu = I*DeltaX*DeltaY + bg from
 * (1, 0), lambda 1e-15, maxIterations iterations; IBg[n][2] = (I, bg), IBg_crlb[n][2] =
 * sqrt(|diag(Fisher^-1)|) (nullable). Spot i's sigma is sigma[i] of the flat array, as in the
 * reference (photonpy passes [n][2] floats). roipos is unused, as in the reference. */
void Gauss2D_EstimateIntensityBg(const float* imageData, float* IBg, float* IBg_crlb, int numspots, const float* xy,
                                 const int* roipos, const float* sigma, int imgw, int maxIterations, bool cuda);
/* Extension (no reference counterpart): astigmatic model with the quartic B term. */
Estimator* Gauss2D_CreatePSF_XYZIBgB(int roisize, const Gauss3D_CalibrationB* calib, bool cuda, Context* ctx);
/* Estimators/CSpline/CubicSplinePSF.cu:55-107. mode 0 flat background (x,y,z,I,bg), 1 tilted
 * background (x,y,z,I,bg,bgx,bgy), 2 background image (x,y,z,I,bg with mu = I psf + bg * image;
 * the image is the spot's roisize*roisize constants). coefs (nullable) overrides calib->coefs.
 * The coefficients are copied to the device at creation. */
Estimator* CSpline_CreatePSF(int roisize, const CSpline_Calibration* calib, const float* coefs, int mode, bool cuda,
                             Context* ctx);
/* Estimators/CSpline/CubicSplinePSF.cu:135-146: z-stack file (header v1) -> coefficients (border 0). */
Estimator* CSpline_CreatePSF_FromFile(int roisize, const char* filename, int mode, bool cuda, Context* ctx);
/* Extension (no reference counterpart; photonpy's spline has one voxel per ROI pixel,
 * CubicSplinePSFModels.h:79-96,120-141): a spline calibration sampled every xyStep ROI pixels in
 * x and y (0 < xyStep <= 1, e.g. 0.5 for a 2x oversampled PSF). Pixel (x, y) of a spot at
 * (theta_x, theta_y) reads the spline at grid coordinate (x - theta_x)/xyStep + N/2; the x/y
 * derivatives scale by 1/xyStep. Modes 0 (flat) and 1 (tilted background). xyStep = 1 gives
 * results identical to CSpline_CreatePSF. */
Estimator* CSpline_CreatePSF_Oversampled(int roisize, const CSpline_Calibration* calib, const float* coefs, int mode,
                                         float xyStep, bool cuda, Context* ctx);
/* Estimators/CSpline/CubicSplinePSF.cu:151-204: spline coefficients of a z-stack, computed on the
 * GPU with the reference's double-precision LUP solve (bit-identical output).
 * coefs[shape-3+2*border][64]. */
void CSpline_Compute(const int* shape, const float* data, float* splineCoefs, int border);
/* Estimators/CSpline/CubicSplinePSF.cu:208-271: value and x/y/z derivatives of the spline at
 * a shifted position; values[(shape-2*border)][4]. */
void CSpline_Evaluate(const int* shape, const float* splineCoefs, const float* shift, int border, float* values);

/* ---- Estimator C API (Estimators/Estimator.h:157-171, Estimator.cpp:45-157) ---------- */
void Estimator_Delete(Estimator* e);
const char* Estimator_ParamFormat(Estimator* e);
void Estimator_GetProperties(Estimator* e, EstimatorProperties* props);
void Estimator_SampleDims(Estimator* e, int* dims);
void Estimator_GetParamLimits(Estimator* e, ParamLimit* limits);
void Estimator_SetLMParams(Estimator* e, const LMParams* p);
void Estimator_GetLMParams(Estimator* e, LMParams* p);
/* ev[numspots][H][W] */
void Estimator_ComputeExpectedValue(Estimator* e, int numspots, const float* params, const float* constants,
                                    const int* spotpos, float* ev);
/* Fit (centre-of-mass start when initial == NULL). params[n][K], iterations[n] (nullable;
 * = i+1 at the stop, maxIterations+1 when capped), trace[n][traceBufLen][K] (nullable),
 * diagnostics: numDiag floats per spot (3 for GLRT estimators; none, untouched, otherwise). */
void Estimator_Estimate(Estimator* e, int numspots, const float* sample, const float* constants, const int* spotpos,
                        const float* initial, float* params, float* diagnostics, int* iterations, float* trace,
                        int traceBufLen);
/* deriv[n][K][H][W], ev[n][H][W] */
void Estimator_ComputeDerivatives(Estimator* e, int numspots, const float* params, const float* constants,
                                  const int* spotpos, float* psf_deriv, float* ev);
/* crlb[n][K], chisq[n] (sample nullable: chi-square not computed, written as 0). */
void Estimator_ChiSquareAndCRLB(Estimator* e, const float* params, const float* sample, const float* constants,
                                const int* spotpos, int numspots, float* crlb, float* chisq);

/* ---- Likelihood-ratio test, Estimators/GLRT_PSF.cu:58-170 ---------------------------
 * GLRT_CreatePSF returns an estimator with the model's parameters, limits and fit whose
 * Estimate also writes 3 diagnostics per spot (numDiag = 3): ll_on = sum d log(mu) - mu at
 * the fitted parameters, ll_off = sum d log(mean) - mean for the background-only model, and
 * mean; d = max(sample, 1e-8), mu clamped at 1e-8 (GLRT_PSF.cu:104-131). The reference takes
 * `mean` from the FIRST ROI of the call for every spot (its inner loop variable shadows the
 * spot index, GLRT_PSF.cu:107-108); here each spot uses its own mean unless
 * PB200_SetGLRTReferenceMean(e, 1) selects the reference's behaviour (extension, returns 0 or
 * -1). The GLRT estimator is a copy of `model` (deleting the model does not affect it). */
Estimator* GLRT_CreatePSF(Estimator* model, Context* ctx);                     /* GLRT_PSF.cu:156 */
int PB200_SetGLRTReferenceMean(Estimator* e, int on);

/* ---- Estimation queue, Estimators/EstimationQueue.h:21-25, 112-126 --------------------
 * Streams ROIs from host memory through the fit + CRLB + chi-square kernels: spots are
 * packed into pinned batches of batchSize; a worker thread launches waiting batches on
 * numStreams CUDA streams (numStreams < 0: 3), several full batches per launch when they
 * are waiting; results are collected per batch. GetResults returns only whole batches,
 * removes them from the queue, and does not keep batch order (sort by id). Differences from
 * the reference, none of which changes a result: maxQueueLen counts SPOTS (waiting or in
 * flight) and EstimQueue_Schedule blocks on entry while that count is at least
 * max(maxQueueLen, batchSize); a batch never mixes spots scheduled with and without initial
 * values (a change flushes the batch); roipos is returned as scheduled; diag receives
 * numDiag floats per spot (the GLRT values for GLRT estimators, none otherwise). Inputs are
 * staged in a bounded pool of pinned buffers: Schedule also waits while all are in use. */
typedef struct EstimQueue EstimQueue;  /* opaque; the reference's EstimationQueue */
typedef struct EstimatorResult {       /* Estimators/EstimationQueue.h:21-25 */
    int id;
    float chisq;
    int iterations;
} EstimatorResult;
EstimQueue* EstimQueue_Create(Estimator* psf, int batchSize, int maxQueueLen, bool keepSamples, int numStreams,
                              Context* ctx);                                   /* EstimationQueue.cpp:317 */
void EstimQueue_Delete(EstimQueue* q);                                         /* EstimationQueue.cpp:336 */
/* ids[n], samples[n][H][W], initial[n][K] (nullable), constants[n][numConst] (nullable when
 * numConst is 0), roipos[n][2]; copied before the call returns. EstimationQueue.cpp:346 */
void EstimQueue_Schedule(EstimQueue* q, int numspots, const int* ids, const float* h_samples, const float* h_initial,
                         const float* h_constants, const int* h_roipos);
void EstimQueue_Flush(EstimQueue* q);                                          /* EstimationQueue.cpp:357 */
bool EstimQueue_IsIdle(EstimQueue* q);                                         /* EstimationQueue.cpp:367 */
int EstimQueue_GetResultCount(EstimQueue* q);                                  /* EstimationQueue.cpp:378 */
int EstimQueue_GetQueueLength(EstimQueue* q);                                  /* EstimationQueue.cpp:389 */
/* Copies whole finished batches while they fit in maxresults; every output nullable (samples
 * only when the queue keeps them). Returns the number of spots copied. EstimationQueue.cpp:402 */
int EstimQueue_GetResults(EstimQueue* q, int maxresults, float* estim, float* diag, float* crlb, int* roipos,
                          float* samples, EstimatorResult* results);

/* ---- Spot detection and ROI extraction, SpotDetection/SpotDetector.h:39-62, 129-137 -----
 * Detection image D = box(frame - bg, u1) - box(frame - bg, u2) (windows clipped at the border);
 * a pixel is a spot where D equals its maxFilterSize maximum, its ROI fits the frame, and
 * minIntensity < D < maxIntensity. Spots come in row-major pixel order. */
typedef struct SpotDetectorConfig { /* layout of photonpy/cpp/spotdetect.py's SpotDetector */
    int uniformFilter1Size, uniformFilter2Size, maxFilterSize;
    int roisize;                    /* border test */
    float minIntensity, maxIntensity;
    float* backgroundImage;         /* host [h][w] or NULL; read at every ProcessFrame call */
} SpotDetectorConfig;
typedef struct SpotDetectorFactory SpotDetectorFactory; /* opaque; the reference's ISpotDetectorFactory */
/* SpotDetector.cu:21-28. Filter windows up to 32 pixels. */
SpotDetectorFactory* SpotDetector_Configure(const SpotDetectorConfig* config);
void SpotDetector_DestroyFactory(SpotDetectorFactory* factory);
/* SpotDetector.cu:101-151: detects the spots of one host frame [height][width], returns their
 * number (at most maxSpots) and writes scores[n], spotZ[n] (0), cornerPosYX[n][2] = (y, x) -
 * roisize/2 and rois[n][roisize][roisize] (pixels clamped to the frame). calib: NULL or a
 * CameraCalibration*; as in the reference the detector sees the calibrated frame and the ROIs
 * are cut from the frame as given. Returns 0 on error. */
int SpotDetector_ProcessFrame(const float* frame, int width, int height, int roisize, int maxSpots, float* spotScores,
                              int* spotZ, int* cornerPosYX, float* rois, SpotDetectorFactory* sdf, void* calib);
/* SpotDetector.cu:155-178: boxes [roiZ][roiY][roiX] at corners startposZYX[n][3] of a frame stack
 * [depth][height][width], y/x clamped. As in the reference, box slice z is read from frame z of
 * the stack whatever the corner's z. */
void ExtractROIs(const float* frames, int width, int height, int depth, int roiX, int roiY, int roiZ,
                 const int* startposZYX, int numspots, float* rois);
/* ---- Camera calibration, CameraCalibration.cu:9-83 ------------------------------------
 * Applied to every frame before detection: gain/offset v = max(0, (x - offset) * gain) (NaN kept),
 * per-pixel gain/offset images the same, sCMOS v = (x - offset[p]) * gain[p]. Owned by ctx
 * (destroyed with it), as in the reference. */
typedef struct CameraCalibration CameraCalibration; /* opaque; the reference's ICalibrationProcessor */
CameraCalibration* GainOffsetCalib_Create(float gain, float offset, Context* ctx);
CameraCalibration* GainOffsetImageCalib_Create(int width, int height, const float* gain, const float* offset,
                                               Context* ctx);
CameraCalibration* sCMOS_Calib_Create(int width, int height, const float* offset, const float* gain,
                                      const float* variance, Context* ctx);

/* ---- ROI queue, ROIQueue.cpp:8-95 --------------------------------------------------------
 * Thread-safe FIFO of ROIs [shape z][y][x] with their info. RQ_Pop takes the `count` oldest ROIs
 * and, as the reference, writes them newest first; it writes nothing when fewer than `count` are
 * queued. shape is zyx (Int3). */
typedef struct ROIQueue ROIQueue; /* opaque */
typedef struct ROIInfo {          /* photonpy/cpp/roi_queue.py ROIInfoDType */
    int id;                       /* frame (or summed-frame) number */
    float score;
    int x, y, z;                  /* ROI corner; z plane of the detector */
} ROIInfo;
ROIQueue* RQ_Create(const int* shapeZYX, Context* ctx);
void RQ_Pop(ROIQueue* q, int count, ROIInfo* rois, float* data);
int RQ_Length(ROIQueue* q);
void RQ_Push(ROIQueue* q, int count, const ROIInfo* info, const float* data);
void RQ_SmpShape(ROIQueue* q, int* shapeZYX);
void RQ_Delete(ROIQueue* q);

/* ---- Frame processors, ImageProcessor.cpp:12-51 ----------------------------------------- */
typedef struct ImageProcessor ImageProcessor; /* opaque */
void ImgProc_Flush(ImageProcessor* q);
void ImgProc_AddFrameU16(ImageProcessor* q, const uint16_t* data);
void ImgProc_AddFrameF32(ImageProcessor* q, const float* data);
int ImgProc_GetQueueLength(ImageProcessor* q);
int ImgProc_ReadFrame(ImageProcessor* q, float* image, float* processed);
int ImgProc_NumFinishedFrames(ImageProcessor* q);
bool ImgProc_IsIdle(ImageProcessor* q);
void ImgProc_Destroy(ImageProcessor* q);
/* ImgFilterQueue.cu:117-346: 16-bit frames in (ImgProc_AddFrameU16), calibrated, summed in
 * groups of sumframes = the ROI queue's z size (as in the reference, the sumframes argument is not
 * used), spots detected on each summed frame with the factory's configuration (copied, with its
 * background image, at creation), and ROIs [sumframes][y][x] of the calibrated frames pushed
 * into roilist with id = summed-frame number, x/y = corner, z = 0, score. Frames are processed
 * in batches of whatever complete groups are waiting, on the GPU, by one worker thread
 * (numDetectionThreads is not used). ImgProc_AddFrameF32 is an error, as in the reference. */
ImageProcessor* SpotExtractionQueue_Create(int width, int height, ROIQueue* roilist, SpotDetectorFactory* sdf,
                                           CameraCalibration* calib, int numDetectionThreads, int sumframes,
                                           Context* ctx);
/* ImageProcessor.cpp:61-233: extraction of predefined ROIs from a stream of 16-bit frames
 * (ImgProc_AddFrameU16, calibrated as above). ROI i takes the roisize x roisize box at
 * (x, y) = cornerpos of numframes frames from startframe (frames numbered from 0 in push order;
 * box coordinates clamped to the frame, where the reference reads outside it); its record is
 * available once its last frame is processed, records in order of last frame, then start
 * frame, then request order. ROIExtractor_GetResults hands out up to numrois records oldest
 * first; slot i of framedata [numrois][roiframes][roisize][roisize] gets min(numframes,
 * roiframes) boxes. NumFinishedFrames counts processed frames (the reference returns 0). */
typedef struct ExtractionROI { /* photonpy/cpp/image_proc.py ROIExtractor.ROIType */
    int cornerpos[2];          /* x, y */
    int startframe, numframes;
} ExtractionROI;
ImageProcessor* ROIExtractor_Create(int imgWidth, int imgHeight, const ExtractionROI* rois, int numrois, int roiframes,
                                    int roisize, CameraCalibration* calib, Context* ctx);
int ROIExtractor_GetResultCount(ImageProcessor* re);
int ROIExtractor_GetResults(ImageProcessor* re, int numrois, ExtractionROI* rois, float* framedata);

/* Extension: detection and ROI cut-out of nframes device frames [n][height][width] on a stream,
 * for feeding the fitter without host copies. d_bg: device [height][width] or NULL (the
 * configuration's host background image is not used here). Outputs (device): d_found[n] (spots
 * found per frame, may exceed maxSpotsPerFrame), d_scores[n][maxSpotsPerFrame] (nullable),
 * d_cornerYX[n][maxSpotsPerFrame][2] and d_rois[n][maxSpotsPerFrame][roisize][roisize] (nullable
 * together); the first min(found, maxSpotsPerFrame) entries of each frame are written.
 * The factory's device scratch (about one frame batch of floats) is kept between calls and
 * grown on demand; calls on one factory from different streams are ordered by an event.
 * Returns 0 or -1. */
int PB200_DetectSpotsDevice(SpotDetectorFactory* sdf, const float* d_frames, const float* d_bg, int nframes,
                            int width, int height, int roisize, int maxSpotsPerFrame, int* d_found, int* d_cornerYX,
                            float* d_scores, float* d_rois, void* stream);
/* Extension (diagnostic): the spot detector's box filters divide a sum by a pixel count k with
 * one multiply by the rounded reciprocal and one FMA correction instead of an IEEE division.
 * This compares the two bit for bit on the current device for every float x and k = 1..maxCount
 * (maxCount <= 32): mismatches[k-1] = number of differing results (NaN vs NaN is equal),
 * lastBadBits[k-1] (nullable) = bits of one such x. Returns 0 or -1. */
int PB200_CheckCountDivision(int maxCount, unsigned long long* mismatches, unsigned* lastBadBits);

/* ---- Loader-time exports bound eagerly by photonpy/cpp/lib.py ------------------------ */
int CudaGetNumDevices(void);                                                        /* CudaUtils.cu:12 */
bool CudaSetDevice(int index);                                                      /* CudaUtils.cu:19 */
bool CudaGetDeviceInfo(int index, int* numMultiprocessors, char* name, int namelen); /* CudaUtils.cu:24 */
void CudaGetMemoryUse(uint64_t* pinnedBytes, uint64_t* devicePitchedBytes, uint64_t* deviceBytes,
                      uint64_t* pitchedNumAllocs);                                  /* CudaUtils.cu:38 */
void SetDebugPrintCallback(int (*cb)(const char* msg));                             /* StringUtils.cpp:45 */
void SetDebugImageCallback(void (*cb)(int w, int h, int n, const float* d, const char* t)); /* DebugImageCallback.h:9 */
void ShowDebugImage(int w, int h, int numImg, const float* data, const char* title); /* DebugImageCallback.h:10 */
/* Out-of-scope exports that lib.py/gaussian.py bind at load time: present so those bindings
 * load; each reports "not provided by photonpy_b200" and does nothing. */
void FFT(const void* src, void* dst, int batchsize, int siglen, int forward);
void FFT2(const void* src, void* dst, int batchsize, int sigw, int sigh, int forward);
void DrawROIs(float* image, int width, int height, const float* rois, int numrois, int roisize, const int* roiposYX);
void Gauss2D_Draw(double* image, int imgw, int imgh, float* spotList, int nspots, float addSigma);
/* Bound by SpotDetectionMethods.__init__ (photonpy/cpp/spotdetect.py:117): the PSF-correlation
 * detector (PSFCorrelationSpotDetector.cu:13). Returns NULL. */
void* PSFCorrelationSpotDetector_Configure(const float* bgImage, int imageWidth, int imageHeight,
                                           const float* psfstack, int roisize, int depth, int maxFilterSizeXY,
                                           float minPhotons, int bgFilterSize, int debugMode);

/* ---- Extensions (no reference counterpart) ------------------------------------------ */
/* Message of the last error on this thread ("" if none); cleared by PB200_ClearError. */
const char* PB200_GetLastError(void);
void PB200_ClearError(void);
/* Localization in one call: LM fit, Fisher/CRLB + chi-square at the fitted parameters (what
 * photonpy's EstimationQueue runs as Estimate followed by ChiSquareAndCRLB,
 * EstimationQueue.cpp:285-289): LM launch, Fisher pass, FP64 inverse. Host pointers; large
 * batches of the flat-background Gaussian models at their default configuration are fitted by
 * one LM launch while a copy stream brings the ROIs in (when the fits outlast the copies,
 * which each estimator's first large call measures), others in chunks pipelined over four
 * CUDA streams. */
void PB200_EstimateCRLB(Estimator* e, int numspots, const float* sample, const float* constants,
                        const float* initial, float* params, int* iterations, float* crlb, float* chisq);
/* Device-pointer variants on a caller stream (cudaStream_t as void*; NULL = legacy default).
 * No host synchronisation; all pointers are device memory. crlb/chisq/iterations/trace nullable. */
void PB200_EstimateDevice(Estimator* e, int numspots, const float* d_sample, const float* d_constants,
                          const float* d_initial, float* d_params, int* d_iterations, float* d_trace, int traceBufLen,
                          float* d_crlb, float* d_chisq, void* stream);
void PB200_ExpectedValueDevice(Estimator* e, int numspots, const float* d_params, const float* d_constants,
                               float* d_ev, float* d_deriv, void* stream);
/* PB200_EstimateDevice with the per-spot diagnostics of the estimator (numDiag floats per spot:
 * 3 for GLRT estimators, none otherwise; d_diag nullable) and without the trace. */
void PB200_EstimateDeviceDiag(Estimator* e, int numspots, const float* d_sample, const float* d_constants,
                              const float* d_initial, float* d_params, float* d_diag, int* d_iterations,
                              float* d_crlb, float* d_chisq, void* stream);
void PB200_ChiSquareAndCRLBDevice(Estimator* e, int numspots, const float* d_params, const float* d_sample,
                                  const float* d_constants, float* d_crlb, float* d_chisq, void* stream);
/* PB200_EstimateDevice without the CRLB, reporting per spot whether any LM step of its fit was
 * re-solved in FP64 (d_rescued[numspots]: 1 or 0). The FP32 damped Cholesky solve hands a step to
 * an FP64 re-solve when a pivot keeps less than a millionth of its diagonal entry (v <= 1e-6 a_kk,
 * or v < 0), where the reference's FP32 Cholesky (SolveMatrix.h:107-125) returns an inaccurate or
 * NaN step; an exactly zero pivot still ends the fit as in the reference. */
void PB200_EstimateDeviceRescued(Estimator* e, int numspots, const float* d_sample, const float* d_constants,
                                 const float* d_initial, float* d_params, int* d_iterations, float* d_trace,
                                 int traceBufLen, int* d_rescued, void* stream);
/* Replaces photonpy's numpy Estimator.FisherMatrix (photonpy/cpp/estimator.py:205-220), which
 * sums Derivatives/ExpectedValue on the host: the Fisher matrices of the Poisson likelihood at
 * params, FI_ij = sum_p J_i J_j / max(mu_p, 1e-8) (FP32 sums, the matrix the CRLB inverts),
 * computed on the GPU by the Fisher pass. Host pointers; fisher[numspots][K][K] (symmetric). */
void PB200_FisherMatrix(Estimator* e, int numspots, const float* params, const float* constants, float* fisher);
/* Device form: packed rows d_fisherRows[numspots][K(K+1)/2 + 1], the upper triangle row by row
 * (FI_00, FI_01, ..., FI_0K-1, FI_11, ...) then one float left 0 (no samples, no chi-square). */
void PB200_FisherMatrixDevice(Estimator* e, int numspots, const float* d_params, const float* d_constants,
                              float* d_fisherRows, void* stream);
/* Adjoint of the summed Poisson NLL (no reference counterpart). For each spot n:
 * nll[n] = sum_p mu_p - x_p log(max(mu_p, 1e-6)); dparams[n][k] = g_n dNLL_n/dtheta_k (true
 * derivatives, also for sigma); d_dcalib is ACCUMULATED into (zero it first): sum_n g_n dNLL_n/dcal
 * for XYIBg (sigma_x, sigma_y: 2 floats), XYZIBg (s0, gamma, d, A, B for x then y: 10 floats) and
 * CSpline (one value per coefficient, the coefficient array's shape). g_n = d_gradOut[n] or 1.
 * `calib` (host, nullable) overrides the estimator's sigma pair (XYIBg) or astig coefficients
 * (XYZIBg, 10 floats); d_coefs (device, nullable) overrides the spline coefficients. Device
 * pointers, caller stream; d_nll/d_dparams/d_dcalib nullable. Returns 0 or -1 (error). */
int PB200_PoissonNLLAdjoint(Estimator* e, int numspots, const float* d_sample, const float* d_params,
                            const float* d_constants, const float* calib, const float* d_coefs, const float* d_gradOut,
                            float* d_nll, float* d_dparams, float* d_dcalib, void* stream);
/* Spline calibration step (no reference counterpart): for a flat-background spline estimator and
 * spots with known parameters d_params[n][5], in one pass over the ROIs: d_nll[n] (nullable), the
 * gradient of the summed NLL with respect to every coefficient ACCUMULATED into d_grad (nullable,
 * the coefficient array's shape), and the diagonal of the Fisher information with respect to the
 * coefficients, sum_n sum_p I_n^2 f_m^2 / mu_p, ACCUMULATED into d_fisherDiag (nullable).
 * d_coefs (device, nullable) replaces the estimator's coefficients. Returns 0 or -1. */
int PB200_SplineCoefGradient(Estimator* e, int numspots, const float* d_sample, const float* d_params,
                             const float* d_coefs, float* d_nll, float* d_grad, float* d_fisherDiag, void* stream);
/* Mixed batches (no reference counterpart; photonpy runs one estimator, i.e. one model and
 * ROI size, per call). A plan binds nbuckets (estimator, count, device buffers) groups; one
 * run fits all of them with two persistent launches (the LM pass over every bucket, then the
 * Fisher/CRLB pass at the fitted parameters) and the FP64 CRLB kernels. In each launch a warp
 * walks the buckets in order and its ROI groups take tileRois consecutive ROIs of the current
 * bucket per claim from the bucket's counter. Buckets must be Gaussian models with ROI size
 * <= 16. d_constants/d_iterations/d_crlb/d_chisq arrays (and their entries) may be NULL. The
 * plan owns its scratch (task tables, ROI counters, Fisher rows). threadsPerBlock selects the
 * kernel's register budget: 128 (3 blocks per SM), 256 (2 blocks per SM), 129 (128 threads,
 * 4 blocks per SM). PB200_MixedPlanCapture records one run into a CUDA graph on `stream`
 * (non-default); later PB200_MixedPlanRun calls replay it. Runs of one plan must not overlap.
 * PB200_MixedPlanInfo's totalTiles is the number of claims, sum of ceil(count / tileRois). */
MixedPlan* PB200_MixedPlanCreate(int nbuckets, Estimator* const* ests, const int* counts, const float* const* d_samples,
                                 const float* const* d_constants, float* const* d_params, int* const* d_iterations,
                                 float* const* d_crlb, float* const* d_chisq, int tileRois, int threadsPerBlock);
int PB200_MixedPlanRun(MixedPlan* plan, void* stream);
int PB200_MixedPlanCapture(MixedPlan* plan, void* stream);
int PB200_MixedPlanInfo(MixedPlan* plan, int* ntasks, int* totalTiles, int* strideFloats);
/* Lanes per ROI each bucket of the plan runs with (lanes[nbuckets], in the order passed to
 * PB200_MixedPlanCreate): 4, or 2 for 7..10 px buckets of at least 1024 ROIs per SM (as the
 * per-bucket launches do by default). Per-bucket launches with these lanes per ROI give the
 * plan's results bit for bit. Returns 0, or -1 on a bad argument. */
int PB200_MixedPlanLanes(MixedPlan* plan, int nbuckets, int* lanes);
/* No counterpart in the reference. standalone[b] = 1 for each bucket that runs as launches of
 * its own (the single-model LM, Fisher and CRLB launches at the default configuration, on a stream
 * forked from the run's stream, because it holds at least PB200_GetMixedStandaloneMin() ROIs per
 * SM), 0 for those fitted inside the persistent mixed kernel.
 * Returns 0, or -1 on a bad argument. */
int PB200_MixedPlanStandalone(MixedPlan* plan, int nbuckets, int* standalone);
/* No counterpart in the reference. ROIs per SM from which a bucket of the mixed plans created
 * afterwards runs as launches of its own (default 0: every bucket; a negative value restores it, a
 * value above any bucket size keeps every bucket in the persistent kernel). Process-wide. */
void PB200_SetMixedStandaloneMin(int roisPerSM);
int PB200_GetMixedStandaloneMin(void);
void PB200_MixedPlanDestroy(MixedPlan* plan);
/* No counterpart in the reference. Fit + CRLB + chi-square in one call like PB200_EstimateDevice,
 * for callers that must not allocate device memory during a fit (real-time acquisition loops
 * with all device memory reserved in advance, hosts whose memory must come from their own
 * pools): it calls no cudaMalloc/cudaFree or other allocating routine. Its scratch, the
 * packed Fisher rows and the ROI counter of the LM launch (zeroed with cudaMemsetAsync), lives in
 * fixed device arrays of 32768 spots x 22 floats (2.75 MiB per GPU that loads the library, kept
 * until exit) and 4 ints, so numspots above 32768 is rejected with an
 * error (split the batch), and so is an estimator of more than 6 parameters (the tilted-
 * background SigmaXY Gaussian, the spline tilted-background mode), whose Fisher rows do not
 * fit a 22-float row; such calls launch nothing. All pointers are device memory; d_crlb is required, d_iterations and
 * d_chisq may be NULL. The first call on a device looks up the arrays' device addresses; make
 * that first call before any stream capture. Every call shares the arrays and overwrites the
 * rows and the counter it uses, so calls whose kernels overlap on the GPU (other streams, other threads) race:
 * serialise them. Returns 0 on success, -1 on error (message in PB200_GetLastError). */
int PB200_EstimateCRLBNoAlloc(Estimator* e, int numspots, const float* d_sample, const float* d_constants,
                              const float* d_initial, float* d_params, int* d_iterations, float* d_crlb,
                              float* d_chisq, void* stream);
/* Kernel configuration used for this estimator: lanes per ROI (2, 4, 8, 16, 32; 0 = automatic;
 * 2 for the column-blocked Gaussian kernel with ROIs up to 10 pixels wide, otherwise the next
 * supported count is used) and threads per block (64..256, a multiple of 32; 0 = automatic).
 * Returns 0 on success. */
int PB200_SetKernelConfig(Estimator* e, int lanesPerRoi, int threadsPerBlock);
/* No counterpart in the reference; diagnostic. Runs the streamed LM launch (the one that host
 * calls use while their ROIs are still being copied in) on device-resident ROIs: with markReady
 * = 1 every ROI block is marked as arrived beforehand, and the results equal PB200_EstimateDevice's;
 * with markReady = 0 none is, so every wait runs out (after about 1-2 s) and the launch ends.
 * Returns 0 (no wait ran out), 1 (a wait ran out; the context stays usable) or -1 on a bad
 * argument. Column-blocked Gaussian estimators without per-spot constants at 2 or 4 lanes per ROI. */
int PB200_StreamedFitProbe(Estimator* e, int numspots, const float* d_sample, float* d_params, int* d_iterations,
                           int markReady);
/* Extension: the host-pointer pipeline of the Estimate/CRLB calls. The ROIs are fitted in chunks of
 * roisPerChunk (0: automatic, which also lets large calls of the flat-background Gaussian models
 * run the streamed path, one fit launch while the ROIs arrive), with `slots` chunks (2..8) in
 * flight: while one chunk is fitted the next ones are copied in and the previous ones copied
 * out. Returns 0 or -1. */
int PB200_SetHostPipeline(Estimator* e, int roisPerChunk, int slots);
/* Lanes per ROI and threads per block the fit kernel of this estimator launches with (for large
 * ROIs the block is smaller than the configured threads per block, so that its groups' shared
 * memory fits). */
void PB200_GetKernelConfig(Estimator* e, int* lanesPerRoi, int* threadsPerBlock);
/* Fit kernel family for the Gaussian models: 0 = column-blocked (default), 1 = generic
 * per-pixel table kernel (the spline model always uses 1). Returns 0 on success. */
int PB200_SetKernelVariant(Estimator* e, int variant);
/* Number of fit-kernel launches issued by this library since load (for launch accounting). */
uint64_t PB200_LaunchCount(void);
/* FP32 FMA-pipe throughput probe (diagnostic): launches blocks x threads threads running
 * 8 independent FMA chains for iters x 16 steps on `stream`; returns the FLOPs issued (time the
 * launch with events) or -1 on a launch error. d_out: device buffer of `blocks` floats. */
double PB200_Fp32ProbeLaunch(int blocks, int threads, int iters, float* d_out, void* stream);
/* Self-check (diagnostic): the float constants sqrt(2 pi), sqrt(2), 1/sqrt(pi) the model set-ups
 * use, and the host-computed fixed-sigma scales 1/(sqrt(2 pi) s), 1/(sqrt(2) s) of the n sigmas
 * h_sigmas, against the device's IEEE square roots and divisions. *mismatches = number of values
 * that differ (0 expected). Returns 0, or -1 on a CUDA error. */
int PB200_CheckModelConstants(int n, const float* h_sigmas, int* mismatches);
/* Model id (0 XYIBg, 1 XYIBgConstSigma, 2 XYIBgSigma, 3 XYIBgSigmaXY, 4 XYZIBg, 5 CSpline) and ROI size. */
int PB200_ModelInfo(Estimator* e, int* roisize);

#ifdef __cplusplus
}
#endif
#endif /* PHOTONPY_B200_H */
