// Spot detection and ROI extraction: the ROI source upstream of the fitter.
//
// Replaces photonpy's SpotDetection/SpotDetector.cu (SpotDetector::Detect :49-84,
// SpotDetector_ProcessFrame :101-151, ExtractROIs :155-178) and the image filters it uses
// (ImageFilters.h:6-105). Same arithmetic, so the same spots, scores and ROIs:
//   D = box(src - bg, u1) - box(src - bg, u2)          box: X pass then Y pass, window
//                                                      [c - win/2, c - win/2 + win) clipped to
//                                                      the image, sequential float sum / count
//   M = max(D, maxFilterSize)                          X pass then Y pass, clipped windows
//   spot at (x, y) when D == M, the ROI fits (x > roisize/2, y > roisize/2,
//   x + roisize - roisize/2 < w - 1, same for y) and minIntensity < M < maxIntensity;
//   spots in row-major pixel order, score M, ROI corner (y, x) - roisize/2 with clamped pixels.
//
// B200 layout. The reference runs six full-frame filter launches through global memory and a
// cub partition per frame. Here one launch filters a batch of frames: each block loads a tile
// plus its halo into shared memory once and computes both box filters, the difference and the
// maximum filter there, writing one score per pixel (the candidate's M, or -inf). Two light
// launches then compact the candidates in pixel order (per-segment counts, then ordered
// writes with block scans), and one cuts the ROIs straight into the fitter's input layout.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/photonpy_b200.h"
#include "host_internal.h"

namespace {

struct SpotError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define PBS_CUDA(call)                                                                              \
    do {                                                                                            \
        cudaError_t err_ = (call);                                                                  \
        if (err_ != cudaSuccess)                                                                    \
            throw SpotError(std::string("CUDA error: ") + cudaGetErrorString(err_) + " in " #call); \
    } while (0)

constexpr int kTile = 32;        // output tile edge of the filter kernel
constexpr int kSeg = 4096;       // pixels per compaction segment
constexpr int kSegThreads = 256;
constexpr int kPerThread = kSeg / kSegThreads;
constexpr int kMaxWindow = 32;   // largest filter window the fused kernel takes

struct FilterParams {
    const float* frames;  // [n][h][w]
    const float* bg;      // [h][w] or null
    float* score;         // [n][h][w]: M at candidates, -inf elsewhere
    int w, h, n;
    int u1, u2, mf, roisize;
    float minI, maxI;
    // tile geometry (host-computed): D region [DW x DH] around the TxT output tile, source
    // region [SW x SH] around the D region
    int mb, DW, DH, SL, SW, SH;
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Box filter at global coordinate g of a line of `extent` samples, window clipped to the line;
// sample i of the line is line[(i - base) * stride].
__device__ __forceinline__ float box_at(const float* line, int stride, int base, int g, int extent, int win) {
    int s = g - win / 2;
    int e = s + win;
    if (s < 0) s = 0;
    if (e > extent) e = extent;
    float sum = 0.0f;
    for (int i = s; i < e; i++) sum = __fadd_rn(sum, line[(i - base) * stride]);
    return __fdiv_rn(sum, (float)(e - s));
}

__device__ __forceinline__ float max_at(const float* line, int stride, int base, int g, int extent, int win) {
    int s = g - win / 2;
    int e = s + win;
    if (s < 0) s = 0;
    if (e > extent) e = extent;
    float v = line[(s - base) * stride];
    for (int i = s + 1; i < e; i++) {
        const float b = line[(i - base) * stride];
        v = v < b ? b : v;  // thrust::maximum
    }
    return v;
}

__global__ void __launch_bounds__(256) detect_filter_kernel(const FilterParams p) {
    extern __shared__ float sm[];
    const int f = blockIdx.z;
    const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile;
    const int Dx0 = x0 - p.mb, Dy0 = y0 - p.mb;  // D region origin (global)
    const int Sx0 = Dx0 - p.SL, Sy0 = Dy0 - p.SL;  // source region origin (global)
    float* S = sm;                                // [SH][SW] source minus background
    float* X1 = S + p.SH * p.SW;                  // [SH][DW] X pass of u1
    float* X2 = X1 + p.SH * p.DW;                 // [SH][DW] X pass of u2
    float* D = X2 + p.SH * p.DW;                  // [DH][DW] detection image
    float* MX = X1;                               // [DH][kTile] X pass of the max filter (X1 reused)
    const float* frame = p.frames + (size_t)f * p.w * p.h;
    const int tid = threadIdx.x, nth = blockDim.x;

    // A: source region (pixels outside the image are never read by the clipped windows)
    for (int i = tid; i < p.SH * p.SW; i += nth) {
        const int gy = Sy0 + i / p.SW, gx = Sx0 + i % p.SW;
        float v = 0.0f;
        if (gx >= 0 && gx < p.w && gy >= 0 && gy < p.h) {
            v = __ldg(frame + (size_t)gy * p.w + gx);
            if (p.bg) v = __fsub_rn(v, __ldg(p.bg + (size_t)gy * p.w + gx));
        }
        S[i] = v;
    }
    __syncthreads();
    // B: X passes of both box filters over every source row, for the D-region columns
    for (int i = tid; i < p.SH * p.DW; i += nth) {
        const int r = i / p.DW, c = i % p.DW;
        const int gy = Sy0 + r, gx = Dx0 + c;
        if (gx < 0 || gx >= p.w || gy < 0 || gy >= p.h) continue;
        const float* line = S + r * p.SW;
        X1[i] = box_at(line, 1, Sx0, gx, p.w, p.u1);
        X2[i] = box_at(line, 1, Sx0, gx, p.w, p.u2);
    }
    __syncthreads();
    // C: Y passes and the difference over the D region
    for (int i = tid; i < p.DH * p.DW; i += nth) {
        const int r = i / p.DW, c = i % p.DW;
        const int gy = Dy0 + r, gx = Dx0 + c;
        if (gx < 0 || gx >= p.w || gy < 0 || gy >= p.h) continue;
        const float a = box_at(X1 + c, p.DW, Sy0, gy, p.h, p.u1);
        const float b = box_at(X2 + c, p.DW, Sy0, gy, p.h, p.u2);
        D[i] = __fsub_rn(a, b);
    }
    __syncthreads();
    // D: X pass of the maximum filter over the D-region rows, for the tile columns
    for (int i = tid; i < p.DH * kTile; i += nth) {
        const int r = i / kTile, c = i % kTile;
        const int gy = Dy0 + r, gx = x0 + c;
        if (gx >= p.w || gy < 0 || gy >= p.h) continue;
        MX[i] = max_at(D + r * p.DW, 1, Dx0, gx, p.w, p.mf);
    }
    __syncthreads();
    // E: Y pass, local-maximum test, score map
    const int half = p.roisize / 2, rest = p.roisize - p.roisize / 2;
    for (int i = tid; i < kTile * kTile; i += nth) {
        const int r = i / kTile, c = i % kTile;
        const int gy = y0 + r, gx = x0 + c;
        if (gx >= p.w || gy >= p.h) continue;
        const float b = max_at(MX + c, kTile, Dy0, gy, p.h, p.mf);
        const float a = D[(gy - Dy0) * p.DW + (gx - Dx0)];
        const bool isMax = a == b && gx > half && gy > half && gx + rest < p.w - 1 && gy + rest < p.h - 1;
        const bool cand = isMax && b > p.minI && b < p.maxI;
        p.score[(size_t)f * p.w * p.h + (size_t)gy * p.w + gx] = cand ? b : -INFINITY;
    }
}

// Candidates per segment of kSeg pixels of each frame.
__global__ void __launch_bounds__(kSegThreads) detect_count_kernel(const float* __restrict__ score, int npix,
                                                                   int nseg, int* __restrict__ counts) {
    const int f = blockIdx.y, seg = blockIdx.x;
    const float* s = score + (size_t)f * npix;
    int c = 0;
    for (int k = 0; k < kPerThread; k++) {
        const int p = seg * kSeg + k * kSegThreads + threadIdx.x;
        if (p < npix && s[p] > -INFINITY) c++;
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    __shared__ int wsum[kSegThreads / 32];
    if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int i = 0; i < kSegThreads / 32; i++) t += wsum[i];
        counts[(size_t)f * nseg + seg] = t;
    }
}

// Ordered write: thread t owns pixels [seg*kSeg + t*kPerThread, +kPerThread), so a block scan of
// the per-thread counts gives row-major ranks. The first maxSpots spots of a frame are written;
// segment 0 also writes the frame's total.
__global__ void __launch_bounds__(kSegThreads) detect_emit_kernel(const float* __restrict__ score, int npix, int nseg,
                                                                  const int* __restrict__ counts, int maxSpots,
                                                                  int* __restrict__ found, int* __restrict__ index,
                                                                  float* __restrict__ scoreOut) {
    const int f = blockIdx.y, seg = blockIdx.x;
    const int* cf = counts + (size_t)f * nseg;
    __shared__ int offset;
    __shared__ int wsum[kSegThreads / 32];
    if (threadIdx.x == 0) {
        int o = 0, t = 0;
        for (int i = 0; i < nseg; i++) {
            if (i < seg) o += cf[i];
            t += cf[i];
        }
        offset = o;
        if (seg == 0) found[f] = t;
    }
    __syncthreads();
    if (offset >= maxSpots) return;  // uniform across the block
    const float* s = score + (size_t)f * npix;
    const int p0 = seg * kSeg + threadIdx.x * kPerThread;
    int c = 0;
    for (int k = 0; k < kPerThread; k++) {
        const int p = p0 + k;
        if (p < npix && s[p] > -INFINITY) c++;
    }
    // exclusive block scan of c
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int incl = c;
    for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int before = 0;
    for (int i = 0; i < warp; i++) before += wsum[i];
    int r = offset + before + incl - c;
    for (int k = 0; k < kPerThread && r < maxSpots; k++) {
        const int p = p0 + k;
        if (p < npix) {
            const float v = s[p];
            if (v > -INFINITY) {
                index[(size_t)f * maxSpots + r] = p;
                scoreOut[(size_t)f * maxSpots + r] = v;
                r++;
            }
        }
    }
}

// One warp per spot: corner (y, x) - roisize/2 and the clamped ROI pixels of the original frame.
__global__ void __launch_bounds__(256) cut_rois_kernel(const float* __restrict__ frames, int w, int h, int roisize,
                                                       int maxSpots, int nframes, const int* __restrict__ found,
                                                       const int* __restrict__ index, int* __restrict__ cornerYX,
                                                       float* __restrict__ rois) {
    const int warpsPerBlock = blockDim.x / 32;
    const long long task = (long long)blockIdx.x * warpsPerBlock + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (task >= (long long)nframes * maxSpots) return;
    const int f = (int)(task / maxSpots), i = (int)(task % maxSpots);
    if (i >= min(found[f], maxSpots)) return;
    const int p = index[(size_t)f * maxSpots + i];
    const int cy = p / w - roisize / 2, cx = p % w - roisize / 2;
    if (lane == 0) {
        cornerYX[((size_t)f * maxSpots + i) * 2] = cy;
        cornerYX[((size_t)f * maxSpots + i) * 2 + 1] = cx;
    }
    const float* frame = frames + (size_t)f * w * h;
    float* out = rois + ((size_t)f * maxSpots + i) * roisize * roisize;
    for (int q = lane; q < roisize * roisize; q += 32) {
        const int fy = clampi(cy + q / roisize, 0, h - 1), fx = clampi(cx + q % roisize, 0, w - 1);
        out[q] = __ldg(frame + (size_t)fy * w + fx);
    }
}

// ExtractROIs: 3D boxes [roiZ][roiY][roiX] at corners (z, y, x) of a frame stack, clamped.
__global__ void extract_rois_kernel(const float* __restrict__ frames, int w, int h, int depth, int rx, int ry, int rz,
                                    const int* __restrict__ start, int n, float* __restrict__ rois) {
    const size_t per = (size_t)rx * ry * rz;
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < per * n; t += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(t / per);
        const int q = (int)(t % per);
        const int z = q / (rx * ry), y = (q / rx) % ry, x = q % rx;
        const int fz = clampi(start[3 * i] + z, 0, depth - 1);
        const int fy = clampi(start[3 * i + 1] + y, 0, h - 1);
        const int fx = clampi(start[3 * i + 2] + x, 0, w - 1);
        // the reference reads frame z (not fz) of the stack: frames[z*w*h + fy*w + fx]
        (void)fz;
        rois[t] = __ldg(frames + (size_t)z * w * h + (size_t)fy * w + fx);
    }
}

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t n) {
        if (n <= bytes) return;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        PBS_CUDA(cudaMalloc(&p, n < 256 ? 256 : n));
        bytes = n < 256 ? 256 : n;
    }
    ~DevMem() {
        if (p) cudaFree(p);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace

// The detector configuration (SpotDetectorConfig, SpotDetector.h:39-62) and the device buffers
// of its standalone per-frame calls.
struct SpotDetectorFactory {
    SpotDetectorConfig cfg;
    std::mutex mtx;
    DevMem frame, bg, score, counts, found, index, scoreOut, corner, rois;
};

namespace {

void check_config(const SpotDetectorConfig& c) {
    if (c.uniformFilter1Size < 1 || c.uniformFilter2Size < 1 || c.maxFilterSize < 1)
        throw SpotError("SpotDetector: filter sizes must be positive");
    if (c.uniformFilter1Size > kMaxWindow || c.uniformFilter2Size > kMaxWindow || c.maxFilterSize > kMaxWindow)
        throw SpotError("SpotDetector: filter sizes above " + std::to_string(kMaxWindow) + " are not provided");
    if (c.roisize < 1) throw SpotError("SpotDetector: roisize must be positive");
}

// Runs the four kernels for `n` frames already on the device. Outputs: found[n],
// index/score[n][maxSpots], and (when rois is set) corner[n][maxSpots][2] + rois.
void detect_device(const SpotDetectorConfig& c, const float* d_frames, const float* d_bg, int n, int w, int h,
                   int roisize, int maxSpots, float* d_score, int* d_counts, int* d_found, int* d_index,
                   float* d_scoreOut, int* d_corner, float* d_rois, cudaStream_t s) {
    check_config(c);
    if (n > 65535) throw SpotError("spot detection: at most 65535 frames per call");
    FilterParams p{};
    p.frames = d_frames;
    p.bg = d_bg;
    p.score = d_score;
    p.w = w;
    p.h = h;
    p.n = n;
    p.u1 = c.uniformFilter1Size;
    p.u2 = c.uniformFilter2Size;
    p.mf = c.maxFilterSize;
    p.roisize = c.roisize;
    p.minI = c.minIntensity;
    p.maxI = c.maxIntensity;
    p.mb = p.mf / 2;
    p.DW = kTile + p.mf - 1;
    p.DH = p.DW;
    const int SLmax = std::max(p.u1 / 2, p.u2 / 2);
    const int SRmax = std::max(p.u1 - p.u1 / 2 - 1, p.u2 - p.u2 / 2 - 1);
    p.SL = SLmax;
    p.SW = p.DW + SLmax + SRmax;
    p.SH = p.SW;
    const size_t smem = sizeof(float) * ((size_t)p.SH * p.SW + 2 * (size_t)p.SH * p.DW + (size_t)p.DH * p.DW);
    if (smem > 48 * 1024)
        PBS_CUDA(cudaFuncSetAttribute(detect_filter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((w + kTile - 1) / kTile, (h + kTile - 1) / kTile, n);
    detect_filter_kernel<<<grid, 256, smem, s>>>(p);
    PBS_CUDA(cudaGetLastError());
    const int npix = w * h, nseg = (npix + kSeg - 1) / kSeg;
    detect_count_kernel<<<dim3(nseg, n), kSegThreads, 0, s>>>(d_score, npix, nseg, d_counts);
    PBS_CUDA(cudaGetLastError());
    detect_emit_kernel<<<dim3(nseg, n), kSegThreads, 0, s>>>(d_score, npix, nseg, d_counts, maxSpots, d_found,
                                                             d_index, d_scoreOut);
    PBS_CUDA(cudaGetLastError());
    if (d_rois) {
        const long long tasks = (long long)n * maxSpots;
        if (tasks > 0) {
            const int blocks = (int)std::min<long long>((tasks + 7) / 8, 1 << 30);
            cut_rois_kernel<<<blocks, 256, 0, s>>>(d_frames, w, h, roisize, maxSpots, n, d_found, d_index, d_corner,
                                                   d_rois);
            PBS_CUDA(cudaGetLastError());
        }
    }
}

template <class F, class R>
R spot_guarded(F&& f, R fallback) {
    try {
        return f();
    } catch (const std::exception& e) {
        pb200::set_last_error(e.what());
        return fallback;
    }
}

}  // namespace

extern "C" {

SpotDetectorFactory* SpotDetector_Configure(const SpotDetectorConfig* config) {
    return spot_guarded(
        [&]() -> SpotDetectorFactory* {
            if (!config) throw SpotError("SpotDetector_Configure: config is null");
            auto* f = new SpotDetectorFactory();
            f->cfg = *config;
            return f;
        },
        (SpotDetectorFactory*)nullptr);
}

void SpotDetector_DestroyFactory(SpotDetectorFactory* factory) { delete factory; }

int SpotDetector_ProcessFrame(const float* frame, int width, int height, int roisize, int maxSpots, float* spotScores,
                              int* spotZ, int* cornerPosYX, float* rois, SpotDetectorFactory* sdf, void* calib) {
    return spot_guarded(
        [&]() -> int {
            if (!frame || !sdf || width <= 0 || height <= 0 || maxSpots < 0 || roisize < 1)
                throw SpotError("SpotDetector_ProcessFrame: bad arguments");
            if (calib) throw SpotError("SpotDetector_ProcessFrame: camera calibration is not provided by photonpy_b200");
            std::lock_guard<std::mutex> g(sdf->mtx);
            const size_t npix = (size_t)width * height;
            const int nseg = (int)((npix + kSeg - 1) / kSeg);
            const int cap = std::max(maxSpots, 1);
            sdf->frame.ensure(sizeof(float) * npix);
            sdf->score.ensure(sizeof(float) * npix);
            sdf->counts.ensure(sizeof(int) * nseg);
            sdf->found.ensure(sizeof(int));
            sdf->index.ensure(sizeof(int) * cap);
            sdf->scoreOut.ensure(sizeof(float) * cap);
            sdf->corner.ensure(sizeof(int) * 2 * cap);
            sdf->rois.ensure(sizeof(float) * (size_t)cap * roisize * roisize);
            PBS_CUDA(cudaMemcpy(sdf->frame.p, frame, sizeof(float) * npix, cudaMemcpyHostToDevice));
            const float* d_bg = nullptr;
            if (sdf->cfg.backgroundImage) {  // the host image the configuration points at
                sdf->bg.ensure(sizeof(float) * npix);
                PBS_CUDA(cudaMemcpy(sdf->bg.p, sdf->cfg.backgroundImage, sizeof(float) * npix, cudaMemcpyHostToDevice));
                d_bg = sdf->bg.as<float>();
            }
            // the reference cuts ROIs of the ProcessFrame call's own roisize, but tests the border
            // with the configuration's
            detect_device(sdf->cfg, sdf->frame.as<float>(), d_bg, 1, width, height, roisize, cap,
                          sdf->score.as<float>(), sdf->counts.as<int>(), sdf->found.as<int>(), sdf->index.as<int>(),
                          sdf->scoreOut.as<float>(), sdf->corner.as<int>(), sdf->rois.as<float>(), 0);
            int found = 0;
            PBS_CUDA(cudaMemcpy(&found, sdf->found.p, sizeof(int), cudaMemcpyDeviceToHost));
            const int n = std::min(found, maxSpots);
            if (n > 0) {
                if (spotScores)
                    PBS_CUDA(cudaMemcpy(spotScores, sdf->scoreOut.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
                if (cornerPosYX)
                    PBS_CUDA(cudaMemcpy(cornerPosYX, sdf->corner.p, sizeof(int) * 2 * n, cudaMemcpyDeviceToHost));
                if (rois)
                    PBS_CUDA(cudaMemcpy(rois, sdf->rois.p, sizeof(float) * (size_t)n * roisize * roisize,
                                        cudaMemcpyDeviceToHost));
                if (spotZ) std::fill(spotZ, spotZ + n, 0);
            }
            return n;
        },
        0);
}

void ExtractROIs(const float* frames, int width, int height, int depth, int roiX, int roiY, int roiZ,
                 const int* startposZYX, int numspots, float* rois) {
    spot_guarded(
        [&]() -> int {
            if (numspots <= 0) return 0;
            if (!frames || !startposZYX || !rois || width <= 0 || height <= 0 || depth <= 0 || roiX <= 0 ||
                roiY <= 0 || roiZ <= 0)
                throw SpotError("ExtractROIs: bad arguments");
            if (roiZ > depth) throw SpotError("ExtractROIs: roiZ exceeds the stack depth");
            DevMem df, ds, dr;
            const size_t nfr = (size_t)width * height * depth;
            const size_t nout = (size_t)roiX * roiY * roiZ * numspots;
            df.ensure(sizeof(float) * nfr);
            ds.ensure(sizeof(int) * 3 * numspots);
            dr.ensure(sizeof(float) * nout);
            PBS_CUDA(cudaMemcpy(df.p, frames, sizeof(float) * nfr, cudaMemcpyHostToDevice));
            PBS_CUDA(cudaMemcpy(ds.p, startposZYX, sizeof(int) * 3 * numspots, cudaMemcpyHostToDevice));
            const int blocks = (int)std::min<size_t>((nout + 255) / 256, 65535 * 8);
            extract_rois_kernel<<<blocks, 256>>>(df.as<float>(), width, height, depth, roiX, roiY, roiZ, ds.as<int>(),
                                                 numspots, dr.as<float>());
            PBS_CUDA(cudaGetLastError());
            PBS_CUDA(cudaMemcpy(rois, dr.p, sizeof(float) * nout, cudaMemcpyDeviceToHost));
            return 0;
        },
        0);
}

int PB200_DetectSpotsDevice(SpotDetectorFactory* sdf, const float* d_frames, const float* d_bg, int nframes,
                            int width, int height, int roisize, int maxSpotsPerFrame, int* d_found, int* d_cornerYX,
                            float* d_scores, float* d_rois, void* stream) {
    return spot_guarded(
        [&]() -> int {
            if (!sdf || !d_frames || !d_found || nframes < 0 || width <= 0 || height <= 0 || maxSpotsPerFrame < 1 ||
                roisize < 1 || (d_rois && !d_cornerYX))
                throw SpotError("PB200_DetectSpotsDevice: bad arguments");
            if (nframes == 0) return 0;
            const cudaStream_t s = (cudaStream_t)stream;
            const size_t npix = (size_t)width * height;
            const int nseg = (int)((npix + kSeg - 1) / kSeg);
            // stream-ordered scratch: score map, segment counts, spot indices (and scores when the
            // caller passes none)
            float* score = nullptr;
            int* counts = nullptr;
            int* index = nullptr;
            float* scoreTmp = nullptr;
            PBS_CUDA(cudaMallocAsync((void**)&score, sizeof(float) * npix * nframes, s));
            PBS_CUDA(cudaMallocAsync((void**)&counts, sizeof(int) * (size_t)nseg * nframes, s));
            PBS_CUDA(cudaMallocAsync((void**)&index, sizeof(int) * (size_t)maxSpotsPerFrame * nframes, s));
            if (!d_scores) PBS_CUDA(cudaMallocAsync((void**)&scoreTmp, sizeof(float) * (size_t)maxSpotsPerFrame * nframes, s));
            try {
                detect_device(sdf->cfg, d_frames, d_bg, nframes, width, height, roisize, maxSpotsPerFrame, score,
                              counts, d_found, index, d_scores ? d_scores : scoreTmp, d_cornerYX, d_rois, s);
            } catch (...) {
                cudaFreeAsync(score, s);
                cudaFreeAsync(counts, s);
                cudaFreeAsync(index, s);
                if (scoreTmp) cudaFreeAsync(scoreTmp, s);
                throw;
            }
            PBS_CUDA(cudaFreeAsync(score, s));
            PBS_CUDA(cudaFreeAsync(counts, s));
            PBS_CUDA(cudaFreeAsync(index, s));
            if (scoreTmp) PBS_CUDA(cudaFreeAsync(scoreTmp, s));
            return 0;
        },
        -1);
}

}  // extern "C"
