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
// maximum filter there. It writes one candidate bit per pixel (a 32-bit word per tile row, so
// word order is row-major pixel order) and the score only at candidates. Two light launches
// then compact the candidates in pixel order from the bit mask (per-segment popcounts, then
// ordered writes with block scans), and one cuts the ROIs straight into the fitter's input
// layout. HBM traffic: the frames once (plus halos through L2), 1/32 of a frame of mask
// words, and the spots.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/photonpy_b200.h"
#include "host_internal.h"
#include "spot_internal.h"

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

constexpr int kTile = 32;          // output tile edge of the filter kernel (one mask word per tile row)
constexpr int kSegThreads = 256;
constexpr int kWordsPerThread = 32;
constexpr int kSegWords = kSegThreads * kWordsPerThread;  // mask words per compaction segment
constexpr int kMaxWindow = 32;     // largest filter window the fused kernel takes

struct FilterParams {
    const float* frames;  // [n][h][w]
    const float* bg;      // [h][w] or null
    unsigned* mask;       // [n][h][ntx]: bit b of word (y, tx) is pixel (32 tx + b, y)
    float* score;         // [n][h][w]: M, written at candidates only
    int w, h, n, ntx;
    int u1, u2, mf, roisize;
    float minI, maxI;
    // Tile geometry (host-computed). D region: the DH x DW detection-image pixels the maximum
    // filter of the 32 x 32 output tile reads, origin (x0 - mb, y0 - mb); padded to DHp x DWp (a
    // multiple of 4, the register strips). Source region: SHp x SWp, SL pixels further up/left.
    // Shared-memory row strides SWs, DWs are odd, so a warp reading one column across rows hits
    // 32 different banks.
    int mb, DW, DH, DWp, DHp, SL, SWp, SHp, SWs, DWs;
    float invSWp, invDWp, invSHp, invDH;  // float reciprocals for the flat-index splits
    float rcp[kMaxWindow + 1];     // rcp[k] = 1/k rounded to nearest (host IEEE division)
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// floor(i / d) for 0 <= i < 2^20 from inv = 1.0f / d: (i + 0.5) / d is at least 0.5 / d away
// from an integer, far more than the two roundings of the product.
__device__ __forceinline__ int div_small(int i, float inv) { return (int)(((float)i + 0.5f) * inv); }

// x / d rounded to nearest for a small positive integer d, from r = 1/d rounded to nearest:
// q = x r, e = x - q d (exact, by FMA), q + e r (P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990). Zeros (the
// sign), quotients near the subnormal range (the remainder is no longer exact there), infinities
// and NaN take the IEEE division. PB200_CheckCountDivision compares the result bit for bit with
// IEEE division for every float x and every d = 1..32, the counts the box filters divide by.
__device__ __forceinline__ bool count_div_in_range(float q) {
    const float a = fabsf(q);
    return a >= 0x1p-100f && a <= 0x1p+126f;  // false for NaN
}
__device__ __forceinline__ float count_div_corrected(float x, float q, float d, float r) {
    const float e = __fmaf_rn(-q, d, x);
    return __fmaf_rn(e, r, q);
}
__device__ __forceinline__ float pb200_count_div(float x, float d, float r) {
    const float q = __fmul_rn(x, r);
    return count_div_in_range(q) ? count_div_corrected(x, q, d, r) : __fdiv_rn(x, d);
}

// Box filter at global coordinate g of a line of `extent` samples, window [g - win/2, g - win/2 +
// win) clipped to the line: sequential sum from 0 over the window, divided by the clipped count.
// The line holds zeros outside [0, extent), and adding +0 leaves a sum that started at +0
// unchanged (round-to-nearest never produces -0 from it), so the whole window is summed.
// Sample i of the line is line[(i - base) * stride].
__device__ __forceinline__ float box_at(const FilterParams& p, const float* line, int stride, int base, int g,
                                        int extent, int win) {
    const int s = g - win / 2;
    const float* q = line + (s - base) * stride;
    float sum = 0.0f;
    for (int j = 0; j < win; j++) sum = __fadd_rn(sum, q[j * stride]);
    const int cnt = min(s + win, extent) - max(s, 0);
    return pb200_count_div(sum, (float)cnt, p.rcp[cnt]);
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

// Four consecutive outputs of both box filters along a line held in registers: v[k] is sample
// (g0 - U2/2 + k) of the line, outputs at g0..g0+3. Same sums as box_at, in the same order.
template <int U1, int U2>
__device__ __forceinline__ void box_strip(const FilterParams& p, const float (&v)[U2 + 3], int g0, int extent,
                                          float (&o1)[4], float (&o2)[4]) {
    constexpr int off1 = U2 / 2 - U1 / 2;  // the u1 window starts off1 samples into the u2 window
    const bool interior = g0 - U2 / 2 >= 0 && g0 + 3 - U2 / 2 + U2 <= extent;  // u1 windows lie inside
#pragma unroll
    for (int j = 0; j < 4; j++) {
        float s1 = 0.0f, s2 = 0.0f;
#pragma unroll
        for (int k = 0; k < U1; k++) s1 = __fadd_rn(s1, v[j + off1 + k]);
#pragma unroll
        for (int k = 0; k < U2; k++) s2 = __fadd_rn(s2, v[j + k]);
        int c1 = U1, c2 = U2;
        if (!interior) {
            const int g = g0 + j;
            c1 = min(g - U1 / 2 + U1, extent) - max(g - U1 / 2, 0);
            c2 = min(g - U2 / 2 + U2, extent) - max(g - U2 / 2, 0);
            c1 = clampi(c1, 1, kMaxWindow);  // outside the line the value is unused
            c2 = clampi(c2, 1, kMaxWindow);
        }
        o1[j] = pb200_count_div(s1, (float)c1, p.rcp[c1]);
        o2[j] = pb200_count_div(s2, (float)c2, p.rcp[c2]);
    }
}

constexpr int kMXs = kTile + 1;  // row stride of the max filter's X-pass buffer (odd: no bank conflicts)

__host__ __device__ constexpr int floor_log2(int v) { return v <= 1 ? 0 : 1 + floor_log2(v / 2); }

// Sliding maximum over MF samples for four consecutive outputs, o[j] = max(v[j .. j + MF)), by a
// doubling table: after level k, L[i] = max(v[i .. i + 2^k)); the output joins two overlapping
// power-of-two windows. Max is only associative without NaN and -0, so this runs on tiles
// whose detection image holds neither (there it equals the reference's left-to-right fold).
template <int MF>
__device__ __forceinline__ void max_strip(const float (&v)[MF + 3], float (&o)[4]) {
    constexpr int K = floor_log2(MF);
    float L[MF + 3];
#pragma unroll
    for (int i = 0; i < MF + 3; i++) L[i] = v[i];
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int span = 1 << k;
#pragma unroll
        for (int i = 0; i < MF + 4 - 2 * span; i++) L[i] = fmaxf(L[i], L[i + span]);
    }
    constexpr int rem = MF - (1 << K);
#pragma unroll
    for (int j = 0; j < 4; j++) o[j] = fmaxf(L[j], L[j + rem]);
}

// Maximum filter (X pass, then Y pass), local-maximum test and mask/score writes for a tile
// whose D region holds -inf outside the image. Strips of four outputs in registers; 256 threads.
template <int MF>
__device__ __forceinline__ void max_phases_fast(const FilterParams& p, const float* D, float* MX, int f, int x0,
                                                int y0, int Dy0) {
    const int tid = threadIdx.x;
    // X pass: MX[r][c] = max(D[r][c .. c + MF)) for the DH rows and 32 tile columns; lanes walk
    // down the rows of one 4-column strip
    for (int i = tid; i < (kTile / 4) * p.DH; i += blockDim.x) {
        const int st = div_small(i, p.invDH), r = i - st * p.DH;
        const int gy = Dy0 + r;
        float o[4] = {-INFINITY, -INFINITY, -INFINITY, -INFINITY};
        if (gy >= 0 && gy < p.h) {
            float v[MF + 3];
            const float* src = D + r * p.DWs + 4 * st;
#pragma unroll
            for (int k = 0; k < MF + 3; k++) v[k] = src[k];
            max_strip<MF>(v, o);
        }
#pragma unroll
        for (int j = 0; j < 4; j++) MX[r * kMXs + 4 * st + j] = o[j];
    }
    __syncthreads();
    // Y pass and test: warp w takes tile rows 4w .. 4w + 3, lane = tile column
    const int lane = tid & 31, warp = tid >> 5;
    float v[MF + 3], o[4];
#pragma unroll
    for (int k = 0; k < MF + 3; k++) v[k] = MX[(4 * warp + k) * kMXs + lane];
    max_strip<MF>(v, o);
    const int half = p.roisize / 2, rest = p.roisize - p.roisize / 2;
    const int gx = x0 + lane;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        const int r = 4 * warp + j, gy = y0 + r;
        if (gy >= p.h) break;  // uniform across the warp
        bool cand = false;
        if (gx < p.w) {
            const float a = D[(r + p.mb) * p.DWs + lane + p.mb];
            const bool isMax = a == o[j] && gx > half && gy > half && gx + rest < p.w - 1 && gy + rest < p.h - 1;
            cand = isMax && o[j] > p.minI && o[j] < p.maxI;
        }
        const unsigned bits = __ballot_sync(0xffffffffu, cand);
        const size_t row = (size_t)f * p.h + gy;
        if (lane == 0) p.mask[row * p.ntx + blockIdx.x] = bits;
        if (cand) p.score[row * p.w + gx] = o[j];
    }
}

// Runs max_phases_fast<MF> when p.mf is in [MF, MFHI]; false when it is not.
template <int MF, int MFHI>
__device__ __forceinline__ bool max_phases_dispatch(const FilterParams& p, const float* D, float* MX, int f, int x0,
                                                    int y0, int Dy0) {
    if constexpr (MF > MFHI) {
        return false;
    } else {
        if (p.mf == MF) {
            max_phases_fast<MF>(p, D, MX, f, x0, y0, Dy0);
            return true;
        }
        return max_phases_dispatch<MF + 1, MFHI>(p, D, MX, f, x0, y0, Dy0);
    }
}

// The fused filter. U1 > 0: both box windows fixed at compile time (U2 = 2 U1), each thread
// computes strips of four outputs from registers, and for the maximum-filter sizes photonpy
// pairs with that box size (maxFilterSize = int(5 sigma) for uniformFilter1Size = int(2 sigma +
// 2)) the maximum filter runs from registers too, on tiles free of NaN and -0. U1 == 0, or any
// other case: one output per thread per pass, left-to-right fold. 256 threads per block.
template <int U1>
__global__ void __launch_bounds__(256) detect_filter_kernel(const FilterParams p) {
    constexpr int U2 = 2 * U1;
    extern __shared__ float sm[];
    const int f = blockIdx.z;
    const int x0 = blockIdx.x * kTile, y0 = blockIdx.y * kTile;
    const int Dx0 = x0 - p.mb, Dy0 = y0 - p.mb;    // D region origin (global)
    const int Sx0 = Dx0 - p.SL, Sy0 = Dy0 - p.SL;  // source region origin (global)
    float* S = sm;                                 // [SHp][SWs] source minus background, 0 outside
    float* X1 = S + p.SHp * p.SWs;                 // [SHp][DWs] X pass of u1, 0 outside
    float* X2 = X1 + p.SHp * p.DWs;                // [SHp][DWs] X pass of u2, 0 outside
    float* D = X2 + p.SHp * p.DWs;                 // [DHp][DWs] detection image
    float* MX = X1;                                // [DH][kMXs] X pass of the max filter (X1 reused)
    const float* frame = p.frames + (size_t)f * p.w * p.h;
    const int tid = threadIdx.x, nth = blockDim.x;

    // A: source region
    for (int i = tid; i < p.SHp * p.SWp; i += nth) {
        const int r = div_small(i, p.invSWp), c = i - r * p.SWp;
        const int gy = Sy0 + r, gx = Sx0 + c;
        float v = 0.0f;
        if (gx >= 0 && gx < p.w && gy >= 0 && gy < p.h) {
            v = __ldg(frame + (size_t)gy * p.w + gx);
            if (p.bg) v = __fsub_rn(v, __ldg(p.bg + (size_t)gy * p.w + gx));
        }
        S[r * p.SWs + c] = v;
    }
    __syncthreads();
    bool odd = false;  // NaN or -0 in this tile's detection image
    if constexpr (U1 > 0) {
        // B: X passes, strips of 4 columns; lanes walk down the rows of one strip
        const int nstrip = p.DWp >> 2;
        for (int i = tid; i < p.SHp * nstrip; i += nth) {
            const int st = div_small(i, p.invSHp), r = i - st * p.SHp;
            const int gy = Sy0 + r, gx0 = Dx0 + 4 * st;
            const float* src = S + r * p.SWs + 4 * st;  // sample gx0 - U2/2 (SL = U2/2)
            float v[U2 + 3];
#pragma unroll
            for (int k = 0; k < U2 + 3; k++) v[k] = src[k];
            float o1[4], o2[4];
            box_strip<U1, U2>(p, v, gx0, p.w, o1, o2);
            const bool rowIn = gy >= 0 && gy < p.h;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const bool in = rowIn && gx0 + j >= 0 && gx0 + j < p.w;
                X1[r * p.DWs + 4 * st + j] = in ? o1[j] : 0.0f;
                X2[r * p.DWs + 4 * st + j] = in ? o2[j] : 0.0f;
            }
        }
        __syncthreads();
        // C: Y passes and the difference, strips of 4 rows; lanes walk along the columns
        for (int i = tid; i < p.DWp * (p.DHp >> 2); i += nth) {
            const int st = div_small(i, p.invDWp), c = i - st * p.DWp;
            const int gx = Dx0 + c, gy0 = Dy0 + 4 * st;
            float v[U2 + 3], o1[4], o2[4], t1[4], t2[4];
            // X1 column: row (4 st + k) of X is sample gy0 - U2/2 + k
#pragma unroll
            for (int k = 0; k < U2 + 3; k++) v[k] = X1[(4 * st + k) * p.DWs + c];
            box_strip<U1, U2>(p, v, gy0, p.h, o1, t2);
#pragma unroll
            for (int k = 0; k < U2 + 3; k++) v[k] = X2[(4 * st + k) * p.DWs + c];
            box_strip<U1, U2>(p, v, gy0, p.h, t1, o2);
            const bool colIn = gx >= 0 && gx < p.w;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int gy = gy0 + j;
                float d = -INFINITY;  // padding for the maximum filter
                if (colIn && gy >= 0 && gy < p.h) {
                    d = __fsub_rn(o1[j], o2[j]);
                    odd |= d != d || __float_as_uint(d) == 0x80000000u;
                }
                D[(4 * st + j) * p.DWs + c] = d;
            }
        }
    } else {
        // B: X passes of both box filters over every source row, for the D-region columns
        for (int i = tid; i < p.SHp * p.DWp; i += nth) {
            const int r = div_small(i, p.invDWp), c = i - r * p.DWp;
            const int gy = Sy0 + r, gx = Dx0 + c;
            float a = 0.0f, b = 0.0f;
            if (gx >= 0 && gx < p.w && gy >= 0 && gy < p.h) {
                const float* line = S + r * p.SWs;
                a = box_at(p, line, 1, Sx0, gx, p.w, p.u1);
                b = box_at(p, line, 1, Sx0, gx, p.w, p.u2);
            }
            X1[r * p.DWs + c] = a;
            X2[r * p.DWs + c] = b;
        }
        __syncthreads();
        // C: Y passes and the difference over the D region
        for (int i = tid; i < p.DHp * p.DWp; i += nth) {
            const int r = div_small(i, p.invDWp), c = i - r * p.DWp;
            const int gy = Dy0 + r, gx = Dx0 + c;
            if (gx < 0 || gx >= p.w || gy < 0 || gy >= p.h) continue;
            const float a = box_at(p, X1 + c, p.DWs, Sy0, gy, p.h, p.u1);
            const float b = box_at(p, X2 + c, p.DWs, Sy0, gy, p.h, p.u2);
            D[r * p.DWs + c] = __fsub_rn(a, b);
        }
    }
    if constexpr (U1 > 0) {
        constexpr int MFLO = (5 * (U1 - 2)) / 2 < 1 ? 1 : (5 * (U1 - 2)) / 2;
        constexpr int MFHI = (5 * (U1 - 1)) / 2 + 1;
        if (!__syncthreads_or(odd) && max_phases_dispatch<MFLO, MFHI>(p, D, MX, f, x0, y0, Dy0)) return;
    } else {
        __syncthreads();
    }
    // D: X pass of the maximum filter over the D-region rows, for the tile columns
    for (int i = tid; i < p.DH * kTile; i += nth) {
        const int r = i >> 5, c = i & 31;
        const int gy = Dy0 + r, gx = x0 + c;
        if (gx >= p.w || gy < 0 || gy >= p.h) continue;
        MX[r * kMXs + c] = max_at(D + r * p.DWs, 1, Dx0, gx, p.w, p.mf);
    }
    __syncthreads();
    // E: Y pass, local-maximum test; one warp per tile row writes that row's mask word
    const int half = p.roisize / 2, rest = p.roisize - p.roisize / 2;
    const int lane = tid & 31;
    for (int r = tid >> 5; r < kTile; r += nth >> 5) {
        const int gy = y0 + r, gx = x0 + lane;
        if (gy >= p.h) break;  // uniform across the warp
        bool cand = false;
        float b = 0.0f;
        if (gx < p.w) {
            b = max_at(MX + lane, kMXs, Dy0, gy, p.h, p.mf);
            const float a = D[(gy - Dy0) * p.DWs + (gx - Dx0)];
            const bool isMax = a == b && gx > half && gy > half && gx + rest < p.w - 1 && gy + rest < p.h - 1;
            cand = isMax && b > p.minI && b < p.maxI;
        }
        const unsigned bits = __ballot_sync(0xffffffffu, cand);
        const size_t row = (size_t)f * p.h + gy;
        if (lane == 0) p.mask[row * p.ntx + blockIdx.x] = bits;
        if (cand) p.score[row * p.w + gx] = b;
    }
}

// Candidates per segment of kSegWords mask words of each frame.
__global__ void __launch_bounds__(kSegThreads) detect_count_kernel(const unsigned* __restrict__ mask, int nw,
                                                                   int nseg, int* __restrict__ counts) {
    const int f = blockIdx.y, seg = blockIdx.x;
    const unsigned* m = mask + (size_t)f * nw;
    int c = 0;
    for (int k = 0; k < kWordsPerThread; k++) {
        const int i = seg * kSegWords + k * kSegThreads + threadIdx.x;
        if (i < nw) c += __popc(__ldg(m + i));
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

// Ordered write: thread t owns words [seg*kSegWords + t*kWordsPerThread, +kWordsPerThread), so a
// block scan of the per-thread counts gives row-major ranks. The first maxSpots spots of a frame
// are written; segment 0 also writes the frame's total.
__global__ void __launch_bounds__(kSegThreads) detect_emit_kernel(const unsigned* __restrict__ mask,
                                                                  const float* __restrict__ score, int w, int ntx,
                                                                  int nw, int nseg, const int* __restrict__ counts,
                                                                  int maxSpots, int* __restrict__ found,
                                                                  int* __restrict__ index,
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
    const unsigned* m = mask + (size_t)f * nw;
    const int w0 = seg * kSegWords + threadIdx.x * kWordsPerThread;
    int c = 0;
    for (int k = 0; k < kWordsPerThread; k++)
        if (w0 + k < nw) c += __popc(__ldg(m + w0 + k));
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
    if (c == 0) return;
    const float* sf = score + (size_t)f * (nw / ntx) * w;  // nw = h * ntx
    for (int k = 0; k < kWordsPerThread && r < maxSpots; k++) {
        const int wi = w0 + k;
        if (wi >= nw) break;
        unsigned bits = __ldg(m + wi);
        if (!bits) continue;
        const int y = wi / ntx, tx = wi - y * ntx;
        while (bits && r < maxSpots) {
            const int b = __ffs(bits) - 1;
            bits &= bits - 1;
            const int pix = y * w + tx * kTile + b;
            index[(size_t)f * maxSpots + r] = pix;
            scoreOut[(size_t)f * maxSpots + r] = sf[pix];
            r++;
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

// Every float x (bit patterns base .. base + count) divided by d both ways; counts the results
// whose bits differ (NaN vs NaN counts as equal) and keeps the last differing x.
__global__ void count_div_check_kernel(float d, float r, unsigned long long* mismatches, unsigned* lastBad) {
    const unsigned stride = gridDim.x * blockDim.x;
    unsigned long long bad = 0;
    for (unsigned long long u = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; u < (1ULL << 32);
         u += stride) {
        const float x = __uint_as_float((unsigned)u);
        const float a = pb200_count_div(x, d, r), b = __fdiv_rn(x, d);
        const bool same = __float_as_uint(a) == __float_as_uint(b) || (a != a && b != b);
        if (!same) {
            bad++;
            *lastBad = (unsigned)u;
        }
    }
    if (bad) atomicAdd(mismatches, bad);
}

// Device buffers of the detector come from a small process-wide cache, so a factory per
// ProcessFrame call (photonpy's usage) costs no cudaMalloc/cudaFree once warm. A buffer goes back
// to the cache only when no kernel uses it any more (its owner has synchronised).
class BufferCache {
   public:
    static BufferCache& get() {
        static BufferCache* c = new BufferCache();  // never destroyed: no CUDA calls at exit
        return *c;
    }
    void* take(size_t n, size_t* got) {
        int dev = 0;
        PBS_CUDA(cudaGetDevice(&dev));
        {
            std::lock_guard<std::mutex> g(mtx_);
            for (size_t i = 0; i < blocks_.size(); i++) {
                Block b = blocks_[i];
                if (b.dev == dev && b.bytes >= n && b.bytes <= 2 * n + (1 << 20)) {
                    blocks_.erase(blocks_.begin() + (long)i);
                    held_ -= b.bytes;
                    *got = b.bytes;
                    return b.p;
                }
            }
        }
        void* p = nullptr;
        PBS_CUDA(cudaMalloc(&p, n));
        *got = n;
        return p;
    }
    void give(void* p, size_t n) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) return;
        std::lock_guard<std::mutex> g(mtx_);
        if (held_ + n > kMaxHeld || blocks_.size() >= 32) {
            cudaFree(p);
            return;
        }
        blocks_.push_back(Block{p, n, dev});
        held_ += n;
    }

   private:
    struct Block {
        void* p;
        size_t bytes;
        int dev;
    };
    static constexpr size_t kMaxHeld = size_t(1) << 30;
    std::mutex mtx_;
    std::vector<Block> blocks_;
    size_t held_ = 0;
};

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t n) {
        if (n <= bytes) return;
        release();
        p = BufferCache::get().take(n < 256 ? 256 : n, &bytes);
    }
    void release() {
        if (p) BufferCache::get().give(p, bytes);
        p = nullptr;
        bytes = 0;
    }
    ~DevMem() { release(); }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace

// The detector configuration (SpotDetectorConfig, SpotDetector.h:39-62), the device buffers of
// its standalone per-frame calls, and the detection scratch (mask, sparse scores, segment
// counts, spot indices) that every call on this factory reuses. `scratchDone` is recorded after
// each call's last kernel; the next call's stream waits on it, so calls on different streams
// never share the scratch at the same time.
struct SpotDetectorFactory {
    SpotDetectorConfig cfg;
    std::mutex mtx;
    DevMem frame, calibFrame, bg, found, scoreOut, corner, rois;  // ProcessFrame
    DevMem mask, score, counts, index, scoreTmp;          // scratch of every call
    cudaEvent_t scratchDone = nullptr;
    ~SpotDetectorFactory() {
        if (scratchDone) {
            cudaEventSynchronize(scratchDone);
            cudaEventDestroy(scratchDone);
        }
    }
};

namespace {

void check_config(const SpotDetectorConfig& c) {
    if (c.uniformFilter1Size < 1 || c.uniformFilter2Size < 1 || c.maxFilterSize < 1)
        throw SpotError("SpotDetector: filter sizes must be positive");
    if (c.uniformFilter1Size > kMaxWindow || c.uniformFilter2Size > kMaxWindow || c.maxFilterSize > kMaxWindow)
        throw SpotError("SpotDetector: filter sizes above " + std::to_string(kMaxWindow) + " are not provided");
    if (c.roisize < 1) throw SpotError("SpotDetector: roisize must be positive");
}

void fill_reciprocals(float* rcp) {
    rcp[0] = 0.0f;
    for (int k = 1; k <= kMaxWindow; k++) rcp[k] = 1.0f / (float)k;  // IEEE single division
}

// The register-strip instantiations cover photonpy's own sizes (u2 = 2 u1, from
// uniformFilter1Size = int(2 sigma + 2)) for sigma up to 3.5 px; anything else runs the generic
// kernel.
const void* filter_kernel_for(int u1, int u2) {
    if (u2 == 2 * u1) {
        switch (u1) {
            case 2: return (const void*)detect_filter_kernel<2>;
            case 3: return (const void*)detect_filter_kernel<3>;
            case 4: return (const void*)detect_filter_kernel<4>;
            case 5: return (const void*)detect_filter_kernel<5>;
            case 6: return (const void*)detect_filter_kernel<6>;
            case 7: return (const void*)detect_filter_kernel<7>;
            case 8: return (const void*)detect_filter_kernel<8>;
            case 9: return (const void*)detect_filter_kernel<9>;
            default: break;
        }
    }
    return (const void*)detect_filter_kernel<0>;
}

// Runs the four kernels for `n` frames already on the device, on stream s, with the factory's
// scratch; the caller holds sdf->mtx. Outputs: found[n], scoreOut[n][maxSpots] (optional),
// indexOut[n][maxSpots] (optional; pixel indices), and (when rois is set) corner[n][maxSpots][2]
// + rois[n][maxSpots][roisize][roisize], cut from d_cutFrames (d_frames when null).
void detect_run(SpotDetectorFactory* sdf, const float* d_frames, const float* d_bg, int n, int w, int h, int roisize,
                int maxSpots, int* d_found, float* d_scoreOut, int* d_corner, float* d_rois, cudaStream_t s,
                int* d_indexOut = nullptr, const float* d_cutFrames = nullptr) {
    const SpotDetectorConfig& c = sdf->cfg;
    check_config(c);
    if (n > 65535) throw SpotError("spot detection: at most 65535 frames per call");
    if ((long long)w * h >= (1LL << 31)) throw SpotError("spot detection: frame too large");
    const int ntx = (w + kTile - 1) / kTile;
    const int nw = h * ntx, nseg = (nw + kSegWords - 1) / kSegWords;
    const size_t npix = (size_t)w * h;
    // grow the scratch only after the previous call's kernels are done with it
    const size_t need[5] = {sizeof(unsigned) * nw * n, sizeof(float) * npix * n, sizeof(int) * (size_t)nseg * n,
                            d_indexOut ? 0 : sizeof(int) * (size_t)maxSpots * n,
                            d_scoreOut ? 0 : sizeof(float) * (size_t)maxSpots * n};
    DevMem* bufs[5] = {&sdf->mask, &sdf->score, &sdf->counts, &sdf->index, &sdf->scoreTmp};
    bool grow = false;
    for (int i = 0; i < 5; i++) grow |= need[i] > bufs[i]->bytes;
    if (!sdf->scratchDone) PBS_CUDA(cudaEventCreateWithFlags(&sdf->scratchDone, cudaEventDisableTiming));
    if (grow) {
        PBS_CUDA(cudaEventSynchronize(sdf->scratchDone));
        for (int i = 0; i < 5; i++) bufs[i]->ensure(need[i]);
    }
    PBS_CUDA(cudaStreamWaitEvent(s, sdf->scratchDone, 0));
    float* scoreOut = d_scoreOut ? d_scoreOut : sdf->scoreTmp.as<float>();
    int* index = d_indexOut ? d_indexOut : sdf->index.as<int>();

    FilterParams p{};
    p.frames = d_frames;
    p.bg = d_bg;
    p.mask = sdf->mask.as<unsigned>();
    p.score = sdf->score.as<float>();
    p.w = w;
    p.h = h;
    p.n = n;
    p.ntx = ntx;
    p.u1 = c.uniformFilter1Size;
    p.u2 = c.uniformFilter2Size;
    p.mf = c.maxFilterSize;
    p.roisize = c.roisize;
    p.minI = c.minIntensity;
    p.maxI = c.maxIntensity;
    p.mb = p.mf / 2;
    p.DW = kTile + p.mf - 1;
    p.DH = p.DW;
    p.DWp = (p.DW + 3) & ~3;
    p.DHp = p.DWp;
    const int SLmax = std::max(p.u1 / 2, p.u2 / 2);
    const int SRmax = std::max(p.u1 - p.u1 / 2 - 1, p.u2 - p.u2 / 2 - 1);
    p.SL = SLmax;
    p.SWp = p.DWp + SLmax + SRmax;
    p.SHp = p.SWp;
    p.SWs = p.SWp | 1;
    p.DWs = p.DWp | 1;
    p.invSWp = 1.0f / (float)p.SWp;
    p.invDWp = 1.0f / (float)p.DWp;
    p.invSHp = 1.0f / (float)p.SHp;
    p.invDH = 1.0f / (float)p.DH;
    fill_reciprocals(p.rcp);
    const size_t smem =
        sizeof(float) * ((size_t)p.SHp * p.SWs + 2 * (size_t)p.SHp * p.DWs + (size_t)p.DHp * p.DWs);
    const void* kern = filter_kernel_for(p.u1, p.u2);
    if (smem > 48 * 1024)
        PBS_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid(ntx, (h + kTile - 1) / kTile, n);
    void* args[] = {&p};
    PBS_CUDA(cudaLaunchKernel(kern, grid, dim3(256), args, smem, s));
    PBS_CUDA(cudaGetLastError());
    detect_count_kernel<<<dim3(nseg, n), kSegThreads, 0, s>>>(p.mask, nw, nseg, sdf->counts.as<int>());
    PBS_CUDA(cudaGetLastError());
    detect_emit_kernel<<<dim3(nseg, n), kSegThreads, 0, s>>>(p.mask, p.score, w, ntx, nw, nseg,
                                                             sdf->counts.as<int>(), maxSpots, d_found, index,
                                                             scoreOut);
    PBS_CUDA(cudaGetLastError());
    if (d_rois) {
        const long long tasks = (long long)n * maxSpots;
        const int blocks = (int)std::min<long long>((tasks + 7) / 8, 1 << 30);
        cut_rois_kernel<<<blocks, 256, 0, s>>>(d_cutFrames ? d_cutFrames : d_frames, w, h, roisize, maxSpots, n,
                                               d_found, index, d_corner, d_rois);
        PBS_CUDA(cudaGetLastError());
    }
    PBS_CUDA(cudaEventRecord(sdf->scratchDone, s));
}

}  // namespace

const SpotDetectorConfig* pb200::spot_factory_config(const SpotDetectorFactory* sdf) { return &sdf->cfg; }

void pb200::spot_detect_indices(SpotDetectorFactory* sdf, const float* d_frames, const float* d_bg, int n, int w,
                                int h, int maxSpots, int* d_found, int* d_index, float* d_score, cudaStream_t s) {
    std::lock_guard<std::mutex> g(sdf->mtx);
    detect_run(sdf, d_frames, d_bg, n, w, h, sdf->cfg.roisize, maxSpots, d_found, d_score, nullptr, nullptr, s,
               d_index);
}

namespace {

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
            std::lock_guard<std::mutex> g(sdf->mtx);
            const size_t npix = (size_t)width * height;
            const int cap = std::max(maxSpots, 1);
            sdf->frame.ensure(sizeof(float) * npix);
            sdf->found.ensure(sizeof(int));
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
            // with a camera calibration the detector sees the calibrated frame, while the ROIs are
            // cut from the frame as given (SpotDetector.cu:104-106, 141)
            const float* d_det = sdf->frame.as<float>();
            if (calib) {
                sdf->calibFrame.ensure(sizeof(float) * npix);
                pb200::camera_calib_apply_f32(static_cast<const CameraCalibration*>(calib), sdf->frame.as<float>(),
                                              sdf->calibFrame.as<float>(), width, height, 1, 0);
                d_det = sdf->calibFrame.as<float>();
            }
            // the reference cuts ROIs of the ProcessFrame call's own roisize, but tests the border
            // with the configuration's
            detect_run(sdf, d_det, d_bg, 1, width, height, roisize, cap, sdf->found.as<int>(),
                       sdf->scoreOut.as<float>(), sdf->corner.as<int>(), sdf->rois.as<float>(), 0, nullptr,
                       sdf->frame.as<float>());
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
            std::lock_guard<std::mutex> g(sdf->mtx);
            detect_run(sdf, d_frames, d_bg, nframes, width, height, roisize, maxSpotsPerFrame, d_found, d_scores,
                       d_cornerYX, d_rois, (cudaStream_t)stream);
            return 0;
        },
        -1);
}

int PB200_CheckCountDivision(int maxCount, unsigned long long* mismatches, unsigned* lastBadBits) {
    return spot_guarded(
        [&]() -> int {
            if (maxCount < 1 || maxCount > kMaxWindow || !mismatches)
                throw SpotError("PB200_CheckCountDivision: bad arguments");
            float rcp[kMaxWindow + 1];
            fill_reciprocals(rcp);
            DevMem dm;
            dm.ensure(sizeof(unsigned long long) * (kMaxWindow + 1) + sizeof(unsigned) * (kMaxWindow + 1));
            auto* d_bad = dm.as<unsigned long long>();
            auto* d_last = reinterpret_cast<unsigned*>(d_bad + kMaxWindow + 1);
            PBS_CUDA(cudaMemset(dm.p, 0, dm.bytes));
            int dev = 0, sms = 0;
            PBS_CUDA(cudaGetDevice(&dev));
            PBS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
            for (int k = 1; k <= maxCount; k++) {
                count_div_check_kernel<<<sms * 8, 256>>>((float)k, rcp[k], d_bad + k, d_last + k);
                PBS_CUDA(cudaGetLastError());
            }
            unsigned long long hb[kMaxWindow + 1];
            unsigned hl[kMaxWindow + 1];
            PBS_CUDA(cudaMemcpy(hb, d_bad, sizeof(hb), cudaMemcpyDeviceToHost));
            PBS_CUDA(cudaMemcpy(hl, d_last, sizeof(hl), cudaMemcpyDeviceToHost));
            for (int k = 1; k <= maxCount; k++) {
                mismatches[k - 1] = hb[k];
                if (lastBadBits) lastBadBits[k - 1] = hl[k];
            }
            return 0;
        },
        -1);
}

}  // extern "C"
