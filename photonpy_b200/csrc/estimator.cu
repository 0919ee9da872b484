// C ABI of the photonpy_b200 estimator: estimator objects, context, host<->device staging,
// kernel dispatch and the spline-coefficient kernels.
//
// Replaces (paths inside photonpy's cpp/SMLMLib):
//   Estimators/Estimator.cpp:45-157         Estimator_* C API
//   Estimators/EstimatorImpl.cu:225-300     cuEstimatorWrapper (host pointers -> device)
//   Estimators/EstimatorImpl.h:58-105       cuPSFImpl kernels (one thread per ROI)
//   Estimators/Gaussian/GaussianPSF.cu      Gauss2D_CreatePSF_* factories and exported limits
//   Estimators/CSpline/CubicSplinePSF.cu    CSpline_CreatePSF / _FromFile / _Compute / _Evaluate
//   Context.cpp, StringUtils.cpp, CudaUtils.cu, DebugImageCallback.cpp (loader-time exports)
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "../../include/photonpy_b200.h"
#include "host_internal.h"
#include "launch.cuh"
#include "mixed.cuh"

using namespace pb200;

// ------------------------------------------------------------------------------------
// errors and debug output
// ------------------------------------------------------------------------------------
namespace {
thread_local std::string t_lastError;
int (*g_debugPrint)(const char*) = nullptr;
void (*g_debugImage)(int, int, int, const float*, const char*) = nullptr;
std::atomic<uint64_t> g_launches{0};

void debug_printf(const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (g_debugPrint) g_debugPrint(buf);
    else fputs(buf, stderr);
}

void report(const std::exception& e) {
    t_lastError = e.what();
    debug_printf("%s\n", e.what());
}

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define PB_CUDA(call)                                                                                  \
    do {                                                                                               \
        cudaError_t err_ = (call);                                                                     \
        if (err_ != cudaSuccess)                                                                       \
            throw Error(std::string("CUDA error: ") + cudaGetErrorString(err_) + " in " #call);       \
    } while (0)

// ------------------------------------------------------------------------------------
// device buffers
// ------------------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    int device = -1;
    void ensure(size_t nbytes) {
        if (nbytes <= bytes) return;
        release();
        size_t want = nbytes < 256 ? 256 : nbytes;
        PB_CUDA(cudaGetDevice(&device));
        PB_CUDA(cudaMalloc(&p, want));
        bytes = want;
    }
    void release() {
        if (p) {
            int cur = -1;
            cudaGetDevice(&cur);
            if (device >= 0 && device != cur) cudaSetDevice(device);
            cudaFree(p);
            if (device >= 0 && device != cur) cudaSetDevice(cur);
        }
        p = nullptr;
        bytes = 0;
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
    ~DevBuf() { release(); }
};


}  // namespace

namespace pb200 {
int num_sms() {
    static int sms[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (!sms[dev]) {
        cudaDeviceProp prop;
        PB_CUDA(cudaGetDeviceProperties(&prop, dev));
        sms[dev] = prop.multiProcessorCount;
    }
    return sms[dev];
}

void count_launch() { g_launches++; }

// Streamed LM launcher (host calls whose ROIs arrive during the launch), or null.
StreamLaunch stream_launcher_for(int model, int G, int CPL) {
    switch (model) {
    case MODEL_XYIBG: return stream_launcher_xyibg(G, CPL);
    case MODEL_XYIBG_CONSTSIGMA: return stream_launcher_constsigma(G, CPL);
    case MODEL_XYIBG_SIGMA: return stream_launcher_sigma(G, CPL);
    case MODEL_XYIBG_SIGMAXY: return stream_launcher_sigmaxy(G, CPL);
    case MODEL_XYZIBG: return stream_launcher_astig(G, CPL);
    }
    return nullptr;
}

FitLaunch fit_launcher_for(int model, int G, int CPL, int variant) {
    switch (model) {
    case MODEL_XYIBG: return fit_launcher_xyibg(G, CPL, variant);
    case MODEL_XYIBG_CONSTSIGMA: return fit_launcher_constsigma(G, CPL, variant);
    case MODEL_XYIBG_SIGMA: return fit_launcher_sigma(G, CPL, variant);
    case MODEL_XYIBG_SIGMAXY: return fit_launcher_sigmaxy(G, CPL, variant);
    case MODEL_XYZIBG: return fit_launcher_astig(G, CPL, variant);
    case MODEL_CSPLINE: return fit_launcher_spline(G, CPL, variant);
    case MODEL_XYITILTEDBG: return fit_launcher_tilted(G, CPL, variant);
    case MODEL_XYITILTEDBG_SIGMAXY: return fit_launcher_tilted_sxy(G, CPL, variant);
    case MODEL_INTENSITYBG: return fit_launcher_intensity_bg(G);
    case MODEL_CSPLINE_TILTED: return fit_launcher_spline_tilted(G);
    case MODEL_CSPLINE_BGIMAGE: return fit_launcher_spline_bgimage(G);
    }
    throw Error("unknown model");
}

AdjointLaunch adjoint_launcher_for(int model) {
    switch (model) {
    case MODEL_XYIBG: return adjoint_launcher_xyibg();
    case MODEL_XYIBG_CONSTSIGMA: return adjoint_launcher_constsigma();
    case MODEL_XYIBG_SIGMA: return adjoint_launcher_sigma();
    case MODEL_XYIBG_SIGMAXY: return adjoint_launcher_sigmaxy();
    case MODEL_XYZIBG: return adjoint_launcher_astig();
    case MODEL_CSPLINE: return adjoint_launcher_spline();
    case MODEL_XYITILTEDBG:
    case MODEL_XYITILTEDBG_SIGMAXY:
    case MODEL_CSPLINE_TILTED:
    case MODEL_CSPLINE_BGIMAGE:
        throw Error("PoissonNLLAdjoint: provided for the flat-background models only");
    }
    throw Error("unknown model");
}

EvalLaunch eval_launcher_for(int model, int G) {
    switch (model) {
    case MODEL_XYIBG: return eval_launcher_xyibg(G);
    case MODEL_XYIBG_CONSTSIGMA: return eval_launcher_constsigma(G);
    case MODEL_XYIBG_SIGMA: return eval_launcher_sigma(G);
    case MODEL_XYIBG_SIGMAXY: return eval_launcher_sigmaxy(G);
    case MODEL_XYZIBG: return eval_launcher_astig(G);
    case MODEL_CSPLINE: return eval_launcher_spline(G);
    case MODEL_XYITILTEDBG: return eval_launcher_tilted(G);
    case MODEL_XYITILTEDBG_SIGMAXY: return eval_launcher_tilted_sxy(G);
    case MODEL_CSPLINE_TILTED: return eval_launcher_spline_tilted(G);
    case MODEL_CSPLINE_BGIMAGE: return eval_launcher_spline_bgimage(G);
    }
    throw Error("unknown model");
}
}  // namespace pb200

namespace {

// Lanes per ROI when no tuned value is set: enough ROIs per warp to amortise the redundant
// K x K solve for small ROIs, enough lanes to keep per-lane pixel loops short for large ones.
// Flat-background Gaussians of 7..10 pixels: 2 lanes per ROI with 4 or 5 columns each (16 ROIs
// per warp in the column-blocked kernel).
bool gauss_two_lanes(int model, int R) { return model <= MODEL_XYZIBG && R >= 7 && R <= 10; }

int default_lanes(int model, int R) {
    if (model_is_spline(model)) return R * R <= 100 ? 8 : 16;
    if (gauss_two_lanes(model, R)) return 2;
    if (R <= 16) return 4;
    if (R <= 32) return 8;
    return 16;
}

// Lanes per ROI and columns per lane of the column-blocked kernel at its default configuration
// (a flat-background Gaussian; the shape Estimator::fit_shape gives without a configuration).
void gauss_default_shape(int model, int R, int& G, int& cpl) {
    G = default_lanes(model, R);
    while (G < 32 && (R + G - 1) / G > gauss_max_cpl(G)) G *= 2;
    cpl = (R + G - 1) / G;
}

}  // namespace

// ------------------------------------------------------------------------------------
// Context and Estimator objects
// ------------------------------------------------------------------------------------
struct Estimator;

struct Context {
    std::mutex mtx;
    std::unordered_set<Estimator*> objects;
    // queues and other non-estimator objects, in registration order (destroyed newest first:
    // a frame queue goes before the ROI queue it fills)
    std::vector<std::pair<void*, void (*)(void*)>> owned;
};

namespace pb200 {
void context_attach(Context* ctx, void* obj, void (*destroy)(void*)) {
    if (!ctx) return;
    std::lock_guard<std::mutex> g(ctx->mtx);
    for (auto& o : ctx->owned)
        if (o.first == obj) {
            o.second = destroy;
            return;
        }
    ctx->owned.push_back({obj, destroy});
}

void context_detach(Context* ctx, void* obj) {
    if (!ctx) return;
    std::lock_guard<std::mutex> g(ctx->mtx);
    for (size_t i = 0; i < ctx->owned.size(); i++)
        if (ctx->owned[i].first == obj) {
            ctx->owned.erase(ctx->owned.begin() + (long)i);
            return;
        }
}

void set_last_error(const std::string& msg) {
    t_lastError = msg;
    debug_printf("%s\n", msg.c_str());
}
}  // namespace pb200

struct Slot {
    cudaStream_t stream = nullptr;
    DevBuf smp, consts, initial, params, iters, trace, crlb, chisq, fisher, glrt;
    DevBuf claim;  // ROI counter of the slot's LM launches
    // copied: the slot's inputs have arrived (recorded on the copy stream); freed: its launches
    // have read them, so the copy stream may refill them (recorded on the slot's stream)
    cudaEvent_t copied = nullptr, freed = nullptr;
};

struct Estimator {
    ModelDesc desc{};
    int K = 0, numconst = 0;
    std::string format;
    std::vector<ParamLimit> limits;
    LMParams lm{30, 1e-15f, 0.0f};  // C++ default of the reference (Estimator.cpp:24)
    Context* ctx = nullptr;
    DevBuf coefs, coefsQ;  // spline coefficients: reference layout and the q-major copy
    int lanes = 0, threads = 0;  // 0: automatic
    int variant = 0;  // 0: column-blocked Gaussian kernel, 1: generic table kernel
    int device = 0;
    // Likelihood-ratio test estimator (GLRT_CreatePSF): diagnostics = {ll_on, ll_off, mean} per spot.
    bool glrt = false;
    bool glrtRefMean = false;  // every spot's mean from the call's first ROI, as the reference
    DevBuf glrtRoi0;
    bool crlbAbs = false;  // CRLB = sqrt(|diag of the inverse|) (the intensity/background fit)
    std::mutex mtx;
    // host-pointer pipeline: ROIs per chunk (0: automatic) and slots (chunks in flight, 2..4)
    int hostChunk = 0;
    static constexpr int kMaxSlots = 8;
    int hostSlots = 4;
    Slot slots[kMaxSlots];
    cudaStream_t copyStream = nullptr;  // the pipeline's host-to-device copies, in chunk order
    // streamed host calls: buffers of a whole call, the ready flags and a pinned block of ones
    // from which the copy stream sets them
    DevBuf stSmp, stConsts, stInitial, stParams, stIters, stCrlb, stChisq, stFisher, stFlags, stClaim;
    int* hostOnes = nullptr;
    int hostOnesCount = 0;
    // 0: not yet known; 1: the streamed path; -1: the slot pipeline (chosen after the first
    // streamed call from how long its fits ran on after the last copy in)
    int streamPref = 0;
    cudaEvent_t stCopyStart = nullptr, stCopyEnd = nullptr, stLmEnd = nullptr;

    Estimator() { PB_CUDA(cudaGetDevice(&device)); }
    ~Estimator() {
        for (auto& s : slots) {
            if (s.stream) cudaStreamDestroy(s.stream);
            if (s.copied) cudaEventDestroy(s.copied);
            if (s.freed) cudaEventDestroy(s.freed);
        }
        if (copyStream) cudaStreamDestroy(copyStream);
        if (hostOnes) cudaFreeHost(hostOnes);
        for (cudaEvent_t ev : {stCopyStart, stCopyEnd, stLmEnd})
            if (ev) cudaEventDestroy(ev);
    }
    int lanes_for() const { return lanes ? lanes : default_lanes(desc.model, desc.roisize); }
    // Lanes per ROI and columns per lane of the fit kernel this configuration launches (cpl 0:
    // the generic table kernel, which starts at 4 lanes).
    void fit_shape(int& G, int& cpl) const {
        G = lanes_for();
        cpl = 0;
        const int R = desc.roisize;
        if (desc.model <= MODEL_XYZIBG && variant == 0) {  // column-blocked kernel: flat-background Gaussians
            while (G < 32 && (R + G - 1) / G > gauss_max_cpl(G)) G *= 2;
            const int c = (R + G - 1) / G;
            if (c <= gauss_max_cpl(G)) {
                cpl = c;
                return;
            }
        }
        if (G < 4) G = 4;
    }
    // Threads per block: 128 for the 2-lane column-blocked kernel (measured faster than 64..256
    // on 10x10 ROIs), 256 for the others.
    int threads_for() const {
        if (threads) return threads;
        int G, cpl;
        fit_shape(G, cpl);
        return (cpl && G == 2) ? 128 : 256;
    }
    // Shared-memory floats per group of the fit kernel this configuration launches.
    int group_stride_floats() const {
        int G, cpl;
        fit_shape(G, cpl);
        const int R = desc.roisize;
        if (cpl) {
            switch (K) {
            case 4: return gauss_group_stride<4>(R, G, cpl);
            case 5: return gauss_group_stride<5>(R, G, cpl);
            default: return gauss_group_stride<6>(R, G, cpl);
            }
        }
        switch (desc.model) {
        case MODEL_XYIBG: return group_smem_floats<GaussModel<MODEL_XYIBG>>(R);
        case MODEL_XYIBG_CONSTSIGMA: return group_smem_floats<GaussModel<MODEL_XYIBG_CONSTSIGMA>>(R);
        case MODEL_XYIBG_SIGMA: return group_smem_floats<GaussModel<MODEL_XYIBG_SIGMA>>(R);
        case MODEL_XYIBG_SIGMAXY: return group_smem_floats<GaussModel<MODEL_XYIBG_SIGMAXY>>(R);
        case MODEL_XYZIBG: return group_smem_floats<GaussModel<MODEL_XYZIBG>>(R);
        case MODEL_XYITILTEDBG: return group_smem_floats<TiltedGaussModel<MODEL_XYITILTEDBG>>(R);
        case MODEL_XYITILTEDBG_SIGMAXY: return group_smem_floats<TiltedGaussModel<MODEL_XYITILTEDBG_SIGMAXY>>(R);
        case MODEL_INTENSITYBG: return group_smem_floats<IntensityBgModel>(R);
        case MODEL_CSPLINE_TILTED: return group_smem_floats<SplineModelT<1>>(R);
        case MODEL_CSPLINE_BGIMAGE: return group_smem_floats<SplineModelT<2>>(R);
        default: return group_smem_floats<SplineModelT<0>>(R);
        }
    }
    // Threads per block the fit kernel actually launches with: threads_for(), halved where the
    // groups of a block would need more shared memory than a block may have (large ROIs).
    int launched_threads_for() const {
        int G, cpl;
        fit_shape(G, cpl);
        return launched_threads(threads_for(), G, group_stride_floats());
    }
    // Fit launcher for this estimator's model, ROI size and kernel configuration.
    FitLaunch fit_launch() const {
        int G, cpl;
        fit_shape(G, cpl);
        return fit_launcher_for(desc.model, G, cpl, cpl ? 0 : 1);
    }
    int npix() const { return desc.roisize * desc.roisize; }
    Slot& slot(int i) {
        Slot& s = slots[i];
        if (!s.stream) PB_CUDA(cudaStreamCreateWithFlags(&s.stream, cudaStreamNonBlocking));
        if (!s.copied) PB_CUDA(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming));
        if (!s.freed) PB_CUDA(cudaEventCreateWithFlags(&s.freed, cudaEventDisableTiming));
        return s;
    }
    cudaStream_t copy_stream() {
        if (!copyStream) PB_CUDA(cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking));
        return copyStream;
    }
};

namespace {

void attach(Estimator* e, Context* ctx) {
    if (!ctx) return;
    std::lock_guard<std::mutex> g(ctx->mtx);
    ctx->objects.insert(e);
    e->ctx = ctx;
}

void detach(Estimator* e) {
    if (!e->ctx) return;
    std::lock_guard<std::mutex> g(e->ctx->mtx);
    e->ctx->objects.erase(e);
    e->ctx = nullptr;
}

Estimator* make_gauss(int model, int roisize, float s0, float s1, const float* ax, const float* ay, float minz,
                      float maxz, Context* ctx) {
    if (roisize < 3 || roisize > 64) throw Error("roisize must be in [3, 64]");
    auto* e = new Estimator();
    e->desc.model = model;
    e->desc.roisize = roisize;
    e->desc.sigma[0] = s0;
    e->desc.sigma[1] = s1;
    for (int i = 0; i < 5; i++) {
        e->desc.astig_x[i] = ax ? ax[i] : 0.0f;
        e->desc.astig_y[i] = ay ? ay[i] : 0.0f;
    }
    e->desc.minz = minz;
    e->desc.maxz = maxz;
    if (model == MODEL_XYIBG) model_desc_fixed_sigma(e->desc);
    e->K = model_num_params(model);
    e->numconst = model_num_consts(model);
    // Exported limits (GaussianPSF.cu:42-48, 92-97, 115-120, 141-147, 168-175).
    const float border = 1.5f;
    const float xyhi = (float)(roisize - 1) - border;
    switch (model) {
    case MODEL_XYIBG:
    case MODEL_XYIBG_CONSTSIGMA:
        e->format = "x,y,I,bg";
        e->limits = {{border, xyhi}, {border, xyhi}, {10.0f, 1e9f}, {1e-6f, 1e9f}};
        break;
    case MODEL_XYIBG_SIGMA:
        e->format = "x,y,\tI,bg,sigma";  // the reference's format string has this tab
        e->limits = {{border, xyhi}, {border, xyhi}, {10.0f, 1e9f}, {1e-6f, 1e9f}, {1.0f, roisize * 2.0f}};
        break;
    case MODEL_XYIBG_SIGMAXY:
        e->format = "x,y,I,bg,sx,sy";
        e->limits = {{border, xyhi}, {border, xyhi}, {10.0f, 1e9f}, {1e-6f, 1e9f},
                     {1.0f, roisize * 2.0f}, {1.0f, roisize * 2.0f}};
        break;
    case MODEL_XYZIBG:
        e->format = "x,y,z,I,bg";
        e->limits = {{border, xyhi}, {border, xyhi}, {minz, maxz}, {10.0f, 1e9f}, {1e-6f, 1e9f}};
        break;
    case MODEL_XYITILTEDBG:  // GaussianPSF.cu:67-74
        e->format = "x,y,I,bg,bgx,bgy";
        e->limits = {{border, xyhi}, {border, xyhi}, {10.0f, 1e9f}, {1e-6f, 1e9f}, {-1e9f, 1e9f}, {-1e9f, 1e9f}};
        break;
    case MODEL_XYITILTEDBG_SIGMAXY:  // GaussianPSF.cu:193-202
        e->format = "x,y,I,bg,bgx,bgy,sx,sy";
        e->limits = {{border, xyhi}, {border, xyhi}, {10.0f, 1e9f}, {1e-6f, 1e9f}, {-1e9f, 1e9f}, {-1e9f, 1e9f},
                     {1.0f, roisize * 2.0f}, {1.0f, roisize * 2.0f}};
        break;
    }
    attach(e, ctx);
    return e;
}

struct Chunking {
    int chunk;
};

// The LM fit, then, when CRLB or GLRT values are requested, the Fisher pass at the fitted
// parameters as a launch of its own (the model launchers in launch.cuh split a request into an
// LM launch and a FIT_CRLB_ONLY launch, each with a kernel instance compiled for that pass).
// The fit kernel could run the Fisher pass itself as a ROI's last trip, but then the groups of a
// warp that are still iterating wait for it and the LM code carries its registers: for 1M
// SigmaXY ROIs of 16x16 that fused form took 31.9 ms, the split 27.3 ms, and the single-pass
// instances 24.4 ms, with the same results bit for bit. The Fisher launch reads the samples once
// more from HBM.
void launch_fit_fisher(Estimator* e, const FitArgs& a, cudaStream_t s) { e->fit_launch()(e->desc, a, e->threads_for(), s); }

// Host-pointer fit through the slot pipeline. The host-to-device copies of all chunks go, in
// chunk order, to one copy stream, so that the copy engines deliver the chunk needed next at
// full bandwidth instead of sharing it with the copies of later chunks (with a copy stream per
// slot the end-to-end time of 1M 16x16 ROIs varied between 25.5 and 28.6 ms from one chunking
// to the next). Chunk c's launches and result copies run on the stream of slot c % slots after
// its inputs have arrived; the copy stream refills a slot once that slot's launches have read
// their inputs.
// h_fisher (with FIT_CRLB_ONLY): the packed FP32 Fisher rows [n][K(K+1)/2 + 1] themselves are
// copied out instead of (or besides) being inverted.
// Largest call (bytes of samples) the streamed path takes; larger calls run through the slots.
constexpr long long kStreamedMaxBytes = 4LL << 30;

// Streamed host-pointer fit of the column-blocked Gaussian kernel: ONE LM launch for the whole
// call, started before the ROIs have arrived. The copy stream copies the per-spot constants and
// start values, then the samples in chunks (in order; after each chunk it sets the ready flag of
// each of its 1024-ROI blocks from pinned host memory, a copy-engine write that needs no SM),
// and the launch's groups wait for the block of each ROI they claim (wait_stream_ready, bounded
// to 1-2 s, after which the call reports an error).
// So the fits run while the ROIs arrive without the end of a launch at every chunk, which in
// the slot pipeline left the GPU mostly idle for about 0.18 ms per chunk. Then the Fisher
// launch, the FP64 CRLB and the copies out. Same kernels and arguments per ROI as the other
// paths: the results are identical.
void host_fit_streamed_body(Estimator* e, StreamLaunch streamLaunch, int n, const float* h_smp,
                            const float* h_consts, const float* h_initial, float* h_params, int* h_iters,
                            float* h_crlb, float* h_chisq, cudaStream_t cs, Slot& ks);

void host_fit_streamed(Estimator* e, StreamLaunch streamLaunch, int n, const float* h_smp, const float* h_consts,
                       const float* h_initial, float* h_params, int* h_iters, float* h_crlb, float* h_chisq) {
    const cudaStream_t cs = e->copy_stream();
    Slot& ks = e->slot(0);
    try {
        host_fit_streamed_body(e, streamLaunch, n, h_smp, h_consts, h_initial, h_params, h_iters, h_crlb, h_chisq, cs,
                               ks);
    } catch (...) {
        // a launch that is still waiting for ROIs ends by its bounded wait; let it end before the
        // buffers and flags are used again
        cudaStreamSynchronize(cs);
        cudaStreamSynchronize(ks.stream);
        throw;
    }
}

void host_fit_streamed_body(Estimator* e, StreamLaunch streamLaunch, int n, const float* h_smp,
                            const float* h_consts, const float* h_initial, float* h_params, int* h_iters,
                            float* h_crlb, float* h_chisq, cudaStream_t cs, Slot& ks) {
    const int K = e->K, NC = e->numconst, npix = e->npix();
    const int nblocks = (n + (1 << kStreamBlockShift) - 1) >> kStreamBlockShift;
    e->stSmp.ensure(sizeof(float) * (size_t)npix * n);
    if (NC) e->stConsts.ensure(sizeof(float) * (size_t)NC * n);
    if (h_initial) e->stInitial.ensure(sizeof(float) * (size_t)K * n);
    e->stParams.ensure(sizeof(float) * (size_t)K * n);
    if (h_iters) e->stIters.ensure(sizeof(int) * (size_t)n);
    if (h_crlb) {
        e->stCrlb.ensure(sizeof(float) * (size_t)K * n);
        e->stFisher.ensure(sizeof(float) * (size_t)fisher_row_floats(K) * n);
    }
    if (h_crlb || h_chisq) e->stChisq.ensure(sizeof(float) * (size_t)n);
    e->stFlags.ensure(sizeof(int) * (size_t)(1 + nblocks));
    e->stClaim.ensure(sizeof(int));
    // chunks of at most 32 MB of samples, whole 1024-ROI blocks; the first three at 1/8, 1/4
    // and 1/2 size so that the fits start early
    const int blk = 1 << kStreamBlockShift;
    int chunk = (int)std::max<long long>(8 * blk, ((32LL << 20) / (4LL * npix)) / (8 * blk) * (8 * blk));
    std::vector<std::pair<int, int>> chunks;
    for (int start = 0, k = 0; start < n; k++) {
        int c = k < 3 ? chunk >> (3 - k) : chunk;
        c = std::min(c, n - start);
        chunks.push_back({start, c});
        start += c;
    }
    const int onesNeeded = chunk / blk + 1;
    if (e->hostOnesCount < onesNeeded) {
        if (e->hostOnes) PB_CUDA(cudaFreeHost(e->hostOnes));
        e->hostOnes = nullptr;
        e->hostOnesCount = 0;
        PB_CUDA(cudaMallocHost(&e->hostOnes, sizeof(int) * onesNeeded));
        for (int i = 0; i < onesNeeded; i++) e->hostOnes[i] = 1;
        e->hostOnesCount = onesNeeded;
    }
    int* d_flags = e->stFlags.as<int>();
    // the flags cleared and the small inputs in place before the launch starts
    PB_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(int) * (size_t)(1 + nblocks), cs));
    if (NC)
        PB_CUDA(cudaMemcpyAsync(e->stConsts.p, h_consts, sizeof(float) * (size_t)NC * n, cudaMemcpyHostToDevice, cs));
    if (h_initial)
        PB_CUDA(cudaMemcpyAsync(e->stInitial.p, h_initial, sizeof(float) * (size_t)K * n, cudaMemcpyHostToDevice, cs));
    PB_CUDA(cudaEventRecord(ks.copied, cs));
    PB_CUDA(cudaStreamWaitEvent(ks.stream, ks.copied, 0));
    FitArgs a{};
    a.smp = e->stSmp.as<float>();
    a.consts = NC ? e->stConsts.as<float>() : nullptr;
    a.initial = h_initial ? e->stInitial.as<float>() : nullptr;
    a.params = e->stParams.as<float>();
    a.iterations = h_iters ? e->stIters.as<int>() : nullptr;
    a.crlb = h_crlb ? e->stCrlb.as<float>() : nullptr;
    a.chisq = (h_crlb || h_chisq) ? e->stChisq.as<float>() : nullptr;
    a.fisher = h_crlb ? e->stFisher.as<float>() : nullptr;
    a.n = n;
    a.maxIter = e->lm.iterations;
    a.lambda = e->lm.lambda;
    a.claim = e->stClaim.as<int>();
    const FitLaunch launch = e->fit_launch();
    const int threads = e->threads_for();
    const bool measure = e->streamPref == 0;
    if (measure && !e->stCopyStart) {
        PB_CUDA(cudaEventCreate(&e->stCopyStart));
        PB_CUDA(cudaEventCreate(&e->stCopyEnd));
        PB_CUDA(cudaEventCreate(&e->stLmEnd));
    }
    streamLaunch(e->desc, a, d_flags, threads, ks.stream);  // LM only (no Fisher outputs)
    if (measure) {
        PB_CUDA(cudaEventRecord(e->stLmEnd, ks.stream));
        PB_CUDA(cudaEventRecord(e->stCopyStart, cs));
    }
    for (const auto& ch : chunks) {
        const int start = ch.first, count = ch.second;
        PB_CUDA(cudaMemcpyAsync(e->stSmp.as<float>() + (size_t)start * npix, h_smp + (size_t)start * npix,
                                sizeof(float) * (size_t)npix * count, cudaMemcpyHostToDevice, cs));
        const int b0 = start >> kStreamBlockShift, b1 = (start + count + blk - 1) >> kStreamBlockShift;
        PB_CUDA(cudaMemcpyAsync(d_flags + 1 + b0, e->hostOnes, sizeof(int) * (size_t)(b1 - b0),
                                cudaMemcpyHostToDevice, cs));
    }
    PB_CUDA(cudaEventRecord(ks.freed, cs));
    if (measure) PB_CUDA(cudaEventRecord(e->stCopyEnd, cs));
    // the parameters and iteration counts go out on the copy stream while the Fisher and CRLB
    // launches run
    PB_CUDA(cudaEventRecord(ks.copied, ks.stream));
    PB_CUDA(cudaStreamWaitEvent(cs, ks.copied, 0));
    if (h_params)
        PB_CUDA(cudaMemcpyAsync(h_params, a.params, sizeof(float) * (size_t)K * n, cudaMemcpyDeviceToHost, cs));
    if (h_iters)
        PB_CUDA(cudaMemcpyAsync(h_iters, a.iterations, sizeof(int) * (size_t)n, cudaMemcpyDeviceToHost, cs));
    PB_CUDA(cudaStreamWaitEvent(ks.stream, ks.freed, 0));  // every ROI in place for the Fisher pass
    if (h_crlb) {
        launch(e->desc, fisher_pass_args(a), threads, ks.stream);
        launch_crlb(K, a.fisher, a.crlb, a.chisq, n, ks.stream, e->crlbAbs);
    }
    if (h_crlb)
        PB_CUDA(cudaMemcpyAsync(h_crlb, a.crlb, sizeof(float) * (size_t)K * n, cudaMemcpyDeviceToHost, ks.stream));
    if (h_chisq)
        PB_CUDA(cudaMemcpyAsync(h_chisq, a.chisq, sizeof(float) * (size_t)n, cudaMemcpyDeviceToHost, ks.stream));
    PB_CUDA(cudaStreamSynchronize(cs));
    PB_CUDA(cudaStreamSynchronize(ks.stream));
    int err = 0;
    PB_CUDA(cudaMemcpy(&err, d_flags, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) throw Error("streamed fit: ROIs did not arrive in device memory in time");
    if (measure) {
        // Fits that end soon after the last ROIs arrived were waiting for the copies: then the
        // slot pipeline, which also overlaps the copies out, is faster (1M ROIs end to end: XYIBg
        // 10x10 7.6 against 8.7 ms, astig 12x12 11.5 against 12.9 ms); fits that run on for
        // longer gain from the single launch (SigmaXY 16x16 24.3 against 26.1 ms).
        float copyMs = 0.0f, tailMs = 0.0f;
        PB_CUDA(cudaEventElapsedTime(&copyMs, e->stCopyStart, e->stCopyEnd));
        PB_CUDA(cudaEventElapsedTime(&tailMs, e->stCopyEnd, e->stLmEnd));
        e->streamPref = tailMs > 0.1f * copyMs ? 1 : -1;
    }
}

void host_fit(Estimator* e, int n, const float* h_smp, const float* h_consts, const float* h_initial,
              float* h_params, int* h_iters, float* h_trace, int traceLen, float* h_crlb, float* h_chisq,
              int flags, float* h_glrt = nullptr, float* h_fisher = nullptr) {
    std::lock_guard<std::mutex> g(e->mtx);
    PB_CUDA(cudaSetDevice(e->device));
    {
        int G = 0, cpl = 0;
        e->fit_shape(G, cpl);
        const bool plain = (flags & FIT_CRLB_ONLY) == 0 && !(h_trace && traceLen > 0) && !h_glrt && !h_fisher;
        const StreamLaunch sl = cpl > 0 ? stream_launcher_for(e->desc.model, G, cpl) : nullptr;
        if (sl && plain && h_smp && e->hostChunk == 0 && e->streamPref >= 0 && n > 16384 &&
            4LL * e->npix() * n <= kStreamedMaxBytes) {
            if (e->numconst && !h_consts) throw Error("this estimator needs per-spot constants");
            host_fit_streamed(e, sl, n, h_smp, h_consts, h_initial, h_params, h_iters, h_crlb, h_chisq);
            return;
        }
    }
    const int K = e->K, NC = e->numconst, npix = e->npix();
    const bool fisherOnly = (flags & FIT_CRLB_ONLY) != 0;
    const bool wantGlrt = h_glrt && e->glrt && !fisherOnly;
    if (wantGlrt && e->glrtRefMean) {
        e->glrtRoi0.ensure(sizeof(float) * npix);
        PB_CUDA(cudaMemcpy(e->glrtRoi0.p, h_smp, sizeof(float) * npix, cudaMemcpyHostToDevice));
    }
    // Chunks of at most 64 MB of samples (at least 16384 ROIs, a sixteenth of the call when that
    // is smaller); the first three are 1/8, 1/4 and 1/2 of that, so the first fit starts early.
    // Every chunk boundary costs the end of a fit launch, whose last ROIs leave most of the GPU
    // idle (about 0.18 ms for 16x16 SigmaXY ROIs, even with the next chunk's launch on another
    // stream); calls whose copies are slower than their fits (which is when this path runs, see
    // host_fit_streamed) gain from the smaller chunks: 1M ROIs end to end, chunks of 65536 / 131072
    // ROIs: XYIBg 10x10 7.60 / 7.79 ms, astig 12x12 11.5 / 11.9 ms.
    int chunk = n;
    if (e->hostChunk > 0) {
        chunk = std::min(n, e->hostChunk);
    } else if (n > 16384) {
        const int cmax = (int)std::max<long long>(4096, (64LL << 20) / (4LL * npix));
        chunk = std::min(cmax, std::max(16384, (n + 15) / 16));
    }
    std::vector<std::pair<int, int>> chunks;  // (start, count)
    for (int start = 0, k = 0; start < n; k++) {
        int c = chunk;
        if (k < 3 && n > chunk) c = std::max(1024, chunk >> (3 - k));
        c = std::min(c, n - start);
        chunks.push_back({start, c});
        start += c;
    }
    const int nchunks = (int)chunks.size();
    const int nslots = e->hostSlots;
    const cudaStream_t cs = e->copy_stream();
    std::vector<char> slotUsed(nslots, 0);
    struct Pending {
        int slot, start, count;
    };
    auto d2h = [&](const Pending& p) {
        Slot& s = e->slot(p.slot);
        if (h_params && !fisherOnly)
            PB_CUDA(cudaMemcpyAsync(h_params + (size_t)p.start * K, s.params.as<float>(), sizeof(float) * K * p.count,
                                    cudaMemcpyDeviceToHost, s.stream));
        if (h_iters)
            PB_CUDA(cudaMemcpyAsync(h_iters + p.start, s.iters.as<int>(), sizeof(int) * p.count,
                                    cudaMemcpyDeviceToHost, s.stream));
        if (h_trace && traceLen > 0)
            PB_CUDA(cudaMemcpyAsync(h_trace + (size_t)p.start * traceLen * K, s.trace.as<float>(),
                                    sizeof(float) * (size_t)traceLen * K * p.count, cudaMemcpyDeviceToHost,
                                    s.stream));
        if (h_crlb)
            PB_CUDA(cudaMemcpyAsync(h_crlb + (size_t)p.start * K, s.crlb.as<float>(), sizeof(float) * K * p.count,
                                    cudaMemcpyDeviceToHost, s.stream));
        if (h_chisq)
            PB_CUDA(cudaMemcpyAsync(h_chisq + p.start, s.chisq.as<float>(), sizeof(float) * p.count,
                                    cudaMemcpyDeviceToHost, s.stream));
        if (wantGlrt)
            PB_CUDA(cudaMemcpyAsync(h_glrt + (size_t)p.start * 3, s.glrt.as<float>(), sizeof(float) * 3 * p.count,
                                    cudaMemcpyDeviceToHost, s.stream));
        if (h_fisher)
            PB_CUDA(cudaMemcpyAsync(h_fisher + (size_t)p.start * fisher_row_floats(K), s.fisher.as<float>(),
                                    sizeof(float) * fisher_row_floats(K) * p.count, cudaMemcpyDeviceToHost,
                                    s.stream));
    };
    for (int c = 0; c < nchunks; c++) {
        const int start = chunks[c].first, count = chunks[c].second;
        const int k = c % nslots;
        Slot& s = e->slot(k);
        if (NC && !h_consts) throw Error("this estimator needs per-spot constants");
        if (h_smp) s.smp.ensure(sizeof(float) * (size_t)npix * count);
        if (NC) s.consts.ensure(sizeof(float) * NC * count);
        if (h_initial) s.initial.ensure(sizeof(float) * K * count);
        if (slotUsed[k]) PB_CUDA(cudaStreamWaitEvent(cs, s.freed, 0));
        if (h_smp)
            PB_CUDA(cudaMemcpyAsync(s.smp.p, h_smp + (size_t)start * npix, sizeof(float) * (size_t)npix * count,
                                    cudaMemcpyHostToDevice, cs));
        if (NC)
            PB_CUDA(cudaMemcpyAsync(s.consts.p, h_consts + (size_t)start * NC, sizeof(float) * NC * count,
                                    cudaMemcpyHostToDevice, cs));
        if (h_initial)
            PB_CUDA(cudaMemcpyAsync(s.initial.p, h_initial + (size_t)start * K, sizeof(float) * K * count,
                                    cudaMemcpyHostToDevice, cs));
        PB_CUDA(cudaEventRecord(s.copied, cs));
        PB_CUDA(cudaStreamWaitEvent(s.stream, s.copied, 0));
        slotUsed[k] = 1;
        s.params.ensure(sizeof(float) * K * count);
        if (h_iters) s.iters.ensure(sizeof(int) * count);
        if (h_trace && traceLen > 0) {
            s.trace.ensure(sizeof(float) * (size_t)traceLen * K * count);
            PB_CUDA(cudaMemsetAsync(s.trace.p, 0, sizeof(float) * (size_t)traceLen * K * count, s.stream));
        }
        if (h_crlb) s.crlb.ensure(sizeof(float) * K * count);
        if (h_crlb || h_fisher) s.fisher.ensure(sizeof(float) * fisher_row_floats(K) * count);
        if (h_chisq || h_crlb) s.chisq.ensure(sizeof(float) * count);
        FitArgs a{};
        a.smp = h_smp ? s.smp.as<float>() : nullptr;
        a.consts = NC ? s.consts.as<float>() : nullptr;
        a.initial = h_initial ? s.initial.as<float>() : nullptr;
        a.params = s.params.as<float>();
        a.iterations = h_iters ? s.iters.as<int>() : nullptr;
        a.trace = (h_trace && traceLen > 0) ? s.trace.as<float>() : nullptr;
        a.traceLen = (h_trace && traceLen > 0) ? traceLen : 0;
        a.crlb = h_crlb ? s.crlb.as<float>() : nullptr;
        a.chisq = (h_chisq || h_crlb) ? s.chisq.as<float>() : nullptr;
        a.n = count;
        a.maxIter = e->lm.iterations;
        a.lambda = e->lm.lambda;
        a.flags = flags;
        a.fisher = (h_crlb || h_fisher) ? s.fisher.as<float>() : nullptr;
        s.claim.ensure(sizeof(int));
        a.claim = s.claim.as<int>();
        if (wantGlrt) {
            s.glrt.ensure(sizeof(float) * 3 * count);
            a.glrt = s.glrt.as<float>();
            a.glrtMeanRoi = e->glrtRefMean ? e->glrtRoi0.as<float>() : nullptr;
        }
        launch_fit_fisher(e, a, s.stream);
        if (h_crlb) launch_crlb(K, a.fisher, a.crlb, a.chisq, count, s.stream, e->crlbAbs);
        PB_CUDA(cudaEventRecord(s.freed, s.stream));
        d2h({k, start, count});
    }
    PB_CUDA(cudaStreamSynchronize(cs));
    for (int i = 0; i < Estimator::kMaxSlots; i++)
        if (e->slots[i].stream) PB_CUDA(cudaStreamSynchronize(e->slots[i].stream));
}

void host_eval(Estimator* e, int n, const float* h_params, const float* h_consts, float* h_ev, float* h_deriv) {
    std::lock_guard<std::mutex> g(e->mtx);
    PB_CUDA(cudaSetDevice(e->device));
    const int K = e->K, NC = e->numconst, npix = e->npix();
    Slot& s = e->slot(0);
    s.initial.ensure(sizeof(float) * K * n);
    PB_CUDA(cudaMemcpyAsync(s.initial.p, h_params, sizeof(float) * K * n, cudaMemcpyHostToDevice, s.stream));
    if (NC) {
        if (!h_consts) throw Error("this estimator needs per-spot constants");
        s.consts.ensure(sizeof(float) * NC * n);
        PB_CUDA(cudaMemcpyAsync(s.consts.p, h_consts, sizeof(float) * NC * n, cudaMemcpyHostToDevice, s.stream));
    }
    if (h_ev) s.smp.ensure(sizeof(float) * (size_t)npix * n);
    if (h_deriv) s.trace.ensure(sizeof(float) * (size_t)npix * K * n);
    int G = e->lanes_for();
    if (G < 8) G = 8;
    eval_launcher_for(e->desc.model, G)(e->desc, s.initial.as<float>(), NC ? s.consts.as<float>() : nullptr,
                                    h_ev ? s.smp.as<float>() : nullptr, h_deriv ? s.trace.as<float>() : nullptr, n,
                                    256, s.stream);
    if (h_ev)
        PB_CUDA(cudaMemcpyAsync(h_ev, s.smp.p, sizeof(float) * (size_t)npix * n, cudaMemcpyDeviceToHost, s.stream));
    if (h_deriv)
        PB_CUDA(cudaMemcpyAsync(h_deriv, s.trace.p, sizeof(float) * (size_t)npix * K * n, cudaMemcpyDeviceToHost,
                                s.stream));
    PB_CUDA(cudaStreamSynchronize(s.stream));
}

// ------------------------------------------------------------------------------------
// Spline coefficients (CubicSplinePSF.cu:151-204) on the GPU.
// The 64x64 power-basis matrix is LUP-factored once on the host in double precision with the
// reference's algorithm; one thread per output voxel runs the reference's forward/backward
// substitution with non-fused double arithmetic, so results are bit-identical.
// ------------------------------------------------------------------------------------
__constant__ double c_splineLU[64 * 64];
__constant__ int c_splineP[65];

__global__ void spline_compute_kernel(const float* __restrict__ data, int s0, int s1, int s2, int border,
                                      float* __restrict__ coefs, int o0, int o1, int o2) {
    const long long total = (long long)o0 * o1 * o2;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < total;
         v += (long long)gridDim.x * blockDim.x) {
        const int k = (int)(v % o2);
        const int j = (int)((v / o2) % o1);
        const int i = (int)(v / ((long long)o1 * o2));
        double b[64], x[64];
#pragma unroll
        for (int m = 0; m < 4; m++)
#pragma unroll
            for (int n = 0; n < 4; n++)
#pragma unroll
                for (int o = 0; o < 4; o++) {
                    int z = min(max(i + m - border, 0), s0 - 1);
                    int y = min(max(j + n - border, 0), s1 - 1);
                    int xx = min(max(k + o - border, 0), s2 - 1);
                    b[m * 16 + n * 4 + o] = (double)data[((size_t)z * s1 + y) * s2 + xx];
                }
        for (int r = 0; r < 64; r++) {
            double t = b[c_splineP[r]];
            for (int q = 0; q < r; q++) t = __dsub_rn(t, __dmul_rn(c_splineLU[r * 64 + q], x[q]));
            x[r] = t;
        }
        for (int r = 63; r >= 0; r--) {
            double t = x[r];
            for (int q = r + 1; q < 64; q++) t = __dsub_rn(t, __dmul_rn(c_splineLU[r * 64 + q], x[q]));
            x[r] = __ddiv_rn(t, c_splineLU[r * 64 + r]);
        }
        float* dst = coefs + 64 * v;
#pragma unroll
        for (int a = 0; a < 64; a++) dst[a] = (float)x[a];
    }
}

void spline_lu_once() {
    static std::once_flag once;
    static int dev_done[64] = {0};
    static double LU[64 * 64];
    static int P[65];
    std::call_once(once, [] {
        const int N = 64;
        for (int i = 0; i < 4; i++)
            for (int j = 0; j < 4; j++)
                for (int k = 0; k < 4; k++)
                    for (int l = 0; l < 4; l++)
                        for (int m = 0; m < 4; m++)
                            for (int n = 0; n < 4; n++)
                                LU[64 * (i * 16 + j * 4 + k) + (l * 16 + m * 4 + n)] =
                                    (double)(powf((float)(i - 1.0), (float)l) * powf((float)(j - 1.0), (float)m) *
                                             powf((float)(k - 1.0), (float)n));
        for (int i = 0; i <= N; i++) P[i] = i;
        for (int i = 0; i < N; i++) {
            double maxA = 0.0, absA;
            int imax = i;
            for (int k = i; k < N; k++)
                if ((absA = std::fabs(LU[k * N + i])) > maxA) { maxA = absA; imax = k; }
            if (imax != i) {
                std::swap(P[i], P[imax]);
                for (int jj = 0; jj < N; jj++) std::swap(LU[i * N + jj], LU[imax * N + jj]);
                P[N]++;
            }
            for (int j = i + 1; j < N; j++) {
                LU[j * N + i] /= LU[i * N + i];
                for (int k = i + 1; k < N; k++) LU[j * N + k] -= LU[j * N + i] * LU[i * N + k];
            }
        }
    });
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !dev_done[dev]) {
        PB_CUDA(cudaMemcpyToSymbol(c_splineLU, LU, sizeof(LU)));
        PB_CUDA(cudaMemcpyToSymbol(c_splineP, P, sizeof(P)));
        dev_done[dev] = 1;
    }
}

void spline_compute_device(const int* shape, const float* d_data, float* d_coefs, int border, cudaStream_t s) {
    spline_lu_once();
    const int o0 = shape[0] - 3 + 2 * border, o1 = shape[1] - 3 + 2 * border, o2 = shape[2] - 3 + 2 * border;
    if (o0 <= 0 || o1 <= 0 || o2 <= 0) throw Error("z-stack too small for a cubic spline");
    const long long total = (long long)o0 * o1 * o2;
    const int threads = 128;
    const int grid = (int)std::min<long long>((total + threads - 1) / threads, 65535);
    spline_compute_kernel<<<grid, threads, 0, s>>>(d_data, shape[0], shape[1], shape[2], border, d_coefs, o0, o1, o2);
    PB_CUDA(cudaGetLastError());
    count_launch();
}

// CSpline_Evaluate (CubicSplinePSF.cu:208-271): values[z][y][x][4] = val, dx, dy, dz.
__global__ void spline_evaluate_kernel(const float* __restrict__ coefs, int s0, int s1, int s2, float d0, float d1,
                                       float d2, float sh0, float sh1, float sh2, int border, float* values) {
    const int n0 = s0 - 2 * border, n1 = s1 - 2 * border, n2 = s2 - 2 * border;
    const long long total = (long long)n0 * n1 * n2;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < total;
         v += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(v % n2) + border;
        const int y = (int)((v / n2) % n1) + border;
        const int z = (int)(v / ((long long)n1 * n2)) + border;
        float df[64], dxf[64], dyf[64], dzf[64];
        for (int q = 0; q < 64; q++) df[q] = dxf[q] = dyf[q] = dzf[q] = 0.0f;
        float zzz = 1.0f;
        for (int m = 0; m <= 3; m++) {
            float yyy = 1.0f;
            for (int n = 0; n <= 3; n++) {
                float xxx = 1.0f;
                for (int o = 0; o <= 3; o++) {
                    const float xyz = MUL(MUL(xxx, yyy), zzz);
                    df[m * 16 + n * 4 + o] = xyz;
                    if (o < 3) dxf[m * 16 + n * 4 + o + 1] = MUL((float)o + 1.0f, xyz);
                    if (n < 3) dyf[m * 16 + (n + 1) * 4 + o] = MUL((float)n + 1.0f, xyz);
                    if (m < 3) dzf[(m + 1) * 16 + n * 4 + o] = MUL((float)m + 1.0f, xyz);
                    xxx = MUL(xxx, d2);
                }
                yyy = MUL(yyy, d1);
            }
            zzz = MUL(zzz, d0);
        }
        const float zz = SUB((float)z, sh0);
        const int k = min(max((int)zz, 0), s0 - 1);
        const float yy = SUB((float)y, sh1);
        const int j = min(max((int)yy, 0), s1 - 1);
        const float xx = SUB((float)x, sh2);
        const int i = min(max((int)xx, 0), s2 - 1);
        float val = 0.0f, dx = 0.0f, dy = 0.0f, dz = 0.0f;
        const float* c = coefs + 64 * (((size_t)k * s1 + j) * s2 + i);
        for (int idx = 0; idx < 64; idx++) {
            const float cf = c[idx];
            val = ADD(val, MUL(df[idx], cf));
            dx = ADD(dx, MUL(dxf[idx], cf));
            dy = ADD(dy, MUL(dyf[idx], cf));
            dz = ADD(dz, MUL(dzf[idx], cf));
        }
        float* out = values + 4 * v;
        out[0] = val;
        out[1] = dx;
        out[2] = dy;
        out[3] = dz;
    }
}

// The q-major copy of the spline coefficients (ModelDesc::coefsQ).
__global__ void coefs_qmajor_kernel(const float4* __restrict__ src, float4* __restrict__ dst, size_t nvox) {
    for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < nvox * 16; t += (size_t)gridDim.x * blockDim.x) {
        const size_t v = t / 16, q = t % 16;
        dst[q * nvox + v] = src[t];
    }
}

void build_coefs_qmajor(Estimator* e) {
    const size_t nvox = (size_t)e->desc.spline_shape[0] * e->desc.spline_shape[1] * e->desc.spline_shape[2];
    e->coefsQ.ensure(sizeof(float) * 64 * nvox);
    const int grid = (int)std::min<size_t>((nvox * 16 + 255) / 256, 65535);
    coefs_qmajor_kernel<<<grid, 256>>>(e->coefs.as<float4>(), e->coefsQ.as<float4>(), nvox);
    PB_CUDA(cudaGetLastError());
    PB_CUDA(cudaDeviceSynchronize());
    e->desc.coefsQ = e->coefsQ.as<float4>();
}

Estimator* make_spline(int roisize, const CSpline_Calibration* calib, const float* h_coefs, int mode, Context* ctx,
                       const float* d_coefs_src, float xyStep = 1.0f) {
    // modes CSPLINE_FLATBG 0, CSPLINE_TILTEDBG 1, CSPLINE_BGIMAGE 2 (CubicSplinePSF.cu:76-101)
    if (mode < 0 || mode > 2) throw Error("Invalid model background mode");
    if (!(xyStep > 0.0f) || !(xyStep <= 1.0f)) throw Error("CSpline_CreatePSF_Oversampled: xyStep must be in (0, 1]");
    if (xyStep != 1.0f && mode == 2) throw Error("CSpline_CreatePSF_Oversampled: the background-image mode takes 1 px voxels");
    if (roisize < 3 || roisize > 64) throw Error("roisize must be in [3, 64]");
    if (!calib) throw Error("CSpline_CreatePSF: calibration is null");
    const int nz = calib->shape[0], ny = calib->shape[1], nx = calib->shape[2];
    if (nz <= 0 || ny <= 0 || nx <= 0) throw Error("CSpline_CreatePSF: empty coefficient grid");
    auto* e = new Estimator();
    try {
        e->desc.model = mode == 0 ? MODEL_CSPLINE : (mode == 1 ? MODEL_CSPLINE_TILTED : MODEL_CSPLINE_BGIMAGE);
        e->desc.roisize = roisize;
        e->desc.spline_shape[0] = nz;
        e->desc.spline_shape[1] = ny;
        e->desc.spline_shape[2] = nx;
        e->desc.spline_zmin = calib->z_min;
        e->desc.spline_zmax = calib->z_max;
        e->desc.spline_q = 1.0f / xyStep;
        const size_t ncoef = (size_t)nz * ny * nx * 64;
        e->coefs.ensure(sizeof(float) * ncoef);
        if (d_coefs_src)
            PB_CUDA(cudaMemcpy(e->coefs.p, d_coefs_src, sizeof(float) * ncoef, cudaMemcpyDeviceToDevice));
        else {
            const float* src = h_coefs ? h_coefs : calib->coefs;
            if (!src) throw Error("CSpline_CreatePSF: no coefficients");
            PB_CUDA(cudaMemcpy(e->coefs.p, src, sizeof(float) * ncoef, cudaMemcpyHostToDevice));
        }
        e->desc.coefs = e->coefs.as<float>();
        build_coefs_qmajor(e);
        e->K = model_num_params(e->desc.model);
        e->numconst = mode == 2 ? roisize * roisize : 0;  // the background image of each spot
        e->format = mode == 1 ? "x,y,z,I,bg,bgx,bgy" : "x,y,z,I,bg";
        const float border = 1.5f;
        const float xyhi = (float)(roisize - 1) - border;
        e->limits = {{border, xyhi}, {border, xyhi}, {calib->z_min, calib->z_max}, {10.0f, 1e9f}, {1e-6f, 1e9f}};
        if (mode == 1) {  // CubicSplinePSF.cu:67-70
            e->limits.push_back({-1e6f, 1e6f});
            e->limits.push_back({-1e6f, 1e6f});
        }
    } catch (...) {
        delete e;
        throw;
    }
    attach(e, ctx);
    return e;
}

// Device-pointer fit on a caller stream. The LM launch's ROI counter and, with a CRLB request,
// the packed Fisher rows go to a stream-ordered scratch allocation (cudaMallocAsync), which is
// freed on the same stream after the last launch has used it; concurrent calls on different
// streams therefore never share it.
// Keep freed stream-ordered allocations in the device's default pool instead of returning them
// to the driver at every synchronisation (repeated calls would otherwise remap memory each time).
void keep_pool_memory() {
    static bool done[64] = {false};
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64 || done[dev]) return;
    cudaMemPool_t pool;
    PB_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t threshold = UINT64_MAX;
    PB_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
    done[dev] = true;
}

void run_fit_device(Estimator* e, FitArgs a, cudaStream_t s) {
    keep_pool_memory();
    constexpr size_t kHead = 256;  // the counter, padded so that the Fisher rows start aligned
    const size_t bytes = kHead + (a.crlb ? sizeof(float) * fisher_row_floats(e->K) * (size_t)a.n : 0);
    void* scratch = nullptr;
    PB_CUDA(cudaMallocAsync(&scratch, bytes, s));
    a.claim = static_cast<int*>(scratch);
    if (a.crlb) a.fisher = reinterpret_cast<float*>(static_cast<char*>(scratch) + kHead);
    try {
        launch_fit_fisher(e, a, s);
        if (a.crlb) launch_crlb(e->K, a.fisher, a.crlb, a.chisq, a.n, s, e->crlbAbs);
    } catch (...) {
        cudaFreeAsync(scratch, s);
        throw;
    }
    PB_CUDA(cudaFreeAsync(scratch, s));
}

void check_estimator(Estimator* e) {
    if (!e) throw Error("estimator is null");
}

}  // namespace

// ------------------------------------------------------------------------------------
// C ABI
// ------------------------------------------------------------------------------------
template <class F>
auto guarded(F&& f, decltype(f()) onerr) -> decltype(f()) {
    try {
        return f();
    } catch (const std::exception& ex) {
        report(ex);
        return onerr;
    }
}

template <class F>
void guarded_void(F&& f) {
    try {
        f();
    } catch (const std::exception& ex) {
        report(ex);
    }
}

extern "C" {

const char* PB200_GetLastError(void) { return t_lastError.c_str(); }
void PB200_ClearError(void) { t_lastError.clear(); }
uint64_t PB200_LaunchCount(void) { return g_launches.load(); }

Context* Context_Create(void) { return new Context(); }

void Context_Destroy(Context* ctx) {
    if (!ctx) return;
    std::vector<Estimator*> objs;
    std::vector<std::pair<void*, void (*)(void*)>> owned;
    {
        std::lock_guard<std::mutex> g(ctx->mtx);
        objs.assign(ctx->objects.begin(), ctx->objects.end());
        ctx->objects.clear();
        owned.assign(ctx->owned.rbegin(), ctx->owned.rend());  // newest first
        ctx->owned.clear();
    }
    for (auto& o : owned) o.second(o.first);  // queues first: they use the estimators
    for (auto* e : objs) {
        e->ctx = nullptr;
        delete e;
    }
    delete ctx;
}

Estimator* Gauss2D_CreatePSF_XYIBg(int roisize, float sigmaX, float sigmaY, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {return make_gauss(MODEL_XYIBG, roisize, sigmaX, sigmaY, nullptr, nullptr, 0, 0, ctx);}, (Estimator*)nullptr);
}

Estimator* Gauss2D_CreatePSF_XYIBgConstSigma(int roisize, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {return make_gauss(MODEL_XYIBG_CONSTSIGMA, roisize, 0, 0, nullptr, nullptr, 0, 0, ctx);}, (Estimator*)nullptr);
}

Estimator* Gauss2D_CreatePSF_XYIBgSigma(int roisize, float initialSigma, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {return make_gauss(MODEL_XYIBG_SIGMA, roisize, initialSigma, initialSigma, nullptr, nullptr, 0, 0, ctx);
           }, (Estimator*)nullptr);
}

Estimator* Gauss2D_CreatePSF_XYIBgSigmaXY(int roisize, float sx, float sy, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {return make_gauss(MODEL_XYIBG_SIGMAXY, roisize, sx, sy, nullptr, nullptr, 0, 0, ctx);}, (Estimator*)nullptr);
}

Estimator* Gauss2D_CreatePSF_XYZIBg(int roisize, const Gauss3D_Calibration* calib, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {
        if (!calib) throw Error("Gauss2D_CreatePSF_XYZIBg: calibration is null");
        float ax[5] = {calib->x[0], calib->x[1], calib->x[2], calib->x[3], 0.0f};
        float ay[5] = {calib->y[0], calib->y[1], calib->y[2], calib->y[3], 0.0f};
        return make_gauss(MODEL_XYZIBG, roisize, 0, 0, ax, ay, calib->minz, calib->maxz, ctx);
        }, (Estimator*)nullptr);
}

Estimator* Gauss2D_CreatePSF_XYZIBgB(int roisize, const Gauss3D_CalibrationB* calib, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {
        if (!calib) throw Error("Gauss2D_CreatePSF_XYZIBgB: calibration is null");
        return make_gauss(MODEL_XYZIBG, roisize, 0, 0, calib->x, calib->y, calib->minz, calib->maxz, ctx);
        }, (Estimator*)nullptr);
}

Estimator* CSpline_CreatePSF(int roisize, const CSpline_Calibration* calib, const float* coefs, int mode, bool,
                             Context* ctx) {
    return guarded([&]() -> Estimator* {return make_spline(roisize, calib, coefs, mode, ctx, nullptr);}, (Estimator*)nullptr);
}

Estimator* CSpline_CreatePSF_Oversampled(int roisize, const CSpline_Calibration* calib, const float* coefs, int mode,
                                         float xyStep, bool, Context* ctx) {
    return guarded([&]() -> Estimator* { return make_spline(roisize, calib, coefs, mode, ctx, nullptr, xyStep); },
                   (Estimator*)nullptr);
}

Estimator* CSpline_CreatePSF_FromFile(int roisize, const char* filename, int mode, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {
        FILE* f = fopen(filename, "rb");
        if (!f) throw Error(std::string("Can't open file ") + (filename ? filename : "(null)"));
        struct {
            int version;
            int shape[3];
            float zmin, zmax;
        } h;
        size_t got = fread(&h, sizeof(h), 1, f);
        if (got != 1 || h.version != 1) {
            fclose(f);
            throw Error("Wrong ZStack file version (should be 1)");
        }
        const size_t nvox = (size_t)h.shape[0] * h.shape[1] * h.shape[2];
        std::vector<float> data(nvox);
        got = fread(data.data(), sizeof(float), nvox, f);
        fclose(f);
        if (got != nvox) throw Error("ZStack file is truncated");
        DevBuf dd, dc;
        dd.ensure(sizeof(float) * nvox);
        PB_CUDA(cudaMemcpy(dd.p, data.data(), sizeof(float) * nvox, cudaMemcpyHostToDevice));
        const int border = 0;
        int os[3] = {h.shape[0] - 3 + 2 * border, h.shape[1] - 3 + 2 * border, h.shape[2] - 3 + 2 * border};
        dc.ensure(sizeof(float) * 64 * (size_t)os[0] * os[1] * os[2]);
        spline_compute_device(h.shape, dd.as<float>(), dc.as<float>(), border, 0);
        PB_CUDA(cudaDeviceSynchronize());
        CSpline_Calibration c;
        c.shape[0] = os[0];
        c.shape[1] = os[1];
        c.shape[2] = os[2];
        c.z_min = h.zmin;
        c.z_max = h.zmax;
        c.coefs = nullptr;
        return make_spline(roisize, &c, nullptr, mode, ctx, dc.as<float>());
        }, (Estimator*)nullptr);
}

void CSpline_Compute(const int* shape, const float* data, float* splineCoefs, int border) {
    guarded_void([&]() {
        if (!shape || !data || !splineCoefs) throw Error("CSpline_Compute: null argument");
        const size_t nvox = (size_t)shape[0] * shape[1] * shape[2];
        const int o0 = shape[0] - 3 + 2 * border, o1 = shape[1] - 3 + 2 * border, o2 = shape[2] - 3 + 2 * border;
        if (o0 <= 0 || o1 <= 0 || o2 <= 0) throw Error("CSpline_Compute: z-stack too small");
        const size_t nout = (size_t)o0 * o1 * o2 * 64;
        DevBuf dd, dc;
        dd.ensure(sizeof(float) * nvox);
        dc.ensure(sizeof(float) * nout);
        PB_CUDA(cudaMemcpy(dd.p, data, sizeof(float) * nvox, cudaMemcpyHostToDevice));
        spline_compute_device(shape, dd.as<float>(), dc.as<float>(), border, 0);
        PB_CUDA(cudaMemcpy(splineCoefs, dc.p, sizeof(float) * nout, cudaMemcpyDeviceToHost));
        });
}

void CSpline_Evaluate(const int* shape, const float* splineCoefs, const float* shift, int border, float* values) {
    guarded_void([&]() {
        if (!shape || !splineCoefs || !shift || !values) throw Error("CSpline_Evaluate: null argument");
        const size_t ncoef = (size_t)shape[0] * shape[1] * shape[2] * 64;
        const int n0 = shape[0] - 2 * border, n1 = shape[1] - 2 * border, n2 = shape[2] - 2 * border;
        if (n0 <= 0 || n1 <= 0 || n2 <= 0) throw Error("CSpline_Evaluate: border too large");
        const size_t nout = (size_t)n0 * n1 * n2 * 4;
        // subpixel position: d = -shift - int(-shift)  (CubicSplinePSF.cu:215)
        float d[3];
        for (int i = 0; i < 3; i++) {
            const float ms = -shift[i];
            d[i] = ms - (float)(int)ms;
        }
        DevBuf dc, dv;
        dc.ensure(sizeof(float) * ncoef);
        dv.ensure(sizeof(float) * nout);
        PB_CUDA(cudaMemcpy(dc.p, splineCoefs, sizeof(float) * ncoef, cudaMemcpyHostToDevice));
        const long long total = (long long)n0 * n1 * n2;
        const int grid = (int)std::min<long long>((total + 127) / 128, 65535);
        spline_evaluate_kernel<<<grid, 128>>>(dc.as<float>(), shape[0], shape[1], shape[2], d[0], d[1], d[2],
                                              shift[0], shift[1], shift[2], border, dv.as<float>());
        PB_CUDA(cudaGetLastError());
        count_launch();
        PB_CUDA(cudaMemcpy(values, dv.p, sizeof(float) * nout, cudaMemcpyDeviceToHost));
        });
}

// GLRT_PSF.cu:156-170. The reference wraps the model estimator; here the GLRT estimator is an
// independent copy of it (same model, calibration, LM and kernel settings) that also writes
// the three diagnostics per spot, so deleting the model estimator does not affect it.
Estimator* GLRT_CreatePSF(Estimator* model, Context* ctx) {
    return guarded([&]() -> Estimator* {
        if (!model) throw Error("GLRT_CreatePSF: model estimator is null");
        PB_CUDA(cudaSetDevice(model->device));
        auto* e = new Estimator();
        try {
            e->desc = model->desc;
            e->K = model->K;
            e->numconst = model->numconst;
            e->format = model->format;
            e->limits = model->limits;
            e->lm = model->lm;
            e->lanes = model->lanes;
            e->threads = model->threads;
            e->variant = model->variant;
            e->glrt = true;
            if (model_is_spline(model->desc.model)) {
                const size_t ncoef = (size_t)model->desc.spline_shape[0] * model->desc.spline_shape[1] *
                                     model->desc.spline_shape[2] * 64;
                e->coefs.ensure(sizeof(float) * ncoef);
                PB_CUDA(cudaMemcpy(e->coefs.p, model->coefs.p, sizeof(float) * ncoef, cudaMemcpyDeviceToDevice));
                e->desc.coefs = e->coefs.as<float>();
                build_coefs_qmajor(e);
            }
        } catch (...) {
            delete e;
            throw;
        }
        attach(e, ctx);
        return e;
    }, (Estimator*)nullptr);
}

int PB200_SetGLRTReferenceMean(Estimator* e, int on) {
    return guarded([&]() -> int {
        check_estimator(e);
        if (!e->glrt) throw Error("PB200_SetGLRTReferenceMean: not a GLRT estimator");
        std::lock_guard<std::mutex> g(e->mtx);
        e->glrtRefMean = on != 0;
        return 0;
    }, -1);
}

void Estimator_Delete(Estimator* e) {
    if (!e) return;
    detach(e);
    delete e;
}

const char* Estimator_ParamFormat(Estimator* e) { return e ? e->format.c_str() : ""; }

void Estimator_GetProperties(Estimator* e, EstimatorProperties* p) {
    if (!e || !p) return;
    p->numParams = e->K;
    p->sampleCount = e->npix();
    p->numDiag = e->glrt ? 3 : 0;
    p->numConst = e->numconst;
    p->sampleIndexDims = 2;
}

void Estimator_SampleDims(Estimator* e, int* dims) {
    if (!e || !dims) return;
    dims[0] = e->desc.roisize;
    dims[1] = e->desc.roisize;
}

void Estimator_GetParamLimits(Estimator* e, ParamLimit* limits) {
    if (!e || !limits) return;
    for (int i = 0; i < e->K; i++) limits[i] = e->limits[i];
}

void Estimator_SetLMParams(Estimator* e, const LMParams* p) {
    if (!e || !p) return;
    std::lock_guard<std::mutex> g(e->mtx);
    e->lm = *p;
}

void Estimator_GetLMParams(Estimator* e, LMParams* p) {
    if (!e || !p) return;
    *p = e->lm;
}

void Estimator_ComputeExpectedValue(Estimator* e, int numspots, const float* params, const float* constants,
                                    const int*, float* ev) {
    if (numspots == 0) return;
    guarded_void([&]() {check_estimator(e); if (numspots < 0 || !params || !ev) throw Error("ExpectedValue: bad arguments");
           host_eval(e, numspots, params, constants, ev, nullptr);});
}

void Estimator_ComputeDerivatives(Estimator* e, int numspots, const float* params, const float* constants,
                                  const int*, float* psf_deriv, float* ev) {
    if (numspots == 0) return;
    guarded_void([&]() {check_estimator(e); if (numspots < 0 || !params) throw Error("Derivatives: bad arguments");
           host_eval(e, numspots, params, constants, ev, psf_deriv);});
}

void Estimator_Estimate(Estimator* e, int numspots, const float* sample, const float* constants, const int*,
                        const float* initial, float* params, float* diagnostics, int* iterations, float* trace,
                        int traceBufLen) {
    if (numspots == 0) return;
    guarded_void([&]() {check_estimator(e); if (numspots < 0 || !sample || !params) throw Error("Estimate: bad arguments");
           host_fit(e, numspots, sample, constants, initial, params, iterations, trace, traceBufLen, nullptr, nullptr,
                    0, e->glrt ? diagnostics : nullptr);
           });
}

void Estimator_ChiSquareAndCRLB(Estimator* e, const float* params, const float* sample, const float* constants,
                                const int*, int numspots, float* crlb, float* chisq) {
    if (numspots == 0) return;
    guarded_void([&]() {check_estimator(e); if (numspots < 0 || !params || !crlb) throw Error("ChiSquareAndCRLB: bad arguments");
           host_fit(e, numspots, sample, constants, params, nullptr, nullptr, nullptr, 0, crlb, chisq,
                    FIT_CRLB_ONLY);
           });
}

void PB200_FisherMatrix(Estimator* e, int numspots, const float* params, const float* constants, float* fisher) {
    if (numspots == 0) return;
    guarded_void([&]() {
        check_estimator(e);
        if (numspots < 0 || !params || !fisher) throw Error("FisherMatrix: bad arguments");
        const int K = e->K, R = fisher_row_floats(K);
        std::vector<float> rows((size_t)numspots * R);
        host_fit(e, numspots, nullptr, constants, params, nullptr, nullptr, nullptr, 0, nullptr, nullptr,
                 FIT_CRLB_ONLY, nullptr, rows.data());
        for (size_t i = 0; i < (size_t)numspots; i++) {
            const float* r = rows.data() + i * R;
            float* f = fisher + i * K * K;
            for (int a = 0, q = 0; a < K; a++)
                for (int b = a; b < K; b++, q++) f[a * K + b] = f[b * K + a] = r[q];
        }
    });
}

void PB200_FisherMatrixDevice(Estimator* e, int numspots, const float* d_params, const float* d_constants,
                              float* d_fisherRows, void* stream) {
    if (numspots == 0) return;
    guarded_void([&]() {
        check_estimator(e);
        if (numspots < 0 || !d_params || !d_fisherRows) throw Error("FisherMatrixDevice: bad arguments");
        if (e->numconst && !d_constants) throw Error("this estimator needs per-spot constants");
        FitArgs a{}; a.smp = nullptr; a.consts = d_constants; a.initial = d_params; a.params = nullptr;
        a.fisher = d_fisherRows; a.n = numspots; a.maxIter = e->lm.iterations; a.lambda = e->lm.lambda;
        a.flags = FIT_CRLB_ONLY;
        launch_fit_fisher(e, a, (cudaStream_t)stream);});
}

void PB200_EstimateCRLB(Estimator* e, int numspots, const float* sample, const float* constants,
                        const float* initial, float* params, int* iterations, float* crlb, float* chisq) {
    if (numspots == 0) return;
    guarded_void([&]() {check_estimator(e); if (numspots < 0 || !sample || !params) throw Error("EstimateCRLB: bad arguments");
           host_fit(e, numspots, sample, constants, initial, params, iterations, nullptr, 0, crlb, chisq, 0);
           });
}

void PB200_EstimateDevice(Estimator* e, int numspots, const float* d_sample, const float* d_constants,
                          const float* d_initial, float* d_params, int* d_iterations, float* d_trace,
                          int traceBufLen, float* d_crlb, float* d_chisq, void* stream) {
    if (numspots == 0) return;
    guarded_void([&]() {
        check_estimator(e); if (numspots < 0 || !d_sample || !d_params) throw Error("EstimateDevice: bad arguments");
        if (e->numconst && !d_constants) throw Error("this estimator needs per-spot constants");
        FitArgs a{}; a.smp = d_sample; a.consts = d_constants; a.initial = d_initial; a.params = d_params;
        a.iterations = d_iterations; a.trace = traceBufLen > 0 ? d_trace : nullptr;
        a.traceLen = traceBufLen > 0 && d_trace ? traceBufLen : 0; a.crlb = d_crlb; a.chisq = d_chisq;
        a.n = numspots; a.maxIter = e->lm.iterations; a.lambda = e->lm.lambda; a.flags = 0;
        run_fit_device(e, a, (cudaStream_t)stream);});
}

void PB200_EstimateDeviceDiag(Estimator* e, int numspots, const float* d_sample, const float* d_constants,
                              const float* d_initial, float* d_params, float* d_diag, int* d_iterations,
                              float* d_crlb, float* d_chisq, void* stream) {
    if (numspots == 0) return;
    guarded_void([&]() {
        check_estimator(e); if (numspots < 0 || !d_sample || !d_params) throw Error("EstimateDeviceDiag: bad arguments");
        if (e->numconst && !d_constants) throw Error("this estimator needs per-spot constants");
        FitArgs a{}; a.smp = d_sample; a.consts = d_constants; a.initial = d_initial; a.params = d_params;
        a.iterations = d_iterations; a.crlb = d_crlb; a.chisq = d_chisq;
        a.n = numspots; a.maxIter = e->lm.iterations; a.lambda = e->lm.lambda; a.flags = 0;
        if (e->glrt && d_diag) {
            a.glrt = d_diag;
            a.glrtMeanRoi = e->glrtRefMean ? d_sample : nullptr;
        }
        run_fit_device(e, a, (cudaStream_t)stream);});
}

void PB200_EstimateDeviceRescued(Estimator* e, int numspots, const float* d_sample, const float* d_constants,
                                 const float* d_initial, float* d_params, int* d_iterations, float* d_trace,
                                 int traceBufLen, int* d_rescued, void* stream) {
    if (numspots == 0) return;
    guarded_void([&]() {
        check_estimator(e);
        if (numspots < 0 || !d_sample || !d_params || !d_rescued) throw Error("EstimateDeviceRescued: bad arguments");
        if (e->numconst && !d_constants) throw Error("this estimator needs per-spot constants");
        FitArgs a{}; a.smp = d_sample; a.consts = d_constants; a.initial = d_initial; a.params = d_params;
        a.iterations = d_iterations; a.trace = traceBufLen > 0 ? d_trace : nullptr;
        a.traceLen = traceBufLen > 0 && d_trace ? traceBufLen : 0; a.diag = d_rescued;
        a.n = numspots; a.maxIter = e->lm.iterations; a.lambda = e->lm.lambda; a.flags = 0;
        run_fit_device(e, a, (cudaStream_t)stream);});
}

void PB200_ExpectedValueDevice(Estimator* e, int numspots, const float* d_params, const float* d_constants,
                               float* d_ev, float* d_deriv, void* stream) {
    if (numspots == 0) return;
    guarded_void([&]() {
        check_estimator(e); if (numspots < 0 || !d_params) throw Error("ExpectedValueDevice: bad arguments");
        if (e->numconst && !d_constants) throw Error("this estimator needs per-spot constants");
        int G = e->lanes_for(); if (G < 8) G = 8;
        eval_launcher_for(e->desc.model, G)(e->desc, d_params, d_constants, d_ev, d_deriv, numspots, 256,
                                        (cudaStream_t)stream);});
}

void PB200_ChiSquareAndCRLBDevice(Estimator* e, int numspots, const float* d_params, const float* d_sample,
                                  const float* d_constants, float* d_crlb, float* d_chisq, void* stream) {
    if (numspots == 0) return;
    guarded_void([&]() {
        check_estimator(e); if (numspots < 0 || !d_params || !d_crlb) throw Error("ChiSquareAndCRLBDevice: bad arguments");
        if (e->numconst && !d_constants) throw Error("this estimator needs per-spot constants");
        FitArgs a{}; a.smp = d_sample; a.consts = d_constants; a.initial = d_params; a.params = nullptr;
        a.crlb = d_crlb; a.chisq = d_chisq; a.n = numspots; a.maxIter = e->lm.iterations; a.lambda = e->lm.lambda;
        a.flags = FIT_CRLB_ONLY;
        run_fit_device(e, a, (cudaStream_t)stream);});
}

int PB200_SetKernelConfig(Estimator* e, int lanesPerRoi, int threadsPerBlock) {
    if (!e) return -1;
    if (lanesPerRoi != 0 && lanesPerRoi != 2 && lanesPerRoi != 4 && lanesPerRoi != 8 && lanesPerRoi != 16 &&
        lanesPerRoi != 32)
        return -1;
    if (threadsPerBlock != 0 && (threadsPerBlock < 64 || threadsPerBlock > 256 || (threadsPerBlock & 31))) return -1;
    std::lock_guard<std::mutex> g(e->mtx);
    e->lanes = lanesPerRoi;
    e->threads = threadsPerBlock;
    return 0;
}

int PB200_SetHostPipeline(Estimator* e, int roisPerChunk, int slots) {
    if (!e || roisPerChunk < 0 || slots < 2 || slots > Estimator::kMaxSlots) return -1;
    std::lock_guard<std::mutex> g(e->mtx);
    e->hostChunk = roisPerChunk;
    e->hostSlots = slots;
    return 0;
}

int PB200_SetKernelVariant(Estimator* e, int variant) {
    if (!e || variant < 0 || variant > 1) return -1;
    std::lock_guard<std::mutex> g(e->mtx);
    e->variant = variant;
    return 0;
}

void PB200_GetKernelConfig(Estimator* e, int* lanesPerRoi, int* threadsPerBlock) {
    if (!e) return;
    if (lanesPerRoi) {
        int cpl;
        e->fit_shape(*lanesPerRoi, cpl);
    }
    if (threadsPerBlock) *threadsPerBlock = e->launched_threads_for();
}

int PB200_ModelInfo(Estimator* e, int* roisize) {
    if (!e) return -1;
    if (roisize) *roisize = e->desc.roisize;
    return e->desc.model;
}

int PB200_PoissonNLLAdjoint(Estimator* e, int numspots, const float* d_sample, const float* d_params,
                            const float* d_constants, const float* calib, const float* d_coefs, const float* d_gradOut,
                            float* d_nll, float* d_dparams, float* d_dcalib, void* stream) {
    if (numspots == 0) return 0;
    return guarded(
        [&]() -> int {
            check_estimator(e);
            if (numspots < 0 || !d_sample || !d_params) throw Error("PoissonNLLAdjoint: bad arguments");
            if (e->numconst && !d_constants) throw Error("this estimator needs per-spot constants");
            ModelDesc d = e->desc;
            if (calib) {
                if (d.model == MODEL_XYIBG) {
                    d.sigma[0] = calib[0];
                    d.sigma[1] = calib[1];
                    model_desc_fixed_sigma(d);
                } else if (d.model == MODEL_XYZIBG) {
                    for (int i = 0; i < 5; i++) {
                        d.astig_x[i] = calib[i];
                        d.astig_y[i] = calib[5 + i];
                    }
                }
            }
            if (d_coefs && d.model == MODEL_CSPLINE) {
                d.coefs = d_coefs;
                d.coefsQ = nullptr;  // the caller's coefficients in the reference layout
            }
            AdjointArgs a{};
            a.smp = d_sample;
            a.params = d_params;
            a.consts = d_constants;
            a.gradOut = d_gradOut;
            a.nll = d_nll;
            a.dparams = d_dparams;
            a.dcalib = d_dcalib;
            a.n = numspots;
            adjoint_launcher_for(d.model)(d, a, (cudaStream_t)stream);
            return 0;
        },
        -1);
}

int PB200_SplineCoefGradient(Estimator* e, int numspots, const float* d_sample, const float* d_params,
                             const float* d_coefs, float* d_nll, float* d_grad, float* d_fisherDiag, void* stream) {
    if (numspots == 0) return 0;
    return guarded(
        [&]() -> int {
            check_estimator(e);
            if (e->desc.model != MODEL_CSPLINE) throw Error("SplineCoefGradient: a flat-background spline estimator is needed");
            if (numspots < 0 || !d_sample || !d_params) throw Error("SplineCoefGradient: bad arguments");
            ModelDesc d = e->desc;
            if (d_coefs) {
                d.coefs = d_coefs;
                d.coefsQ = nullptr;  // the caller's coefficients in the reference layout
            }
            AdjointArgs a{};
            a.smp = d_sample;
            a.params = d_params;
            a.nll = d_nll;
            a.dcalib = d_grad;
            a.curv = d_fisherDiag;
            a.n = numspots;
            adjoint_launcher_for(d.model)(d, a, (cudaStream_t)stream);
            return 0;
        },
        -1);
}

// ---- mixed-model, mixed-size batches in one persistent launch ----
}  // extern "C"

#ifndef PB200_MIXED_TWO_LANES
#define PB200_MIXED_TWO_LANES 1
#endif
// ROIs per SM from which a bucket of a mixed plan runs as launches of its own (the single-model
// kernels at their default configuration, on a stream of its own) instead of inside the
// persistent mixed kernel. The single-model kernels fit a ROI faster than the mixed kernel,
// which carries every model's handler in one register budget, and launches on several streams
// share the GPU, so that the small buckets fill it together: on a B200 a 12-bucket batch ran
// 1.03x (4M ROIs) to 1.7x (40k ROIs) faster with every bucket alone than in the persistent
// kernel. Default 0 (every bucket); PB200_SetMixedStandaloneMin changes it for the plans created
// afterwards.
std::atomic<int> g_aloneMinRoisPerSM{0};
// ROIs per SM from which a 7..10 px bucket of a mixed plan runs 2 lanes per ROI (about 4 per
// resident 2-lane group at 2 blocks of 256 threads per SM)
constexpr int kTwoLaneMinRoisPerSM = 1024;

// A bucket of a mixed plan that runs as launches of its own: the LM and Fisher launches of the
// single-model kernel, then the FP64 CRLB.
struct MixedAlone {
    FitLaunch launch = nullptr;
    ModelDesc d{};
    FitArgs a{};  // a.fisher: the plan's Fisher rows; a.claim: the plan's counter of this bucket
    int threads = 0, K = 0;
};

struct MixedPlan {
    int device = 0;
    int ntasks = 0, totalTiles = 0, tileRois = 32, variant = 0, strideFloats = 0;
    std::vector<MixedTask> tasks;  // the buckets of the persistent mixed kernel
    std::vector<int> K;
    std::vector<int> twoLane;      // per task: it runs 2 lanes per ROI
    std::vector<int> bucketLanes;  // per bucket as passed in: lanes per ROI of its launches
    std::vector<MixedAlone> alone;  // the buckets that run as launches of their own
    std::vector<int> bucketAlone;   // per bucket as passed in: 1 if it runs as launches of its own
    DevBuf dTasks, dTasksFisher, dCounter, dFisher;  // dCounter: per-bucket ROI counters of the two passes
    DevBuf dAloneClaims;
    // one stream per bucket that runs alone, forked from the caller's stream and joined back
    std::vector<cudaStream_t> side;
    std::vector<cudaEvent_t> sideDone;
    cudaEvent_t fork = nullptr;
    bool anyFisher = false;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graphExec = nullptr;
    ~MixedPlan() {
        if (graphExec) cudaGraphExecDestroy(graphExec);
        if (graph) cudaGraphDestroy(graph);
        for (cudaStream_t st : side) cudaStreamDestroy(st);
        for (cudaEvent_t ev : sideDone) cudaEventDestroy(ev);
        if (fork) cudaEventDestroy(fork);
    }
};

namespace {
// The persistent mixed kernel's buckets: the LM pass over every bucket, the Fisher pass at the
// fitted parameters (buckets without a CRLB request have no ROIs in it), then the FP64 CRLB of
// each bucket.
void mixed_enqueue_kernel(MixedPlan* p, cudaStream_t s) {
    PB_CUDA(cudaMemsetAsync(p->dCounter.p, 0, 2 * sizeof(int) * p->ntasks, s));
    launch_mixed(p->dTasks.as<MixedTask>(), p->ntasks, p->totalTiles, p->tileRois, p->dCounter.as<int>(),
                 p->strideFloats, p->variant, false, s);
    // A Fisher pass is one trip per ROI, so with one ROI per claim the claims themselves
    // (atomics on a few counters) took a tenth of the LM pass's time on 4M ROIs. Its groups take
    // about eight claims each instead (claims of 1..32 ROIs; 128 resident groups per SM).
    if (p->anyFisher) {
        long long fisherRois = 0;
        for (const MixedTask& t : p->tasks)
            if (t.a.crlb) fisherRois += t.a.n;
        const long long perClaim = fisherRois / (8LL * 128 * num_sms());
        const int chunk = (int)std::min<long long>(32, std::max<long long>(p->tileRois, perClaim));
        launch_mixed(p->dTasksFisher.as<MixedTask>(), p->ntasks, p->totalTiles, chunk,
                     p->dCounter.as<int>() + p->ntasks, p->strideFloats, p->variant, true, s);
    }
    for (int b = 0; b < p->ntasks; b++) {
        const FitArgs& a = p->tasks[b].a;
        if (a.crlb) launch_crlb(p->K[b], a.fisher, a.crlb, a.chisq, a.n, s);
    }
}

// The launches of each bucket that runs alone on a stream of its own, forked from `s`, and on
// `s` the persistent mixed kernel for the others; `s` then waits for the forked streams. The GPU
// runs the launches side by side, so that one bucket's last ROIs share the SMs with another
// bucket's ROIs instead of leaving them idle. In a stream capture the fork and join become graph
// edges.
void mixed_enqueue(MixedPlan* p, cudaStream_t s) {
    if (!p->alone.empty()) PB_CUDA(cudaEventRecord(p->fork, s));
    for (size_t i = 0; i < p->alone.size(); i++) {
        const MixedAlone& m = p->alone[i];
        const cudaStream_t si = p->side[i];
        PB_CUDA(cudaStreamWaitEvent(si, p->fork, 0));
        m.launch(m.d, m.a, m.threads, si);
        if (m.a.crlb) launch_crlb(m.K, m.a.fisher, m.a.crlb, m.a.chisq, m.a.n, si);
        PB_CUDA(cudaEventRecord(p->sideDone[i], si));
    }
    if (p->ntasks) mixed_enqueue_kernel(p, s);
    for (size_t i = 0; i < p->alone.size(); i++) PB_CUDA(cudaStreamWaitEvent(s, p->sideDone[i], 0));
}
}  // namespace

extern "C" {

MixedPlan* PB200_MixedPlanCreate(int nbuckets, Estimator* const* ests, const int* counts, const float* const* d_samples,
                                 const float* const* d_constants, float* const* d_params, int* const* d_iterations,
                                 float* const* d_crlb, float* const* d_chisq, int tileRois, int threadsPerBlock) {
    return guarded(
        [&]() -> MixedPlan* {
            if (nbuckets <= 0 || !ests || !counts || !d_samples || !d_params)
                throw Error("MixedPlanCreate: bad arguments");
            if (tileRois < 1) tileRois = 32;
            auto* p = new MixedPlan();
            try {
                PB_CUDA(cudaGetDevice(&p->device));
                p->tileRois = tileRois;
                // threadsPerBlock picks the kernel variant: 128 (3 blocks/SM, inlined handlers),
                // 256 (2 blocks/SM, separate handlers), 129 (128 threads, 4 blocks/SM, separate handlers)
                p->variant = threadsPerBlock == 256 ? 1 : (threadsPerBlock == 129 ? 2 : 0);
                const int G = mixed_lanes();
                size_t fisherFloats = 0;
                for (int b = 0; b < nbuckets; b++) {
                    Estimator* e = ests[b];
                    check_estimator(e);
                    const int R = e->desc.roisize;
                    const int cpl = (R + G - 1) / G;
                    if (e->desc.model > MODEL_XYZIBG || cpl > 4)
                        throw Error("MixedPlanCreate: buckets must be Gaussian models with ROI size <= 16");
                    if (counts[b] < 0) throw Error("MixedPlanCreate: negative count");
                    if (e->numconst && counts[b] > 0 && (!d_constants || !d_constants[b]))
                        throw Error("MixedPlanCreate: a bucket needs per-spot constants");
                    if (d_crlb && d_crlb[b]) fisherFloats += (size_t)fisher_row_floats(e->K) * counts[b];
                }
                p->dFisher.ensure(sizeof(float) * (fisherFloats ? fisherFloats : 1));
                size_t off = 0;
                std::vector<int> laneOf(nbuckets, G), aloneOf(nbuckets, 0);
                const int aloneMin = g_aloneMinRoisPerSM.load();
                for (int b = 0; b < nbuckets; b++) {
                    Estimator* e = ests[b];
                    if (counts[b] == 0) continue;
                    MixedTask t{};
                    t.d = e->desc;
                    FitArgs& a = t.a;
                    a.smp = d_samples[b];
                    a.consts = d_constants ? d_constants[b] : nullptr;
                    a.params = d_params[b];
                    a.iterations = d_iterations ? d_iterations[b] : nullptr;
                    a.crlb = d_crlb ? d_crlb[b] : nullptr;
                    a.chisq = d_chisq ? d_chisq[b] : nullptr;
                    a.n = counts[b];
                    a.maxIter = e->lm.iterations;
                    a.lambda = e->lm.lambda;
                    if (a.crlb) {
                        a.fisher = p->dFisher.as<float>() + off;
                        off += (size_t)fisher_row_floats(e->K) * counts[b];
                    }
                    const int R = e->desc.roisize;
                    if ((long long)counts[b] >= (long long)aloneMin * num_sms()) {
                        MixedAlone m;
                        int Ga = 0, cpla = 0;
                        gauss_default_shape(e->desc.model, R, Ga, cpla);
                        m.launch = fit_launcher_for(e->desc.model, Ga, cpla, 0);
                        m.d = e->desc;
                        m.a = a;
                        m.threads = Ga == 2 ? 128 : 256;
                        m.K = e->K;
                        p->alone.push_back(m);
                        laneOf[b] = Ga;
                        aloneOf[b] = 1;
                        continue;
                    }
                    const int cpl = (R + G - 1) / G;
                    t.handler = mixed_handler(e->desc.model, G, cpl);
                    p->totalTiles += (counts[b] + tileRois - 1) / tileRois;
                    int base4 = 0;
                    switch (e->K) {
                    case 4: base4 = gauss_group_base_floats<4>(R); break;
                    case 5: base4 = gauss_group_base_floats<5>(R); break;
                    default: base4 = gauss_group_base_floats<6>(R); break;
                    }
                    p->strideFloats = std::max(p->strideFloats, base4);
                    // 7..10 px buckets with at least kTwoLaneMinRoisPerSM ROIs per SM in two 2-lane
                    // groups per 4-lane slot, each with half of the slot (pixels + y-terms or FP64
                    // re-solve scratch; the Fisher pass stores its rows in the plan's scratch, so
                    // neither pass needs in-kernel Fisher scratch). A 2-lane group takes about twice
                    // as long per ROI: with few ROIs per group the last ROIs of a bucket would end
                    // late (a 12-bucket batch of 40k ROIs: 24.2 against 28.8 M/s), with many the
                    // fuller lanes win (4M ROIs: 118.7 against 112.9 M/s).
                    if (PB200_MIXED_TWO_LANES && R >= 7 && R <= 10 &&
                        (long long)counts[b] >= (long long)kTwoLaneMinRoisPerSM * num_sms()) {
                        p->twoLane.push_back(1);
                        laneOf[b] = 2;
                        p->strideFloats = std::max(p->strideFloats,
                                                   2 * round_up(round_up(R * R, 4) + cmax(4 * R, rescue_floats(e->K)), 4));
                    } else {
                        p->twoLane.push_back(0);
                    }
                    p->tasks.push_back(t);
                    p->K.push_back(e->K);
                }
                p->ntasks = (int)p->tasks.size();
                p->bucketLanes = laneOf;
                p->bucketAlone = aloneOf;
                p->dAloneClaims.ensure(sizeof(int) * std::max<size_t>(1, p->alone.size()));
                for (size_t i = 0; i < p->alone.size(); i++) p->alone[i].a.claim = p->dAloneClaims.as<int>() + i;
                if (!p->alone.empty()) PB_CUDA(cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming));
                for (size_t i = 0; i < p->alone.size(); i++) {
                    cudaStream_t st = nullptr;
                    cudaEvent_t ev = nullptr;
                    PB_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
                    p->side.push_back(st);
                    PB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
                    p->sideDone.push_back(ev);
                }
                bool anyTwo = false;
                for (int b = 0; b < p->ntasks; b++) anyTwo = anyTwo || p->twoLane[b];
                {
                    // group stride: of the largest bucket's floats + 0, 4, ..., 28 (multiples of 8 when
                    // 2-lane groups take half a slot each, so that each half stays 16-byte aligned), the
                    // one with the fewest modelled bank conflicts over the buckets, weighted by their
                    // ROI counts
                    const int step = anyTwo ? 8 : 4;
                    const int base = round_up(p->strideFloats, step);
                    long long bestCost = -1;
                    for (int S = base; S < base + 32; S += step) {
                        long long cost = 0;
                        for (int b = 0; b < p->ntasks; b++) {
                            const MixedTask& t = p->tasks[b];
                            const int R = t.d.roisize;
                            if (p->twoLane[b])
                                cost += (long long)t.a.n * gauss_stride_conflicts(S / 2, round_up(R * R, 4), R, 2, (R + 1) / 2);
                            else
                                cost += (long long)t.a.n * gauss_stride_conflicts(S, round_up(R * R, 4), R, G, (R + G - 1) / G);
                        }
                        if (bestCost < 0 || cost < bestCost) {
                            bestCost = cost;
                            p->strideFloats = S;
                        }
                    }
                }
                std::vector<MixedTask> lmTasks(p->tasks), fiTasks(p->tasks);
                for (int b = 0; b < p->ntasks; b++) {
                    if (p->twoLane[b]) {
                        lmTasks[b].handler = mixed_handler(lmTasks[b].d.model, 2, (lmTasks[b].d.roisize + 1) / 2);
                        fiTasks[b].handler = lmTasks[b].handler;
                    }
                    lmTasks[b].a = lm_pass_args(p->tasks[b].a);
                    fiTasks[b].a = fisher_pass_args(p->tasks[b].a);
                    if (!p->tasks[b].a.crlb) fiTasks[b].a.n = 0;  // its tiles end at once
                    else p->anyFisher = true;
                }
                p->dTasks.ensure(sizeof(MixedTask) * std::max(1, p->ntasks));
                p->dTasksFisher.ensure(sizeof(MixedTask) * std::max(1, p->ntasks));
                if (p->ntasks) {
                    PB_CUDA(cudaMemcpy(p->dTasks.p, lmTasks.data(), sizeof(MixedTask) * p->ntasks,
                                       cudaMemcpyHostToDevice));
                    PB_CUDA(cudaMemcpy(p->dTasksFisher.p, fiTasks.data(), sizeof(MixedTask) * p->ntasks,
                                       cudaMemcpyHostToDevice));
                }
                p->dCounter.ensure(2 * sizeof(int) * std::max(1, p->ntasks));
            } catch (...) {
                delete p;
                throw;
            }
            return p;
        },
        (MixedPlan*)nullptr);
}

int PB200_MixedPlanRun(MixedPlan* p, void* stream) {
    return guarded(
        [&]() -> int {
            if (!p) throw Error("MixedPlanRun: null plan");
            if (p->ntasks == 0 && p->alone.empty()) return 0;
            const cudaStream_t s = (cudaStream_t)stream;
            if (p->graphExec) {
                PB_CUDA(cudaGraphLaunch(p->graphExec, s));
                // the graph holds the LM (+ Fisher and CRLB) launches of each bucket that runs
                // alone, the LM and Fisher passes of the mixed kernel and one CRLB kernel per bucket
                for (const MixedAlone& m : p->alone) {
                    count_launch();
                    if (m.a.crlb) {
                        count_launch();
                        count_launch();
                    }
                }
                if (p->ntasks) count_launch();
                if (p->anyFisher) count_launch();
                for (int b = 0; b < p->ntasks; b++)
                    if (p->tasks[b].a.crlb) count_launch();
            } else {
                mixed_enqueue(p, s);
            }
            return 0;
        },
        -1);
}

int PB200_MixedPlanCapture(MixedPlan* p, void* stream) {
    return guarded(
        [&]() -> int {
            if (!p) throw Error("MixedPlanCapture: null plan");
            if (p->ntasks == 0 && p->alone.empty()) return 0;
            const cudaStream_t s = (cudaStream_t)stream;
            if (!s) throw Error("MixedPlanCapture: needs a non-default stream");
            if (p->graphExec) {
                cudaGraphExecDestroy(p->graphExec);
                p->graphExec = nullptr;
            }
            if (p->graph) {
                cudaGraphDestroy(p->graph);
                p->graph = nullptr;
            }
            PB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
            try {
                mixed_enqueue(p, s);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(s, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            PB_CUDA(cudaStreamEndCapture(s, &p->graph));
            PB_CUDA(cudaGraphInstantiate(&p->graphExec, p->graph, 0));
            return 0;
        },
        -1);
}

int PB200_MixedPlanInfo(MixedPlan* p, int* ntasks, int* totalTiles, int* strideFloats) {
    if (!p) return -1;
    if (ntasks) *ntasks = p->ntasks;
    if (totalTiles) *totalTiles = p->totalTiles;
    if (strideFloats) *strideFloats = p->strideFloats;
    return 0;
}

int PB200_MixedPlanLanes(MixedPlan* p, int nbuckets, int* lanes) {
    if (!p || !lanes || nbuckets != (int)p->bucketLanes.size()) return -1;
    for (int b = 0; b < nbuckets; b++) lanes[b] = p->bucketLanes[b];
    return 0;
}

void PB200_SetMixedStandaloneMin(int roisPerSM) { g_aloneMinRoisPerSM.store(roisPerSM < 0 ? 0 : roisPerSM); }
int PB200_GetMixedStandaloneMin(void) { return g_aloneMinRoisPerSM.load(); }

int PB200_StreamedFitProbe(Estimator* e, int numspots, const float* d_sample, float* d_params, int* d_iterations,
                           int markReady) {
    return guarded(
        [&]() -> int {
            check_estimator(e);
            if (numspots <= 0 || !d_sample || !d_params) throw Error("StreamedFitProbe: bad arguments");
            int G = 0, cpl = 0;
            e->fit_shape(G, cpl);
            const StreamLaunch sl = cpl > 0 ? stream_launcher_for(e->desc.model, G, cpl) : nullptr;
            if (!sl) throw Error("StreamedFitProbe: no streamed kernel for this estimator's configuration");
            if (e->numconst) throw Error("StreamedFitProbe: estimators with per-spot constants are not supported");
            std::lock_guard<std::mutex> g(e->mtx);
            const int nblocks = (numspots + (1 << kStreamBlockShift) - 1) >> kStreamBlockShift;
            Slot& ks = e->slot(0);
            e->stFlags.ensure(sizeof(int) * (size_t)(1 + nblocks));
            e->stClaim.ensure(sizeof(int));
            int* flags = e->stFlags.as<int>();
            PB_CUDA(cudaMemsetAsync(flags, 0, sizeof(int), ks.stream));
            PB_CUDA(cudaMemsetAsync(flags + 1, markReady ? 1 : 0, sizeof(int) * (size_t)nblocks, ks.stream));
            FitArgs a{};
            a.smp = d_sample;
            a.params = d_params;
            a.iterations = d_iterations;
            a.n = numspots;
            a.maxIter = e->lm.iterations;
            a.lambda = e->lm.lambda;
            a.claim = e->stClaim.as<int>();
            sl(e->desc, a, flags, e->threads_for(), ks.stream);
            PB_CUDA(cudaStreamSynchronize(ks.stream));
            int err = 0;
            PB_CUDA(cudaMemcpy(&err, flags, sizeof(int), cudaMemcpyDeviceToHost));
            return err ? 1 : 0;
        },
        -1);
}

int PB200_MixedPlanStandalone(MixedPlan* p, int nbuckets, int* standalone) {
    if (!p || !standalone || nbuckets != (int)p->bucketAlone.size()) return -1;
    for (int b = 0; b < nbuckets; b++) standalone[b] = p->bucketAlone[b];
    return 0;
}

void PB200_MixedPlanDestroy(MixedPlan* p) { delete p; }

// ---- allocation-free fused fit + CRLB ----
// Some callers must not allocate device memory while they fit: acquisition software that
// fits frames from a real-time loop with all of its device memory reserved up front (a
// cudaMalloc or cudaFree there can stall until other streams finish, or fail half-way through
// a run), and host frameworks whose memory may only come from their own pools. For them the
// fused path keeps its scratch, the packed Fisher rows and the LM launch's ROI counter, in the
// fixed arrays below.
}  // extern "C"

namespace {
// Largest batch one PB200_EstimateCRLBNoAlloc call accepts.
constexpr int kNoAllocMaxSpots = 32768;
// Packed Fisher matrix of up to K = 6 parameters (21 floats) plus the chi-square.
constexpr int kNoAllocRowFloats = 22;
// 32768 x 22 floats = 2.75 MiB, reserved on every GPU that loads this library until exit.
static __device__ __align__(256) float g_noallocFisher[kNoAllocMaxSpots * kNoAllocRowFloats];
// ROI counter of the LM launch (FitArgs::claim)
static __device__ __align__(16) int g_noallocClaim[4];

// Device addresses of g_noallocFisher and g_noallocClaim on the current device. In host code the
// arrays' names are only host-side stand-ins, so the real addresses are looked up once per
// device, with that device current, and cached.
struct NoAllocScratch {
    float* fisher = nullptr;
    int* claim = nullptr;
};
NoAllocScratch noalloc_scratch() {
    static std::mutex mtx;
    static NoAllocScratch addr[64];
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error("PB200_EstimateCRLBNoAlloc: device index out of range");
    std::lock_guard<std::mutex> g(mtx);
    if (!addr[dev].fisher) {
        void *f = nullptr, *c = nullptr;
        cudaError_t rc = cudaGetSymbolAddress(&f, g_noallocFisher);
        if (rc == cudaSuccess) rc = cudaGetSymbolAddress(&c, g_noallocClaim);
        if (rc != cudaSuccess)
            throw Error(std::string("PB200_EstimateCRLBNoAlloc: cudaGetSymbolAddress failed: ") +
                        cudaGetErrorString(rc));
        addr[dev].claim = static_cast<int*>(c);
        addr[dev].fisher = static_cast<float*>(f);
    }
    return addr[dev];
}
}  // namespace

extern "C" {

int PB200_EstimateCRLBNoAlloc(Estimator* e, int numspots, const float* d_sample, const float* d_constants,
                              const float* d_initial, float* d_params, int* d_iterations, float* d_crlb,
                              float* d_chisq, void* stream) {
    if (numspots == 0) return 0;
    return guarded(
        [&]() -> int {
            check_estimator(e);
            if (numspots < 0 || numspots > kNoAllocMaxSpots)
                throw Error("PB200_EstimateCRLBNoAlloc: numspots must be in [0, " + std::to_string(kNoAllocMaxSpots) +
                            "], got " + std::to_string(numspots) + "; split the batch");
            if (!d_sample || !d_params || !d_crlb) throw Error("PB200_EstimateCRLBNoAlloc: null sample/params/crlb");
            if (e->numconst && !d_constants) throw Error("this estimator needs per-spot constants");
            if (fisher_row_floats(e->K) > kNoAllocRowFloats) throw Error("PB200_EstimateCRLBNoAlloc: too many parameters");
            const NoAllocScratch scratch = noalloc_scratch();
            FitArgs a{};
            a.smp = d_sample;
            a.consts = d_constants;
            a.initial = d_initial;
            a.params = d_params;
            a.iterations = d_iterations;
            a.crlb = d_crlb;
            a.chisq = d_chisq;
            a.fisher = scratch.fisher;
            a.claim = scratch.claim;
            a.n = numspots;
            a.maxIter = e->lm.iterations;
            a.lambda = e->lm.lambda;
            a.flags = 0;
            const cudaStream_t s = (cudaStream_t)stream;
            launch_fit_fisher(e, a, s);
            launch_crlb(e->K, scratch.fisher, d_crlb, d_chisq, numspots, s, e->crlbAbs);
            return 0;
        },
        -1);
}

// ---- loader-time exports ----
int CudaGetNumDevices(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

bool CudaSetDevice(int index) { return cudaSetDevice(index) == cudaSuccess; }

bool CudaGetDeviceInfo(int index, int* numMultiprocessors, char* name, int namelen) {
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, index) != cudaSuccess) return false;
    if (numMultiprocessors) *numMultiprocessors = prop.multiProcessorCount;
    if (name && namelen > 0) {
        strncpy(name, prop.name, namelen - 1);
        name[namelen - 1] = 0;
    }
    return true;
}

void CudaGetMemoryUse(uint64_t* pinnedBytes, uint64_t* devicePitchedBytes, uint64_t* deviceBytes,
                      uint64_t* pitchedNumAllocs) {
    size_t freeB = 0, totalB = 0;
    cudaMemGetInfo(&freeB, &totalB);
    if (pinnedBytes) *pinnedBytes = 0;
    if (devicePitchedBytes) *devicePitchedBytes = 0;
    if (deviceBytes) *deviceBytes = totalB - freeB;
    if (pitchedNumAllocs) *pitchedNumAllocs = 0;
}

void SetDebugPrintCallback(int (*cb)(const char* msg)) { g_debugPrint = cb; }
void SetDebugImageCallback(void (*cb)(int, int, int, const float*, const char*)) { g_debugImage = cb; }
void ShowDebugImage(int w, int h, int numImg, const float* data, const char* title) {
    if (g_debugImage) g_debugImage(w, h, numImg, data, title);
}

static void not_provided(const char* fn) {
    t_lastError = std::string(fn) + " is not provided by photonpy_b200";
    debug_printf("%s\n", t_lastError.c_str());
}
void FFT(const void*, void*, int, int, int) { not_provided("FFT"); }
void FFT2(const void*, void*, int, int, int, int) { not_provided("FFT2"); }
void DrawROIs(float*, int, int, const float*, int, int, const int*) { not_provided("DrawROIs"); }
void Gauss2D_Draw(double*, int, int, float*, int, float) { not_provided("Gauss2D_Draw"); }
void* PSFCorrelationSpotDetector_Configure(const float*, int, int, const float*, int, int, int, float, int, int) {
    not_provided("PSFCorrelationSpotDetector_Configure");
    return nullptr;
}
// GaussianPSF.cu:216-240: intensity and background of each spot at a known position xy[i]
// and width, by the LM fit of mu = I * DeltaX DeltaY + bg from (1, 0) with lambda 1e-15 and
// maxIterations iterations, and their CRLB (sqrt of the |diagonal| of the inverse Fisher
// matrix, inverted here in FP64). As in the reference, spot i's sigma is sigma[i] of the flat array
// (photonpy passes [n][2] floats, so spot i gets element i of that array), and roipos is
// unused. One fused fit + CRLB launch on the current device.
void Gauss2D_EstimateIntensityBg(const float* imageData, float* IBg, float* IBg_crlb, int numspots, const float* xy,
                                 const int* roipos, const float* sigma, int imgw, int maxIterations, bool cuda) {
    (void)roipos;
    (void)cuda;
    if (numspots <= 0) return;
    guarded_void([&]() {
        if (!imageData || !IBg || !xy || !sigma) throw Error("Gauss2D_EstimateIntensityBg: null argument");
        if (imgw < 3 || imgw > 64) throw Error("Gauss2D_EstimateIntensityBg: imgw must be in [3, 64]");
        Estimator e;
        e.desc.model = MODEL_INTENSITYBG;
        e.desc.roisize = imgw;
        e.K = 2;
        e.numconst = 3;
        e.lm = LMParams{maxIterations, 1e-15f, 0.0f};  // LevMarOptimize's default step (Estimation.h:196)
        e.crlbAbs = true;
        std::vector<float> consts((size_t)3 * numspots), init((size_t)2 * numspots);
        for (int i = 0; i < numspots; i++) {
            consts[3 * (size_t)i] = xy[2 * (size_t)i];
            consts[3 * (size_t)i + 1] = xy[2 * (size_t)i + 1];
            consts[3 * (size_t)i + 2] = sigma[i];
            init[2 * (size_t)i] = 1.0f;
            init[2 * (size_t)i + 1] = 0.0f;
        }
        host_fit(&e, numspots, imageData, consts.data(), init.data(), IBg, nullptr, nullptr, 0, IBg_crlb, nullptr, 0);
    });
}
Estimator* Gauss2D_CreatePSF_XYITiltedBg(int roisize, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {
        return make_gauss(MODEL_XYITILTEDBG, roisize, 0, 0, nullptr, nullptr, 0, 0, ctx);
    }, (Estimator*)nullptr);
}
Estimator* Gauss2D_CreatePSF_XYITiltedBgSigmaXY(int roisize, float sx, float sy, bool, Context* ctx) {
    return guarded([&]() -> Estimator* {
        return make_gauss(MODEL_XYITILTEDBG_SIGMAXY, roisize, sx, sy, nullptr, nullptr, 0, 0, ctx);
    }, (Estimator*)nullptr);
}

}  // extern "C"
