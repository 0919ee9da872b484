// Estimation queue: streams ROIs from host memory through the fused fit + CRLB + chi-square
// kernels. Replaces photonpy's Estimators/EstimationQueue.cpp (class at lines 11-314, C API at
// lines 317-420) with the same C API and results.
//
// Layout and flow.
//  * Spots are packed into Batches of batchSize spots, each one pinned host allocation holding
//    ids, samples, constants, roipos, initial values / estimates, CRLB, chi-square and
//    iteration counts (the reference's Batch, EstimationQueue.h:54-66).
//  * A full (or flushed) batch goes to the `todo` list. One worker thread takes the waiting
//    batches in order and launches them on the first free Lane (one CUDA stream with device
//    buffers): all waiting batches with the same initial-value mode, up to the lane's
//    capacity, become ONE fit launch, so small batches (the reference's default is 256 spots)
//    do not each pay a kernel launch and a CRLB launch. Per batch the lane issues one H2D copy
//    per input array into consecutive slices of its device buffers, one
//    PB200_EstimateDevice call over all of them (LM fit, Fisher rows, FP64 CRLB, chi-square),
//    then one D2H copy per output array back into each batch.
//  * Completion is signalled by a host function enqueued behind the copies
//    (cudaLaunchHostFunc): it moves the lane's batches to `finished` and frees the lane under
//    the queue mutex. It makes no CUDA call. Nothing polls.
//  * GetResults copies whole finished batches out and recycles their pinned memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/photonpy_b200.h"
#include "host_internal.h"

namespace {

struct QueueError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define PBQ_CUDA(call)                                                                           \
    do {                                                                                         \
        cudaError_t err_ = (call);                                                               \
        if (err_ != cudaSuccess)                                                                 \
            throw QueueError(std::string("CUDA error: ") + cudaGetErrorString(err_) + " in " #call); \
    } while (0)

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Host side of up to `cap` spots in one pinned allocation.
struct Batch {
    int cap = 0, n = 0;
    bool hasInitial = false;
    void* mem = nullptr;
    int* ids = nullptr;
    float* smp = nullptr;
    float* consts = nullptr;
    int* roipos = nullptr;
    float* params = nullptr;  // initial values on the way in, estimates on the way out
    float* crlb = nullptr;
    float* chisq = nullptr;
    int* iters = nullptr;

    Batch(int cap_, int K, int NC, int npix, int dims) : cap(cap_) {
        size_t off[8], o = 0;
        const size_t sz[8] = {sizeof(int) * cap, sizeof(float) * (size_t)npix * cap, sizeof(float) * (size_t)NC * cap,
                              sizeof(int) * (size_t)dims * cap, sizeof(float) * (size_t)K * cap,
                              sizeof(float) * (size_t)K * cap, sizeof(float) * cap, sizeof(int) * cap};
        for (int i = 0; i < 8; i++) {
            off[i] = o;
            o = align_up(o + sz[i], 256);
        }
        PBQ_CUDA(cudaHostAlloc(&mem, o, cudaHostAllocPortable));
        char* b = static_cast<char*>(mem);
        ids = reinterpret_cast<int*>(b + off[0]);
        smp = reinterpret_cast<float*>(b + off[1]);
        consts = reinterpret_cast<float*>(b + off[2]);
        roipos = reinterpret_cast<int*>(b + off[3]);
        params = reinterpret_cast<float*>(b + off[4]);
        crlb = reinterpret_cast<float*>(b + off[5]);
        chisq = reinterpret_cast<float*>(b + off[6]);
        iters = reinterpret_cast<int*>(b + off[7]);
    }
    ~Batch() {
        if (mem) cudaFreeHost(mem);
    }
    Batch(const Batch&) = delete;
    Batch& operator=(const Batch&) = delete;
};

struct DeviceArray {
    void* p = nullptr;
    DeviceArray() = default;
    DeviceArray(const DeviceArray&) = delete;
    DeviceArray& operator=(const DeviceArray&) = delete;
    void alloc(size_t bytes) { PBQ_CUDA(cudaMalloc(&p, bytes < 256 ? 256 : bytes)); }
    ~DeviceArray() {
        if (p) cudaFree(p);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

}  // namespace

struct EstimQueue;

namespace {

// One CUDA stream with device buffers for up to `cap` spots.
struct Lane {
    EstimQueue* q = nullptr;
    cudaStream_t stream = nullptr;
    DeviceArray smp, consts, initial, params, crlb, chisq, iters;
    std::vector<Batch*> inflight;
    int spots = 0;
    bool busy = false;
    Lane() = default;
    Lane(const Lane&) = delete;
    ~Lane() {
        if (stream) cudaStreamDestroy(stream);
    }
};

}  // namespace

struct EstimQueue {
    Estimator* est = nullptr;
    Context* ctx = nullptr;
    int K = 0, NC = 0, npix = 0, dims = 2;
    int batchSize = 0, limitSpots = 0, launchCap = 0;
    bool keepSamples = false;
    int device = 0;

    std::mutex m;                 // todo, finished, recycle, counters, lanes' busy state
    std::condition_variable cv;   // any change of the above
    std::deque<Batch*> todo, finished, recycle;
    size_t recycleMax = 0;
    long long queuedSpots = 0, activeSpots = 0;
    std::deque<Lane> lanes;  // deque: lanes never move (host functions hold their address)
    bool stop = false;
    std::string failure;  // first error raised on the worker thread, reported once to the user

    std::mutex schedMtx;  // the batch being filled
    Batch* next = nullptr;

    std::thread worker;

    EstimQueue(Estimator* e, int batchSize_, int maxQueueLen, bool keep, int numStreams, Context* c)
        : est(e), ctx(c), batchSize(batchSize_), keepSamples(keep) {
        if (!e) throw QueueError("EstimQueue_Create: estimator is null");
        if (batchSize <= 0) throw QueueError("EstimQueue_Create: batchSize must be positive");
        EstimatorProperties p{};
        Estimator_GetProperties(e, &p);
        K = p.numParams;
        NC = p.numConst;
        npix = p.sampleCount;
        dims = p.sampleIndexDims;
        if (K <= 0 || npix <= 0) throw QueueError("EstimQueue_Create: not a valid estimator");
        if (numStreams < 0) numStreams = 3;  // the reference's default (EstimationQueue.cpp:16-17)
        if (numStreams == 0) numStreams = 1;
        limitSpots = std::max(maxQueueLen, batchSize);
        // Launch capacity: whole batches, at most 64 MiB of samples and 65536 spots per launch.
        const long long bySmp = (64ll << 20) / ((long long)npix * 4 * batchSize);
        const long long byCount = 65536ll / batchSize;
        const long long nb = std::max(1ll, std::min(bySmp, byCount));
        launchCap = (int)(nb * batchSize);
        recycleMax = (size_t)(numStreams * nb + limitSpots / batchSize + 2);
        PBQ_CUDA(cudaGetDevice(&device));
        for (int i = 0; i < numStreams; i++) {
            Lane& L = lanes.emplace_back();
            L.q = this;
            PBQ_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
            const size_t cap = launchCap;
            L.smp.alloc(sizeof(float) * npix * cap);
            if (NC) L.consts.alloc(sizeof(float) * NC * cap);
            L.initial.alloc(sizeof(float) * K * cap);
            L.params.alloc(sizeof(float) * K * cap);
            L.crlb.alloc(sizeof(float) * K * cap);
            L.chisq.alloc(sizeof(float) * cap);
            L.iters.alloc(sizeof(int) * cap);
        }
        worker = std::thread([this]() { run(); });
    }

    ~EstimQueue() {
        cudaSetDevice(device);
        {
            std::lock_guard<std::mutex> g(m);
            stop = true;
        }
        cv.notify_all();
        if (worker.joinable()) worker.join();
        // Work already issued completes (its host functions need `m`, which is free now).
        for (auto& L : lanes)
            if (L.stream) cudaStreamSynchronize(L.stream);
        for (auto* b : todo) delete b;
        for (auto* b : finished) delete b;
        for (auto* b : recycle) delete b;
        delete next;
    }

    // ---------------------------------------------------------------- worker thread
    static void CUDART_CB lane_done(void* arg) {
        Lane* L = static_cast<Lane*>(arg);
        EstimQueue* q = L->q;
        {
            std::lock_guard<std::mutex> g(q->m);
            for (auto* b : L->inflight) q->finished.push_back(b);
            q->activeSpots -= L->spots;
            L->inflight.clear();
            L->spots = 0;
            L->busy = false;
        }
        q->cv.notify_all();
    }

    int free_lane() const {
        for (size_t i = 0; i < lanes.size(); i++)
            if (!lanes[i].busy) return (int)i;
        return -1;
    }

    void run() {
        cudaSetDevice(device);
        std::unique_lock<std::mutex> lk(m);
        for (;;) {
            cv.wait(lk, [&]() { return stop || (!todo.empty() && free_lane() >= 0); });
            if (stop) break;
            Lane& L = lanes[free_lane()];
            const bool init = todo.front()->hasInitial;
            int total = 0;
            while (!todo.empty() && todo.front()->hasInitial == init && total + todo.front()->n <= launchCap) {
                total += todo.front()->n;
                L.inflight.push_back(todo.front());
                todo.pop_front();
            }
            queuedSpots -= total;
            activeSpots += total;
            L.spots = total;
            L.busy = true;
            lk.unlock();
            std::string err;
            try {
                issue(L, total, init);
            } catch (const std::exception& ex) {
                err = ex.what();
            }
            if (!err.empty()) {
                // Nothing of this launch is trusted: wait for what was issued, mark the spots
                // as failed (NaN estimates, 0 iterations) and hand the batches back.
                cudaStreamSynchronize(L.stream);
                cudaGetLastError();
                for (auto* b : L.inflight) {
                    std::fill(b->params, b->params + (size_t)K * b->n, std::numeric_limits<float>::quiet_NaN());
                    std::fill(b->crlb, b->crlb + (size_t)K * b->n, std::numeric_limits<float>::quiet_NaN());
                    std::fill(b->chisq, b->chisq + b->n, std::numeric_limits<float>::quiet_NaN());
                    std::fill(b->iters, b->iters + b->n, 0);
                }
                {
                    std::lock_guard<std::mutex> g(m);
                    if (failure.empty()) failure = "EstimQueue: " + err;
                }
                lane_done(&L);
            }
            lk.lock();
        }
    }

    void issue(Lane& L, int total, bool init) {
        cudaStream_t s = L.stream;
        int off = 0;
        for (auto* b : L.inflight) {
            PBQ_CUDA(cudaMemcpyAsync(L.smp.as<float>() + (size_t)off * npix, b->smp, sizeof(float) * npix * b->n,
                                     cudaMemcpyHostToDevice, s));
            if (NC)
                PBQ_CUDA(cudaMemcpyAsync(L.consts.as<float>() + (size_t)off * NC, b->consts,
                                         sizeof(float) * NC * b->n, cudaMemcpyHostToDevice, s));
            if (init)
                PBQ_CUDA(cudaMemcpyAsync(L.initial.as<float>() + (size_t)off * K, b->params, sizeof(float) * K * b->n,
                                         cudaMemcpyHostToDevice, s));
            off += b->n;
        }
        PB200_ClearError();
        PB200_EstimateDevice(est, total, L.smp.as<float>(), NC ? L.consts.as<float>() : nullptr,
                             init ? L.initial.as<float>() : nullptr, L.params.as<float>(), L.iters.as<int>(), nullptr,
                             0, L.crlb.as<float>(), L.chisq.as<float>(), s);
        const char* msg = PB200_GetLastError();
        if (msg && msg[0]) throw QueueError(msg);
        off = 0;
        for (auto* b : L.inflight) {
            PBQ_CUDA(cudaMemcpyAsync(b->params, L.params.as<float>() + (size_t)off * K, sizeof(float) * K * b->n,
                                     cudaMemcpyDeviceToHost, s));
            PBQ_CUDA(cudaMemcpyAsync(b->crlb, L.crlb.as<float>() + (size_t)off * K, sizeof(float) * K * b->n,
                                     cudaMemcpyDeviceToHost, s));
            PBQ_CUDA(cudaMemcpyAsync(b->chisq, L.chisq.as<float>() + off, sizeof(float) * b->n,
                                     cudaMemcpyDeviceToHost, s));
            PBQ_CUDA(cudaMemcpyAsync(b->iters, L.iters.as<int>() + off, sizeof(int) * b->n, cudaMemcpyDeviceToHost,
                                     s));
            off += b->n;
        }
        PBQ_CUDA(cudaLaunchHostFunc(s, &EstimQueue::lane_done, &L));
    }

    // ---------------------------------------------------------------- user threads
    void report_failure() {
        std::string f;
        {
            std::lock_guard<std::mutex> g(m);
            f.swap(failure);
        }
        if (!f.empty()) pb200::set_last_error(f);
    }

    Batch* take_batch() {
        {
            std::lock_guard<std::mutex> g(m);
            if (!recycle.empty()) {
                Batch* b = recycle.back();
                recycle.pop_back();
                b->n = 0;
                b->hasInitial = false;
                return b;
            }
        }
        return new Batch(batchSize, K, NC, npix, dims);
    }

    // Moves the batch being filled to `todo` (caller holds schedMtx).
    void flush_next() {
        if (!next || next->n == 0) return;
        {
            std::lock_guard<std::mutex> g(m);
            todo.push_back(next);
            queuedSpots += next->n;
        }
        next = nullptr;
        cv.notify_all();
    }

    void schedule(int count, const int* ids, const float* smp, const float* initial, const float* consts,
                  const int* roipos) {
        report_failure();
        if (count < 0) throw QueueError("EstimQueue_Schedule: negative spot count");
        if (count == 0) return;
        if (!smp) throw QueueError("EstimQueue_Schedule: samples is null");
        if (NC && !consts) throw QueueError("EstimQueue_Schedule: this estimator needs per-spot constants");
        {
            // Back-pressure on entry (EstimationQueue.cpp:240-242), in spots.
            std::unique_lock<std::mutex> lk(m);
            cv.wait(lk, [&]() { return queuedSpots + activeSpots < limitSpots || stop; });
        }
        std::lock_guard<std::mutex> g(schedMtx);
        const bool init = initial != nullptr;
        int i = 0;
        while (i < count) {
            if (next && next->n > 0 && next->hasInitial != init) flush_next();
            if (!next) next = take_batch();
            Batch* b = next;
            b->hasInitial = init;
            const int m_ = std::min(b->cap - b->n, count - i);
            const int o = b->n;
            if (ids) std::memcpy(b->ids + o, ids + i, sizeof(int) * m_);
            else std::fill(b->ids + o, b->ids + o + m_, 0);
            std::memcpy(b->smp + (size_t)o * npix, smp + (size_t)i * npix, sizeof(float) * npix * m_);
            if (NC) std::memcpy(b->consts + (size_t)o * NC, consts + (size_t)i * NC, sizeof(float) * NC * m_);
            if (roipos) std::memcpy(b->roipos + (size_t)o * dims, roipos + (size_t)i * dims, sizeof(int) * dims * m_);
            else std::fill(b->roipos + (size_t)o * dims, b->roipos + (size_t)(o + m_) * dims, 0);
            if (init) std::memcpy(b->params + (size_t)o * K, initial + (size_t)i * K, sizeof(float) * K * m_);
            b->n += m_;
            i += m_;
            if (b->n == b->cap) flush_next();
        }
    }

    void flush() {
        report_failure();
        std::lock_guard<std::mutex> g(schedMtx);
        flush_next();
    }

    bool idle() {
        report_failure();
        std::lock_guard<std::mutex> g(m);
        return todo.empty() && activeSpots == 0;
    }

    int result_count() {
        report_failure();
        std::lock_guard<std::mutex> g(m);
        long long total = 0;
        for (auto* b : finished) total += b->n;
        return (int)total;
    }

    int queue_length() {
        report_failure();
        std::lock_guard<std::mutex> g(m);
        return (int)(queuedSpots + activeSpots);
    }

    int results(int maxresults, float* estim, float* diag, float* crlb, int* roipos, float* samples,
                EstimatorResult* res) {
        (void)diag;  // numDiag is 0
        report_failure();
        int copied = 0;
        for (;;) {
            Batch* b = nullptr;
            {
                std::lock_guard<std::mutex> g(m);
                if (finished.empty() || finished.front()->n > maxresults - copied) break;
                b = finished.front();
                finished.pop_front();
            }
            const int n = b->n;
            if (res)
                for (int i = 0; i < n; i++) res[copied + i] = EstimatorResult{b->ids[i], b->chisq[i], b->iters[i]};
            if (estim) std::memcpy(estim + (size_t)copied * K, b->params, sizeof(float) * K * n);
            if (crlb) std::memcpy(crlb + (size_t)copied * K, b->crlb, sizeof(float) * K * n);
            if (roipos) std::memcpy(roipos + (size_t)copied * dims, b->roipos, sizeof(int) * dims * n);
            if (samples && keepSamples) std::memcpy(samples + (size_t)copied * npix, b->smp, sizeof(float) * npix * n);
            copied += n;
            b->n = 0;
            bool keep;
            {
                std::lock_guard<std::mutex> g(m);
                keep = recycle.size() < recycleMax;
                if (keep) recycle.push_back(b);
            }
            if (!keep) delete b;
        }
        return copied;
    }
};

namespace {

template <class F, class R>
R queue_guarded(F&& f, R fallback) {
    try {
        return f();
    } catch (const std::exception& e) {
        pb200::set_last_error(e.what());
        return fallback;
    }
}

void destroy_queue(void* p) { delete static_cast<EstimQueue*>(p); }

}  // namespace

extern "C" {

EstimQueue* EstimQueue_Create(Estimator* psf, int batchSize, int maxQueueLen, bool keepSamples, int numStreams,
                              Context* ctx) {
    return queue_guarded(
        [&]() -> EstimQueue* {
            auto* q = new EstimQueue(psf, batchSize, maxQueueLen, keepSamples, numStreams, ctx);
            pb200::context_attach(ctx, q, &destroy_queue);
            return q;
        },
        (EstimQueue*)nullptr);
}

void EstimQueue_Delete(EstimQueue* q) {
    if (!q) return;
    pb200::context_detach(q->ctx, q);
    delete q;
}

void EstimQueue_Schedule(EstimQueue* q, int numspots, const int* ids, const float* h_samples, const float* h_initial,
                         const float* h_constants, const int* h_roipos) {
    queue_guarded(
        [&]() {
            if (!q) throw QueueError("EstimQueue_Schedule: queue is null");
            q->schedule(numspots, ids, h_samples, h_initial, h_constants, h_roipos);
            return 0;
        },
        0);
}

void EstimQueue_Flush(EstimQueue* q) {
    queue_guarded(
        [&]() {
            if (q) q->flush();
            return 0;
        },
        0);
}

bool EstimQueue_IsIdle(EstimQueue* q) {
    return queue_guarded([&]() { return q ? q->idle() : true; }, true);
}

int EstimQueue_GetResultCount(EstimQueue* q) {
    return queue_guarded([&]() { return q ? q->result_count() : 0; }, 0);
}

int EstimQueue_GetQueueLength(EstimQueue* q) {
    return queue_guarded([&]() { return q ? q->queue_length() : 0; }, 0);
}

int EstimQueue_GetResults(EstimQueue* q, int maxresults, float* estim, float* diag, float* crlb, int* roipos,
                          float* samples, EstimatorResult* results) {
    return queue_guarded(
        [&]() { return q ? q->results(maxresults, estim, diag, crlb, roipos, samples, results) : 0; }, 0);
}

}  // extern "C"
