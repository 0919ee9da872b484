// Estimation queue: streams ROIs from host memory through the fused fit + CRLB + chi-square
// kernels. Replaces photonpy's Estimators/EstimationQueue.cpp (class at lines 11-314, C API at
// lines 317-420) with the same C API and results.
//
// Layout and flow.
//  * Spots are packed into Batches of batchSize spots (the reference's Batch,
//    EstimationQueue.h:54-66). A batch's inputs (samples, constants, initial values) go into a
//    pinned Stage taken from a bounded pool of pinned buffers that are allocated once and
//    reused; its per-spot results live in ordinary host memory. Schedule copies the samples
//    into the stages with a small pool of host threads, one launch-sized window at a time.
//  * A full (or flushed) batch goes to the `todo` list. One worker thread takes the waiting
//    batches in order and launches them on the first free Lane (one CUDA stream with device
//    buffers and pinned result buffers): all waiting batches with the same initial-value mode,
//    up to the lane's capacity, become ONE fit launch, so small batches (the reference's
//    default is 256 spots) do not each pay a kernel launch and a CRLB launch. The lane issues
//    one H2D copy per batch input array into consecutive slices of its device buffers, one
//    PB200_EstimateDeviceDiag call over all of them (LM fit, Fisher rows, FP64 CRLB,
//    chi-square, GLRT diagnostics) and one D2H copy per result array.
//  * Completion is a host function enqueued behind the copies (cudaLaunchHostFunc): it
//    scatters the lane's pinned results into the batches, returns their stages to the pool,
//    moves the batches to `finished` and frees the lane, under the queue mutex. It makes no
//    CUDA call. Nothing polls.
//  * GetResults copies whole finished batches out and recycles them.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <limits>
#include <map>
#include <memory>
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

#define PBQ_CUDA(call)                                                                               \
    do {                                                                                             \
        cudaError_t err_ = (call);                                                                   \
        if (err_ != cudaSuccess)                                                                     \
            throw QueueError(std::string("CUDA error: ") + cudaGetErrorString(err_) + " in " #call); \
    } while (0)

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Process-wide cache of pinned host blocks, keyed by size. Pinning memory costs about as much
// as copying it, so blocks of deleted queues are kept (up to kPinnedCacheBytes) for the next
// queue instead of being returned to the driver.
class PinnedCache {
public:
    static PinnedCache& get() {
        static PinnedCache* c = new PinnedCache();  // never destroyed: outlives every queue
        return *c;
    }
    void* take(size_t bytes) {
        {
            std::lock_guard<std::mutex> g(m_);
            auto it = free_.find(bytes);
            if (it != free_.end()) {
                void* p = it->second;
                free_.erase(it);
                held_ -= bytes;
                return p;
            }
        }
        void* p = nullptr;
        PBQ_CUDA(cudaHostAlloc(&p, bytes, cudaHostAllocPortable));
        return p;
    }
    void give(void* p, size_t bytes) {
        {
            std::lock_guard<std::mutex> g(m_);
            if (held_ + bytes <= kPinnedCacheBytes) {
                free_.emplace(bytes, p);
                held_ += bytes;
                return;
            }
        }
        cudaFreeHost(p);
    }

private:
    static constexpr size_t kPinnedCacheBytes = size_t(2) << 30;
    std::mutex m_;
    std::multimap<size_t, void*> free_;
    size_t held_ = 0;
};

}  // namespace

void* pb200::pinned_take(size_t bytes) { return PinnedCache::get().take(bytes); }
void pb200::pinned_give(void* p, size_t bytes) { PinnedCache::get().give(p, bytes); }

namespace {

// One pinned allocation split into consecutive 256-byte aligned arrays of the given sizes.
struct PinnedBlock {
    void* mem = nullptr;
    size_t bytes = 0;
    std::vector<char*> parts;
    PinnedBlock(std::initializer_list<size_t> sizes) {
        size_t o = 0;
        std::vector<size_t> off;
        for (size_t s : sizes) {
            off.push_back(o);
            o = align_up(o + s, 256);
        }
        bytes = o ? o : 256;
        mem = PinnedCache::get().take(bytes);
        for (size_t x : off) parts.push_back(static_cast<char*>(mem) + x);
    }
    ~PinnedBlock() {
        if (mem) PinnedCache::get().give(mem, bytes);
    }
    PinnedBlock(const PinnedBlock&) = delete;
    PinnedBlock& operator=(const PinnedBlock&) = delete;
    template <class T>
    T* part(int i) const { return reinterpret_cast<T*>(parts[i]); }
};

// Pinned inputs of one batch.
struct Stage {
    PinnedBlock block;
    float* smp;
    float* consts;
    float* initial;
    Stage(int cap, int K, int NC, int npix)
        : block({sizeof(float) * (size_t)npix * cap, sizeof(float) * (size_t)NC * cap, sizeof(float) * (size_t)K * cap}) {
        smp = block.part<float>(0);
        consts = block.part<float>(1);
        initial = block.part<float>(2);
    }
};

// Host side of up to `cap` spots: ids and roipos as scheduled, results after the launch.
struct Batch {
    int n = 0;
    bool hasInitial = false;
    Stage* stage = nullptr;
    std::vector<int> ids, roipos, iters;
    std::vector<float> params, crlb, chisq, diag, samples;
    Batch(int cap, int K, int dims, int numDiag, int npix, bool keepSamples)
        : ids(cap), roipos((size_t)dims * cap), iters(cap), params((size_t)K * cap), crlb((size_t)K * cap),
          chisq(cap), diag((size_t)numDiag * cap) {
        if (keepSamples) samples.resize((size_t)npix * cap);
    }
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

// A fixed set of host threads for the memcpy work of Schedule (the calling thread takes part):
// copying ROIs into pinned staging buffers is the host-side cost of the queue, and one thread
// does not reach the bandwidth of the host's memory.
class CopyPool {
public:
    struct Job {
        void* dst;
        const void* src;
        size_t bytes;
    };

    explicit CopyPool(int threads) {
        for (int i = 1; i < threads; i++) workers_.emplace_back([this]() { worker(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : workers_) t.join();
    }
    CopyPool(const CopyPool&) = delete;
    CopyPool& operator=(const CopyPool&) = delete;

    // Runs every job; returns when all bytes are copied.
    void run(const std::vector<Job>& jobs) {
        size_t total = 0;
        for (const auto& j : jobs) total += j.bytes;
        if (workers_.empty() || total < kSerialBytes) {
            for (const auto& j : jobs) std::memcpy(j.dst, j.src, j.bytes);
            return;
        }
        auto run = std::make_shared<Run>();
        for (const auto& j : jobs)
            for (size_t o = 0; o < j.bytes; o += kPiece)
                run->pieces.push_back({static_cast<char*>(j.dst) + o, static_cast<const char*>(j.src) + o,
                                       std::min(kPiece, j.bytes - o)});
        run->remaining = run->pieces.size();
        {
            std::lock_guard<std::mutex> g(m_);
            current_ = run;
        }
        cv_.notify_all();
        work(*run);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [&]() { return run->remaining == 0; });
        if (current_ == run) current_.reset();
    }

private:
    static constexpr size_t kPiece = 1u << 20;
    static constexpr size_t kSerialBytes = 4u << 20;
    struct Run {
        std::vector<Job> pieces;
        std::atomic<size_t> next{0};
        size_t remaining = 0;  // guarded by m_
    };

    void work(Run& r) {
        size_t done = 0;
        for (;;) {
            const size_t i = r.next.fetch_add(1);
            if (i >= r.pieces.size()) break;
            std::memcpy(r.pieces[i].dst, r.pieces[i].src, r.pieces[i].bytes);
            done++;
        }
        if (done) {
            std::lock_guard<std::mutex> g(m_);
            r.remaining -= done;
            if (r.remaining == 0) done_.notify_all();
        }
    }

    void worker() {
        std::shared_ptr<Run> seen;
        for (;;) {
            std::shared_ptr<Run> r;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&]() { return stop_ || (current_ && current_ != seen); });
                if (stop_) return;
                r = current_;
            }
            seen = r;
            work(*r);
        }
    }

    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    std::shared_ptr<Run> current_;
    bool stop_ = false;
};

}  // namespace

struct EstimQueue;

namespace {

// One CUDA stream with device buffers and pinned result buffers for up to `cap` spots.
struct Lane {
    EstimQueue* q = nullptr;
    cudaStream_t stream = nullptr;
    DeviceArray smp, consts, initial, params, crlb, chisq, iters, diag;
    PinnedBlock* out = nullptr;  // params, crlb, chisq, iters, diag
    std::vector<Batch*> inflight;
    int spots = 0;
    bool busy = false;
    Lane() = default;
    Lane(const Lane&) = delete;
    ~Lane() {
        if (stream) cudaStreamDestroy(stream);
        delete out;
    }
};

}  // namespace

struct EstimQueue {
    Estimator* est = nullptr;
    Context* ctx = nullptr;
    int K = 0, NC = 0, npix = 0, dims = 2, numDiag = 0;
    int batchSize = 0, limitSpots = 0, launchCap = 0, batchesPerLaunch = 1;
    bool keepSamples = false;
    int device = 0;
    std::unique_ptr<CopyPool> copier;

    std::mutex m;                // everything below up to schedMtx
    std::condition_variable cv;  // any change of it
    std::deque<Batch*> todo, finished, recycle;
    size_t recycleMax = 0;
    std::vector<Stage*> stageFree;
    int stageCount = 0, stageMax = 0;
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
        numDiag = p.numDiag;
        if (K <= 0 || npix <= 0) throw QueueError("EstimQueue_Create: not a valid estimator");
        if (numStreams < 0) numStreams = 3;  // the reference's default (EstimationQueue.cpp:16-17)
        if (numStreams == 0) numStreams = 1;
        limitSpots = std::max(maxQueueLen, batchSize);
        // Launch capacity: whole batches, at most 64 MiB of samples and 65536 spots per launch.
        const long long bySmp = (64ll << 20) / ((long long)npix * 4 * batchSize);
        const long long byCount = 65536ll / batchSize;
        batchesPerLaunch = (int)std::max(1ll, std::min(bySmp, byCount));
        launchCap = batchesPerLaunch * batchSize;
        // Pinned stages: enough for every lane's launch plus a full launch waiting, and for
        // the spots the queue limit admits.
        stageMax = std::max((numStreams + 1) * batchesPerLaunch + 2, limitSpots / batchSize + 2);
        recycleMax = (size_t)stageMax;
        const unsigned hw = std::thread::hardware_concurrency();
        copier.reset(new CopyPool((int)std::max(1u, std::min(8u, hw / 2))));
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
            if (numDiag) L.diag.alloc(sizeof(float) * numDiag * cap);
            L.out = new PinnedBlock({sizeof(float) * K * cap, sizeof(float) * K * cap, sizeof(float) * cap,
                                     sizeof(int) * cap, sizeof(float) * numDiag * cap});
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
        auto drop = [&](Batch* b) {
            if (b && b->stage) stageFree.push_back(b->stage);
            delete b;
        };
        for (auto* b : todo) drop(b);
        for (auto* b : finished) drop(b);
        for (auto* b : recycle) drop(b);
        drop(next);
        for (auto* s : stageFree) delete s;
    }

    // ---------------------------------------------------------------- completion
    static void CUDART_CB lane_done(void* arg) {
        Lane* L = static_cast<Lane*>(arg);
        EstimQueue* q = L->q;
        const int K = q->K, ND = q->numDiag;
        const float* hp = L->out->part<float>(0);
        const float* hc = L->out->part<float>(1);
        const float* hx = L->out->part<float>(2);
        const int* hi = L->out->part<int>(3);
        const float* hd = L->out->part<float>(4);
        int off = 0;
        for (auto* b : L->inflight) {
            const int n = b->n;
            std::memcpy(b->params.data(), hp + (size_t)off * K, sizeof(float) * K * n);
            std::memcpy(b->crlb.data(), hc + (size_t)off * K, sizeof(float) * K * n);
            std::memcpy(b->chisq.data(), hx + off, sizeof(float) * n);
            std::memcpy(b->iters.data(), hi + off, sizeof(int) * n);
            if (ND) std::memcpy(b->diag.data(), hd + (size_t)off * ND, sizeof(float) * ND * n);
            off += n;
        }
        q->retire(L);
    }

    // Moves the lane's batches to `finished`, returns their stages and frees the lane.
    void retire(Lane* L) {
        {
            std::lock_guard<std::mutex> g(m);
            for (auto* b : L->inflight) {
                stageFree.push_back(b->stage);
                b->stage = nullptr;
                finished.push_back(b);
            }
            activeSpots -= L->spots;
            L->inflight.clear();
            L->spots = 0;
            L->busy = false;
        }
        cv.notify_all();
    }

    // ---------------------------------------------------------------- worker thread
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
                const float nan = std::numeric_limits<float>::quiet_NaN();
                for (auto* b : L.inflight) {
                    std::fill(b->params.begin(), b->params.end(), nan);
                    std::fill(b->crlb.begin(), b->crlb.end(), nan);
                    std::fill(b->chisq.begin(), b->chisq.end(), nan);
                    std::fill(b->diag.begin(), b->diag.end(), nan);
                    std::fill(b->iters.begin(), b->iters.end(), 0);
                }
                {
                    std::lock_guard<std::mutex> g(m);
                    if (failure.empty()) failure = "EstimQueue: " + err;
                }
                retire(&L);
            }
            lk.lock();
        }
    }

    void issue(Lane& L, int total, bool init) {
        cudaStream_t s = L.stream;
        int off = 0;
        for (auto* b : L.inflight) {
            PBQ_CUDA(cudaMemcpyAsync(L.smp.as<float>() + (size_t)off * npix, b->stage->smp,
                                     sizeof(float) * npix * b->n, cudaMemcpyHostToDevice, s));
            if (NC)
                PBQ_CUDA(cudaMemcpyAsync(L.consts.as<float>() + (size_t)off * NC, b->stage->consts,
                                         sizeof(float) * NC * b->n, cudaMemcpyHostToDevice, s));
            if (init)
                PBQ_CUDA(cudaMemcpyAsync(L.initial.as<float>() + (size_t)off * K, b->stage->initial,
                                         sizeof(float) * K * b->n, cudaMemcpyHostToDevice, s));
            off += b->n;
        }
        PB200_ClearError();
        PB200_EstimateDeviceDiag(est, total, L.smp.as<float>(), NC ? L.consts.as<float>() : nullptr,
                                 init ? L.initial.as<float>() : nullptr, L.params.as<float>(),
                                 numDiag ? L.diag.as<float>() : nullptr, L.iters.as<int>(), L.crlb.as<float>(),
                                 L.chisq.as<float>(), s);
        const char* msg = PB200_GetLastError();
        if (msg && msg[0]) throw QueueError(msg);
        PBQ_CUDA(cudaMemcpyAsync(L.out->part<float>(0), L.params.p, sizeof(float) * K * total,
                                 cudaMemcpyDeviceToHost, s));
        PBQ_CUDA(cudaMemcpyAsync(L.out->part<float>(1), L.crlb.p, sizeof(float) * K * total,
                                 cudaMemcpyDeviceToHost, s));
        PBQ_CUDA(cudaMemcpyAsync(L.out->part<float>(2), L.chisq.p, sizeof(float) * total, cudaMemcpyDeviceToHost, s));
        PBQ_CUDA(cudaMemcpyAsync(L.out->part<int>(3), L.iters.p, sizeof(int) * total, cudaMemcpyDeviceToHost, s));
        if (numDiag)
            PBQ_CUDA(cudaMemcpyAsync(L.out->part<float>(4), L.diag.p, sizeof(float) * numDiag * total,
                                     cudaMemcpyDeviceToHost, s));
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

    // An empty batch with a stage; waits for a stage when the pool is exhausted (the launches
    // in flight return theirs).
    Batch* take_batch() {
        Batch* b = nullptr;
        Stage* st = nullptr;
        bool allocate = false;
        {
            std::unique_lock<std::mutex> lk(m);
            cv.wait(lk, [&]() { return stop || !stageFree.empty() || stageCount < stageMax; });
            if (stop) throw QueueError("EstimQueue: queue is being deleted");
            if (!stageFree.empty()) {
                st = stageFree.back();
                stageFree.pop_back();
            } else {
                stageCount++;
                allocate = true;
            }
            if (!recycle.empty()) {
                b = recycle.back();
                recycle.pop_back();
            }
        }
        try {
            if (allocate) st = new Stage(batchSize, K, NC, npix);
            if (!b) b = new Batch(batchSize, K, dims, numDiag, npix, keepSamples);
        } catch (...) {
            std::lock_guard<std::mutex> g(m);
            if (allocate) stageCount--;
            else stageFree.push_back(st);
            if (b) recycle.push_back(b);
            throw;
        }
        b->n = 0;
        b->hasInitial = false;
        b->stage = st;
        return b;
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
        // Windows of at most one launch (batchesPerLaunch batches, about 64 MiB of samples):
        // take the batches, copy the window's samples with the copy pool, then hand the full
        // batches to the worker in order. A window never holds more stages than one launch, so
        // the stage pool (sized for every lane's launch plus one) cannot run dry inside it.
        int i = 0;
        while (i < count) {
            std::vector<CopyPool::Job> jobs;
            std::vector<Batch*> full;
            int taken = 0;
            while (i < count && taken < batchesPerLaunch) {
                if (next && next->n > 0 && next->hasInitial != init) {
                    full.push_back(next);
                    next = nullptr;
                }
                if (!next) {
                    next = take_batch();
                    taken++;
                }
                Batch* b = next;
                b->hasInitial = init;
                const int m_ = std::min(batchSize - b->n, count - i);
                const int o = b->n;
                if (ids) std::memcpy(b->ids.data() + o, ids + i, sizeof(int) * m_);
                else std::fill(b->ids.begin() + o, b->ids.begin() + o + m_, 0);
                const size_t nb = sizeof(float) * npix * m_;
                jobs.push_back({b->stage->smp + (size_t)o * npix, smp + (size_t)i * npix, nb});
                if (keepSamples) jobs.push_back({b->samples.data() + (size_t)o * npix, smp + (size_t)i * npix, nb});
                if (NC)
                    std::memcpy(b->stage->consts + (size_t)o * NC, consts + (size_t)i * NC, sizeof(float) * NC * m_);
                if (roipos)
                    std::memcpy(b->roipos.data() + (size_t)o * dims, roipos + (size_t)i * dims,
                                sizeof(int) * dims * m_);
                else
                    std::fill(b->roipos.begin() + (size_t)o * dims, b->roipos.begin() + (size_t)(o + m_) * dims, 0);
                if (init)
                    std::memcpy(b->stage->initial + (size_t)o * K, initial + (size_t)i * K, sizeof(float) * K * m_);
                b->n += m_;
                i += m_;
                if (b->n == batchSize) {
                    full.push_back(b);
                    next = nullptr;
                }
            }
            copier->run(jobs);
            if (!full.empty()) {
                long long spots = 0;
                {
                    std::lock_guard<std::mutex> g2(m);
                    for (auto* b : full) {
                        todo.push_back(b);
                        spots += b->n;
                    }
                    queuedSpots += spots;
                }
                cv.notify_all();
            }
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
            if (estim) std::memcpy(estim + (size_t)copied * K, b->params.data(), sizeof(float) * K * n);
            if (crlb) std::memcpy(crlb + (size_t)copied * K, b->crlb.data(), sizeof(float) * K * n);
            if (diag && numDiag)
                std::memcpy(diag + (size_t)copied * numDiag, b->diag.data(), sizeof(float) * numDiag * n);
            if (roipos) std::memcpy(roipos + (size_t)copied * dims, b->roipos.data(), sizeof(int) * dims * n);
            if (samples && keepSamples)
                std::memcpy(samples + (size_t)copied * npix, b->samples.data(), sizeof(float) * npix * n);
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
