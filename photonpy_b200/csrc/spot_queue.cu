// Frame source of the fitter: camera calibration, the ROI queue and the spot-extraction frame
// queue.
//
// Replaces photonpy's CameraCalibration.cu (gain/offset transforms, :9-83), ROIQueue.cpp (a
// thread-safe FIFO of ROIs, :8-95), ImageProcessor.cpp (the ImgProc_* frame-processor ABI,
// :12-51) and the spot-extraction pipeline of ImgFilterQueue.cu (:110-360: raw 16-bit frames ->
// calibration -> sums of `sumframes` frames -> spot detection -> ROIs of the calibrated frames).
//
// B200 layout. The reference moves every frame through a chain of host threads, each with its
// own stream, one frame at a time, and calibrates on the host. Here the frames a caller pushes
// land in a pinned ring; one worker thread takes every complete group of frames waiting (up to
// 64 MB of raw pixels) as one batch: one copy in, one kernel that converts and calibrates, one
// that sums the groups, the batched detector of spot_detect.cu, and one kernel that cuts the
// ROI stacks of all spots of the batch into a packed array, which comes back in one copy. The
// batch grows with the backlog, so launches stay large when frames arrive faster than they are
// processed and latency stays one batch when they do not.
#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/photonpy_b200.h"
#include "host_internal.h"
#include "spot_internal.h"

namespace {

struct FrameQueueError : std::runtime_error {
    using std::runtime_error::runtime_error;
};

#define PBF_CUDA(call)                                                                                   \
    do {                                                                                                 \
        cudaError_t err_ = (call);                                                                       \
        if (err_ != cudaSuccess)                                                                         \
            throw FrameQueueError(std::string("CUDA error: ") + cudaGetErrorString(err_) + " in " #call); \
    } while (0)

template <class F, class R>
R fq_guarded(F&& f, R fallback) {
    try {
        return f();
    } catch (const std::exception& e) {
        pb200::set_last_error(e.what());
        return fallback;
    }
}

// Grow-only device array.
struct DBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t n) {
        if (n <= bytes) return;
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
        PBF_CUDA(cudaMalloc(&p, n < 256 ? 256 : n));
        bytes = n < 256 ? 256 : n;
    }
    ~DBuf() {
        if (p) cudaFree(p);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

// Grow-only pinned host array from the process-wide pinned cache.
struct HBuf {
    void* p = nullptr;
    size_t bytes = 0;
    void ensure(size_t n) {
        if (n <= bytes) return;
        release();
        bytes = n < 256 ? 256 : n;
        p = pb200::pinned_take(bytes);
    }
    void release() {
        if (p) pb200::pinned_give(p, bytes);
        p = nullptr;
        bytes = 0;
    }
    ~HBuf() { release(); }
    template <class T>
    T* as() const { return static_cast<T*>(p); }
};

enum CalibKind { CALIB_NONE = 0, CALIB_GAIN_OFFSET = 1, CALIB_GAIN_OFFSET_IMAGE = 2, CALIB_SCMOS = 3 };

}  // namespace

// ---------------------------------------------------------------------------------------------
// Camera calibration
// ---------------------------------------------------------------------------------------------
struct CameraCalibration {
    int kind = CALIB_NONE;
    float gain = 1.0f, offset = 0.0f;
    int w = 0, h = 0;
    std::vector<float> gainImg, offsetImg;
    Context* ctx = nullptr;
    std::mutex mtx;
    int dev = -1;
    DBuf dGain, dOffset;  // device copies of the images on `dev`

    // Device copies of the per-pixel images on the current device (uploaded on first use).
    void device_images(const float** g, const float** o) {
        std::lock_guard<std::mutex> lk(mtx);
        int cur = 0;
        PBF_CUDA(cudaGetDevice(&cur));
        if (dev != cur) {
            if (dev >= 0) throw FrameQueueError("camera calibration: used on a second device");
            const size_t n = sizeof(float) * (size_t)w * h;
            dGain.ensure(n);
            dOffset.ensure(n);
            PBF_CUDA(cudaMemcpy(dGain.p, gainImg.data(), n, cudaMemcpyHostToDevice));
            PBF_CUDA(cudaMemcpy(dOffset.p, offsetImg.data(), n, cudaMemcpyHostToDevice));
            dev = cur;
        }
        *g = dGain.as<float>();
        *o = dOffset.as<float>();
    }
};

namespace {

// CameraCalibration.cu:19-57 per pixel, in the reference's operation order (subtract, then
// multiply, each rounded; negative results of the gain/offset transforms set to 0).
template <class T>
__global__ void calib_kernel(const T* __restrict__ in, float* __restrict__ out, int npix, int kind, float gain,
                             float offset, const float* __restrict__ gimg, const float* __restrict__ oimg) {
    const size_t base = (size_t)blockIdx.y * npix;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        float v = (float)in[base + p];
        if (kind == CALIB_GAIN_OFFSET) {
            v = __fmul_rn(__fsub_rn(v, offset), gain);
            if (v < 0.0f) v = 0.0f;
        } else if (kind == CALIB_GAIN_OFFSET_IMAGE) {
            v = __fmul_rn(__fsub_rn(v, oimg[p]), gimg[p]);
            if (v < 0.0f) v = 0.0f;
        } else if (kind == CALIB_SCMOS) {
            v = __fmul_rn(__fsub_rn(v, oimg[p]), gimg[p]);
        }
        out[base + p] = v;
    }
}

template <class T>
void calib_launch(const CameraCalibration* c, const T* d_in, float* d_out, int w, int h, int n, cudaStream_t s) {
    if (n <= 0) return;
    if (n > 65535) throw FrameQueueError("camera calibration: at most 65535 frames per call");
    const int npix = w * h;
    int kind = c ? c->kind : CALIB_NONE;
    const float* g = nullptr;
    const float* o = nullptr;
    if (kind == CALIB_GAIN_OFFSET_IMAGE || kind == CALIB_SCMOS) {
        if (c->w != w || c->h != h)
            throw FrameQueueError("camera calibration: image size " + std::to_string(c->w) + "x" + std::to_string(c->h) +
                                  " does not match the frames (" + std::to_string(w) + "x" + std::to_string(h) + ")");
        const_cast<CameraCalibration*>(c)->device_images(&g, &o);
    }
    const int threads = 256;
    const int bx = std::min((npix + threads - 1) / threads, 1024);
    calib_kernel<T><<<dim3(bx, n), threads, 0, s>>>(d_in, d_out, npix, kind, c ? c->gain : 1.0f,
                                                     c ? c->offset : 0.0f, g, o);
    PBF_CUDA(cudaGetLastError());
}

}  // namespace

void pb200::camera_calib_apply_f32(const CameraCalibration* c, const float* d_in, float* d_out, int w, int h, int n,
                                   cudaStream_t s) {
    calib_launch<float>(c, d_in, d_out, w, h, n, s);
}

void pb200::camera_calib_apply_u16(const CameraCalibration* c, const uint16_t* d_in, float* d_out, int w, int h,
                                   int n, cudaStream_t s) {
    calib_launch<uint16_t>(c, d_in, d_out, w, h, n, s);
}

// ---------------------------------------------------------------------------------------------
// ROI queue
// ---------------------------------------------------------------------------------------------
struct ROIQueue {
    int shape[3];  // z, y, x
    size_t smp;
    Context* ctx = nullptr;
    // ROIs in blocks of consecutive entries; the front block is consumed from `first`
    struct Block {
        std::vector<ROIInfo> info;
        std::vector<float> data;
        size_t first = 0;
    };
    std::mutex mtx;
    std::deque<Block> blocks;
    size_t length = 0;

    void push(int count, const ROIInfo* info, const float* data) {
        if (count <= 0) return;
        std::lock_guard<std::mutex> lk(mtx);
        if (blocks.empty() || blocks.back().info.size() >= 4096) blocks.emplace_back();
        Block& b = blocks.back();
        b.info.insert(b.info.end(), info, info + count);
        b.data.insert(b.data.end(), data, data + smp * count);
        length += count;
    }

    // ROIQueue::PopROIs (ROIQueue.cpp:33-52): the `count` oldest, written newest first.
    void pop(int count, ROIInfo* dst, float* data) {
        if (count <= 0) return;
        std::lock_guard<std::mutex> lk(mtx);
        if ((size_t)count > length) return;
        for (int i = 0; i < count; i++) {
            Block& b = blocks.front();
            const int o = count - 1 - i;
            if (dst) dst[o] = b.info[b.first];
            if (data) std::memcpy(data + smp * o, b.data.data() + smp * b.first, sizeof(float) * smp);
            if (++b.first == b.info.size()) blocks.pop_front();
        }
        length -= count;
    }

    int len() {
        std::lock_guard<std::mutex> lk(mtx);
        return (int)length;
    }
};

// ---------------------------------------------------------------------------------------------
// Frame processors
// ---------------------------------------------------------------------------------------------
struct ImageProcessor {
    Context* ctx = nullptr;
    virtual ~ImageProcessor() {}
    virtual void AddFrameU16(const uint16_t* data) = 0;
    virtual void AddFrameF32(const float* data) = 0;
    virtual int GetQueueLength() = 0;
    virtual int NumFinishedFrames() { return 0; }
    virtual int ReadFrame(float*, float*) { return 0; }
    virtual bool IsIdle() = 0;
    virtual void Flush() {}
};

namespace {

// Sum of each group of sf consecutive frames, left to right (ImgFilterQueue.cu:229-236).
__global__ void sum_groups_kernel(const float* __restrict__ frames, float* __restrict__ sums, int sf, int npix) {
    const int g = blockIdx.y;
    const float* src = frames + (size_t)g * sf * npix;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        float v = src[p];
        for (int z = 1; z < sf; z++) v = __fadd_rn(v, src[(size_t)z * npix + p]);
        sums[(size_t)g * npix + p] = v;
    }
}

// One warp per spot: spot i of summed frame g goes to slot offsets[g] + i of the packed outputs,
// with its corner (x, y) = centre - roi size / 2 and the ROI stack [sf][rh][rw] of the group's
// calibrated frames, coordinates clamped to the frame (ImgFilterQueue.cu:176-201).
__global__ void cut_stacks_kernel(const float* __restrict__ frames, int w, int h, int sf, int rw, int rh, int groups,
                                  int C, const int* __restrict__ found, const int* __restrict__ offsets,
                                  const int* __restrict__ index, const float* __restrict__ score,
                                  int* __restrict__ cornerXY, float* __restrict__ scoreOut,
                                  float* __restrict__ rois) {
    const long long task = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (task >= (long long)groups * C) return;
    const int g = (int)(task / C), i = (int)(task % C);
    if (i >= found[g]) return;
    const int pix = index[(size_t)g * C + i];
    const int cx = pix % w - rw / 2, cy = pix / w - rh / 2;
    const int o = offsets[g] + i;
    if (lane == 0) {
        cornerXY[2 * (size_t)o] = cx;
        cornerXY[2 * (size_t)o + 1] = cy;
        scoreOut[o] = score[(size_t)g * C + i];
    }
    const int per = rw * rh;
    float* dst = rois + (size_t)o * sf * per;
    const float* src = frames + (size_t)g * sf * w * h;
    for (int q = lane; q < sf * per; q += 32) {
        const int z = q / per, r = q - z * per;
        const int fy = min(max(cy + r / rw, 0), h - 1), fx = min(max(cx + r % rw, 0), w - 1);
        dst[q] = __ldg(src + (size_t)z * w * h + (size_t)fy * w + fx);
    }
}

// Pinned ring of raw 16-bit frames and the worker thread that takes every complete unit of
// `group` frames waiting (up to 64 MB of raw pixels) and hands them to process(), the
// derived queue's GPU batch. Units are numbered from 0 in push order.
class FrameRing : public ImageProcessor {
   public:
    FrameRing(int w, int h, int group, const char* name)
        : w_(w), h_(h), npix_((size_t)w * h), group_(group), name_(name) {
        if (w < 1 || h < 1 || npix_ >= (1u << 31)) throw FrameQueueError(std::string(name) + ": bad frame size");
        if (group < 1) throw FrameQueueError(std::string(name) + ": bad group size");
        PBF_CUDA(cudaGetDevice(&dev_));
        const size_t frameBytes = sizeof(uint16_t) * npix_;
        int bmax = (int)std::min<size_t>(4096, std::max<size_t>(1, (size_t(64) << 20) / frameBytes));
        bmax = std::max(group_, bmax / group_ * group_);
        bmax = std::min(bmax, 65535 / group_ * group_);  // kernel grid limit on frames per launch
        maxUnits_ = bmax / group_;
        cap_ = 2 * bmax;  // the ring holds two batches
        ringBytes_ = frameBytes * cap_;
        ring_ = static_cast<uint16_t*>(pb200::pinned_take(ringBytes_));
        PBF_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    }

    ~FrameRing() override {
        stop_worker();
        if (stream_) cudaStreamDestroy(stream_);
        if (ring_) pb200::pinned_give(ring_, ringBytes_);
    }

    void AddFrameU16(const uint16_t* data) override {
        if (!data) throw FrameQueueError("ImgProc_AddFrameU16: null frame");
        std::unique_lock<std::mutex> lk(mtx_);
        cvSpace_.wait(lk, [&]() { return count_ < cap_ || stop_; });
        if (stop_) return;
        const int slot = (head_ + count_) % cap_;
        std::memcpy(ring_ + (size_t)slot * npix_, data, sizeof(uint16_t) * npix_);
        count_++;
        cvWork_.notify_one();
    }

    void AddFrameF32(const float*) override {
        throw FrameQueueError(name_ + ": float frames are not accepted (16-bit frames only)");
    }

    int GetQueueLength() override {
        std::lock_guard<std::mutex> lk(mtx_);
        return count_;
    }

    int NumFinishedFrames() override {
        std::lock_guard<std::mutex> lk(mtx_);
        return finished_;
    }

    bool IsIdle() override {
        std::lock_guard<std::mutex> lk(mtx_);
        return !busy_ && count_ / group_ == 0;
    }

   protected:
    // Starts the worker; the derived constructor calls it last.
    void start_worker() {
        worker_ = std::thread([this]() { run(); });
    }
    // Stops the worker after its current batch; the derived destructor calls it first, so that
    // process() never runs on a half-destroyed object.
    void stop_worker() {
        {
            std::lock_guard<std::mutex> lk(mtx_);
            stop_ = true;
        }
        cvWork_.notify_all();
        cvSpace_.notify_all();
        if (worker_.joinable()) worker_.join();
    }
    // Raw frames of units [unitBase, unitBase + units) at ring_ + first * npix_ (contiguous).
    virtual void process(int first, int units, int unitBase) = 0;

    int w_, h_;
    size_t npix_;
    int group_;
    std::string name_;
    int dev_ = 0;
    cudaStream_t stream_ = nullptr;
    uint16_t* ring_ = nullptr;  // [head_, head_ + count_) waiting, modulo cap_

   private:
    void run() {
        cudaSetDevice(dev_);
        while (true) {
            int first, units, unitBase;
            {
                std::unique_lock<std::mutex> lk(mtx_);
                cvWork_.wait(lk, [&]() { return stop_ || count_ / group_ > 0; });
                if (stop_) return;
                first = head_;
                units = std::min({count_ / group_, maxUnits_, (cap_ - head_) / group_});
                unitBase = finished_;
                busy_ = true;
            }
            try {
                process(first, units, unitBase);
            } catch (const std::exception& e) {
                pb200::set_last_error(name_ + ": " + e.what() + " (frames dropped)");
                cudaStreamSynchronize(stream_);
            }
            {
                std::lock_guard<std::mutex> lk(mtx_);
                head_ = (head_ + units * group_) % cap_;
                count_ -= units * group_;
                finished_ += units;
                busy_ = false;
            }
            cvSpace_.notify_all();
        }
    }

    size_t ringBytes_ = 0;
    int cap_ = 0, head_ = 0, count_ = 0, maxUnits_ = 1;
    int finished_ = 0;
    bool busy_ = false, stop_ = false;
    std::mutex mtx_;
    std::condition_variable cvWork_, cvSpace_;
    std::thread worker_;
};

class SpotExtractionQueue : public FrameRing {
   public:
    SpotExtractionQueue(int w, int h, ROIQueue* out, const SpotDetectorConfig& cfg, CameraCalibration* calib)
        : FrameRing(w, h, out->shape[0], "SpotExtractionQueue"), out_(out), calib_(calib) {
        sf_ = out->shape[0];
        rh_ = out->shape[1];
        rw_ = out->shape[2];
        if (rh_ < 1 || rw_ < 1) throw FrameQueueError("SpotExtractionQueue: bad ROI queue shape");
        SpotDetectorConfig c = cfg;
        if (cfg.backgroundImage) {  // copied now: the caller's array need not outlive the queue
            dBg_.ensure(sizeof(float) * npix_);
            PBF_CUDA(cudaMemcpy(dBg_.p, cfg.backgroundImage, sizeof(float) * npix_, cudaMemcpyHostToDevice));
        }
        c.backgroundImage = nullptr;
        det_ = SpotDetector_Configure(&c);
        if (!det_) throw FrameQueueError("SpotExtractionQueue: detector configuration failed");
        start_worker();
    }

    ~SpotExtractionQueue() override {
        stop_worker();
        if (det_) SpotDetector_DestroyFactory(det_);
    }

   private:
    void process(int first, int groups, int idBase) {
        const int nf = groups * sf_;
        const size_t npix = npix_;
        dRaw_.ensure(sizeof(uint16_t) * npix * nf);
        dOrig_.ensure(sizeof(float) * npix * nf);
        PBF_CUDA(cudaMemcpyAsync(dRaw_.p, ring_ + (size_t)first * npix, sizeof(uint16_t) * npix * nf,
                                 cudaMemcpyHostToDevice, stream_));
        pb200::camera_calib_apply_u16(calib_, dRaw_.as<uint16_t>(), dOrig_.as<float>(), w_, h_, nf, stream_);
        const float* dDet = dOrig_.as<float>();
        if (sf_ > 1) {
            dSum_.ensure(sizeof(float) * npix * groups);
            const int bx = (int)std::min<size_t>((npix + 255) / 256, 1024);
            sum_groups_kernel<<<dim3(bx, groups), 256, 0, stream_>>>(dOrig_.as<float>(), dSum_.as<float>(), sf_,
                                                                      (int)npix);
            PBF_CUDA(cudaGetLastError());
            dDet = dSum_.as<float>();
        }
        dFound_.ensure(sizeof(int) * groups);
        hFound_.ensure(sizeof(int) * groups);
        int* hf = hFound_.as<int>();
        // the detector keeps the first C spots of a frame; the reference keeps all, so a batch
        // with a fuller frame runs again with a larger C
        while (true) {
            dIndex_.ensure(sizeof(int) * (size_t)C_ * groups);
            dScore_.ensure(sizeof(float) * (size_t)C_ * groups);
            pb200::spot_detect_indices(det_, dDet, dBg_.as<float>(), groups, w_, h_, C_, dFound_.as<int>(),
                                       dIndex_.as<int>(), dScore_.as<float>(), stream_);
            PBF_CUDA(cudaMemcpyAsync(hf, dFound_.p, sizeof(int) * groups, cudaMemcpyDeviceToHost, stream_));
            PBF_CUDA(cudaStreamSynchronize(stream_));
            int mx = 0;
            for (int g = 0; g < groups; g++) mx = std::max(mx, hf[g]);
            if (mx <= C_) break;
            while (C_ < mx) C_ *= 2;
        }
        std::vector<int> offsets(groups);
        long long total = 0;
        for (int g = 0; g < groups; g++) {
            offsets[g] = (int)total;
            total += hf[g];
        }
        if (total > (1LL << 30)) throw FrameQueueError("too many spots in one batch");
        if (total == 0) return;
        const size_t per = (size_t)sf_ * rh_ * rw_;
        dOffsets_.ensure(sizeof(int) * groups);
        dCorner_.ensure(sizeof(int) * 2 * total);
        dScoreOut_.ensure(sizeof(float) * total);
        dRois_.ensure(sizeof(float) * per * total);
        hCorner_.ensure(sizeof(int) * 2 * total);
        hScore_.ensure(sizeof(float) * total);
        hRois_.ensure(sizeof(float) * per * total);
        PBF_CUDA(cudaMemcpyAsync(dOffsets_.p, offsets.data(), sizeof(int) * groups, cudaMemcpyHostToDevice, stream_));
        const long long tasks = (long long)groups * C_;
        const int blocks = (int)std::min<long long>((tasks + 7) / 8, 1 << 30);
        cut_stacks_kernel<<<blocks, 256, 0, stream_>>>(dOrig_.as<float>(), w_, h_, sf_, rw_, rh_, groups, C_,
                                                       dFound_.as<int>(), dOffsets_.as<int>(), dIndex_.as<int>(),
                                                       dScore_.as<float>(), dCorner_.as<int>(),
                                                       dScoreOut_.as<float>(), dRois_.as<float>());
        PBF_CUDA(cudaGetLastError());
        PBF_CUDA(cudaMemcpyAsync(hCorner_.p, dCorner_.p, sizeof(int) * 2 * total, cudaMemcpyDeviceToHost, stream_));
        PBF_CUDA(cudaMemcpyAsync(hScore_.p, dScoreOut_.p, sizeof(float) * total, cudaMemcpyDeviceToHost, stream_));
        PBF_CUDA(cudaMemcpyAsync(hRois_.p, dRois_.p, sizeof(float) * per * total, cudaMemcpyDeviceToHost, stream_));
        PBF_CUDA(cudaStreamSynchronize(stream_));
        info_.resize((size_t)total);
        const int* hc = hCorner_.as<int>();
        const float* hs = hScore_.as<float>();
        for (int g = 0; g < groups; g++) {
            for (int i = 0; i < hf[g]; i++) {
                const int o = offsets[g] + i;
                ROIInfo& r = info_[o];
                r.id = idBase + g;
                r.score = hs[o];
                r.x = hc[2 * o];
                r.y = hc[2 * o + 1];
                r.z = 0;
            }
        }
        out_->push((int)total, info_.data(), hRois_.as<float>());
    }

    int sf_ = 1, rh_ = 1, rw_ = 1;
    ROIQueue* out_;
    CameraCalibration* calib_;
    SpotDetectorFactory* det_ = nullptr;
    int C_ = 256;  // spot slots per summed frame in the detector outputs
    DBuf dBg_, dRaw_, dOrig_, dSum_, dFound_, dIndex_, dScore_, dOffsets_, dCorner_, dScoreOut_, dRois_;
    HBuf hFound_, hCorner_, hScore_, hRois_;
    std::vector<ROIInfo> info_;
};

// Gathers the ROI pixels of a batch: task t copies the roisize x roisize box at corner
// (x, y) = (task.x, task.y) of frame task.z of the batch (coordinates clamped to the frame)
// into out[t]. One warp per task.
__global__ void gather_boxes_kernel(const float* __restrict__ frames, int w, int h, int roisize,
                                    const int4* __restrict__ tasks, int ntasks, float* __restrict__ out) {
    const long long t = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    if (t >= ntasks) return;
    const int lane = threadIdx.x & 31;
    const int4 k = tasks[t];
    const float* src = frames + (size_t)k.z * w * h;
    float* dst = out + (size_t)t * roisize * roisize;
    for (int q = lane; q < roisize * roisize; q += 32) {
        const int fy = min(max(k.y + q / roisize, 0), h - 1), fx = min(max(k.x + q % roisize, 0), w - 1);
        dst[q] = __ldg(src + (size_t)fy * w + fx);
    }
}

// The ROI extractor (ImageProcessor.cpp:61-233): 16-bit frames in (calibrated like the spot
// queue's), and for each requested ROI the boxes of its numframes frames from startframe on,
// collected into one record that becomes available once its last frame has been processed.
// Records come out in the order the reference hands them out: by last frame, then by start
// frame, then in request order. As a difference, box coordinates are clamped to the frame
// (the reference reads outside the frame for boxes that cross its border).
class ROIExtractorQueue : public FrameRing {
   public:
    ROIExtractorQueue(int w, int h, const ExtractionROI* rois, int n, int roiframes, int roisize,
                      CameraCalibration* calib)
        : FrameRing(w, h, 1, "ROIExtractor"), roiframes_(roiframes), rs_(roisize), calib_(calib) {
        if (n < 0 || (n > 0 && !rois) || roisize < 1 || roiframes < 0)
            throw FrameQueueError("ROIExtractor_Create: bad arguments");
        spots_.resize(n);
        int last = -1;
        for (int i = 0; i < n; i++) {
            if (rois[i].startframe < 0) throw FrameQueueError("ROIExtractor_Create: negative startframe");
            spots_[i].roi = rois[i];  // its pixel buffer is allocated when its first box arrives
            last = std::max(last, rois[i].startframe);
        }
        // activation order: by start frame, then request order (a stable sort)
        order_.resize(n);
        for (int i = 0; i < n; i++) order_[i] = i;
        std::stable_sort(order_.begin(), order_.end(),
                         [&](int a, int b) { return rois[a].startframe < rois[b].startframe; });
        start_worker();
    }

    ~ROIExtractorQueue() override { stop_worker(); }

    int result_count() {
        std::lock_guard<std::mutex> lk(resMtx_);
        return (int)results_.size();
    }

    // ROIExtractor::GetResults (ImageProcessor.cpp:105-126): up to n records, oldest first; slot
    // i of framedata holds roiframes boxes, of which min(numframes, roiframes) are written.
    int results(int n, ExtractionROI* rois, float* framedata) {
        std::vector<int> take;
        {
            std::lock_guard<std::mutex> lk(resMtx_);
            while ((int)take.size() < n && !results_.empty()) {
                take.push_back(results_.front());
                results_.pop_front();
            }
        }
        const size_t box = (size_t)rs_ * rs_;
        for (size_t i = 0; i < take.size(); i++) {
            Spot& sp = spots_[take[i]];
            if (rois) rois[i] = sp.roi;
            if (framedata && !sp.data.empty()) {
                const int nf = std::min(std::max(0, sp.roi.numframes), roiframes_);
                std::memcpy(framedata + (size_t)roiframes_ * box * i, sp.data.data(), sizeof(float) * box * nf);
            }
            std::vector<float>().swap(sp.data);  // handed out
        }
        return (int)take.size();
    }

   private:
    struct Spot {
        ExtractionROI roi;
        std::vector<float> data;  // [numframes][roisize][roisize]
    };

    void process(int first, int units, int frameBase) override {
        const int nf = units;
        const size_t npix = npix_;
        dRaw_.ensure(sizeof(uint16_t) * npix * nf);
        dFrames_.ensure(sizeof(float) * npix * nf);
        PBF_CUDA(cudaMemcpyAsync(dRaw_.p, ring_ + (size_t)first * npix, sizeof(uint16_t) * npix * nf,
                                 cudaMemcpyHostToDevice, stream_));
        pb200::camera_calib_apply_u16(calib_, dRaw_.as<uint16_t>(), dFrames_.as<float>(), w_, h_, nf, stream_);
        // boxes wanted from these frames, in activation order
        const int f0 = frameBase, f1 = frameBase + nf;
        const int n = (int)order_.size();
        while (live_ < n && last_frame(spots_[order_[live_]].roi) < f0) live_++;  // done before this batch
        tasks_.clear();
        dest_.clear();
        for (int o = live_; o < n; o++) {
            const int i = order_[o];
            const ExtractionROI& r = spots_[i].roi;
            if (r.startframe >= f1) break;  // order_ is sorted by start frame
            const int lo = std::max(r.startframe, f0), hi = std::min(r.startframe + r.numframes, f1);
            for (int f = lo; f < hi; f++) {
                tasks_.push_back(make_int4(r.cornerpos[0], r.cornerpos[1], f - f0, 0));
                dest_.push_back({i, f - r.startframe});
            }
        }
        const int T = (int)tasks_.size();
        const size_t box = (size_t)rs_ * rs_;
        if (T > 0) {
            dTasks_.ensure(sizeof(int4) * T);
            dBoxes_.ensure(sizeof(float) * box * T);
            hBoxes_.ensure(sizeof(float) * box * T);
            PBF_CUDA(cudaMemcpyAsync(dTasks_.p, tasks_.data(), sizeof(int4) * T, cudaMemcpyHostToDevice, stream_));
            gather_boxes_kernel<<<(T + 7) / 8, 256, 0, stream_>>>(dFrames_.as<float>(), w_, h_, rs_,
                                                                 dTasks_.as<int4>(), T, dBoxes_.as<float>());
            PBF_CUDA(cudaGetLastError());
            PBF_CUDA(cudaMemcpyAsync(hBoxes_.p, dBoxes_.p, sizeof(float) * box * T, cudaMemcpyDeviceToHost,
                                     stream_));
        }
        PBF_CUDA(cudaStreamSynchronize(stream_));  // also keeps the ring slots until the copy is done
        const float* hb = hBoxes_.as<float>();
        for (int t = 0; t < T; t++) {
            Spot& sp = spots_[dest_[t].first];
            if (sp.data.empty()) sp.data.assign((size_t)sp.roi.numframes * box, 0.0f);
            std::memcpy(sp.data.data() + box * dest_[t].second, hb + box * t, sizeof(float) * box);
        }
        // records complete at frame startframe + max(numframes, 1) - 1: hand them out frame by
        // frame, each frame's in activation order
        std::lock_guard<std::mutex> lk(resMtx_);
        for (int f = f0; f < f1; f++)
            for (int o = live_; o < n; o++) {
                const int i = order_[o];
                const ExtractionROI& r = spots_[i].roi;
                if (r.startframe > f) break;
                if (last_frame(r) == f) results_.push_back(i);
            }
    }

    static int last_frame(const ExtractionROI& r) { return r.startframe + std::max(r.numframes, 1) - 1; }

    int roiframes_, rs_;
    CameraCalibration* calib_;
    std::vector<Spot> spots_;
    std::vector<int> order_;
    int live_ = 0;  // order_[0, live_) are complete
    std::vector<int4> tasks_;
    std::vector<std::pair<int, int>> dest_;  // (spot, frame within the spot) of each task
    std::mutex resMtx_;
    std::deque<int> results_;
    DBuf dRaw_, dFrames_, dTasks_, dBoxes_;
    HBuf hBoxes_;
};

void destroy_calib(void* p) { delete static_cast<CameraCalibration*>(p); }
void destroy_roiqueue(void* p) { delete static_cast<ROIQueue*>(p); }
void destroy_imgproc(void* p) { delete static_cast<ImageProcessor*>(p); }

CameraCalibration* calib_register(CameraCalibration* c, Context* ctx) {
    c->ctx = ctx;
    pb200::context_attach(ctx, c, destroy_calib);
    return c;
}

}  // namespace

extern "C" {

CameraCalibration* GainOffsetCalib_Create(float gain, float offset, Context* ctx) {
    return fq_guarded(
        [&]() -> CameraCalibration* {
            auto* c = new CameraCalibration();
            c->kind = CALIB_GAIN_OFFSET;
            c->gain = gain;
            c->offset = offset;
            return calib_register(c, ctx);
        },
        (CameraCalibration*)nullptr);
}

CameraCalibration* GainOffsetImageCalib_Create(int width, int height, const float* gain, const float* offset,
                                               Context* ctx) {
    return fq_guarded(
        [&]() -> CameraCalibration* {
            if (width < 1 || height < 1 || !gain || !offset) throw FrameQueueError("GainOffsetImageCalib_Create: bad arguments");
            auto* c = new CameraCalibration();
            c->kind = CALIB_GAIN_OFFSET_IMAGE;
            c->w = width;
            c->h = height;
            c->gainImg.assign(gain, gain + (size_t)width * height);
            c->offsetImg.assign(offset, offset + (size_t)width * height);
            return calib_register(c, ctx);
        },
        (CameraCalibration*)nullptr);
}

CameraCalibration* sCMOS_Calib_Create(int width, int height, const float* offset, const float* gain,
                                      const float* variance, Context* ctx) {
    (void)variance;  // the reference keeps var/gain^2 for the estimators and does not apply it here
    return fq_guarded(
        [&]() -> CameraCalibration* {
            if (width < 1 || height < 1 || !gain || !offset) throw FrameQueueError("sCMOS_Calib_Create: bad arguments");
            auto* c = new CameraCalibration();
            c->kind = CALIB_SCMOS;
            c->w = width;
            c->h = height;
            c->gainImg.assign(gain, gain + (size_t)width * height);
            c->offsetImg.assign(offset, offset + (size_t)width * height);
            return calib_register(c, ctx);
        },
        (CameraCalibration*)nullptr);
}

ROIQueue* RQ_Create(const int* shapeZYX, Context* ctx) {
    return fq_guarded(
        [&]() -> ROIQueue* {
            if (!shapeZYX || shapeZYX[0] < 1 || shapeZYX[1] < 1 || shapeZYX[2] < 1)
                throw FrameQueueError("RQ_Create: bad shape");
            auto* q = new ROIQueue();
            for (int i = 0; i < 3; i++) q->shape[i] = shapeZYX[i];
            q->smp = (size_t)shapeZYX[0] * shapeZYX[1] * shapeZYX[2];
            q->ctx = ctx;
            pb200::context_attach(ctx, q, destroy_roiqueue);
            return q;
        },
        (ROIQueue*)nullptr);
}

void RQ_Pop(ROIQueue* q, int count, ROIInfo* rois, float* data) {
    if (q) q->pop(count, rois, data);
}

int RQ_Length(ROIQueue* q) { return q ? q->len() : 0; }

void RQ_Push(ROIQueue* q, int count, const ROIInfo* info, const float* data) {
    fq_guarded(
        [&]() -> int {
            if (!q || (count > 0 && (!info || !data))) throw FrameQueueError("RQ_Push: bad arguments");
            q->push(count, info, data);
            return 0;
        },
        0);
}

void RQ_SmpShape(ROIQueue* q, int* shapeZYX) {
    if (!q || !shapeZYX) return;
    for (int i = 0; i < 3; i++) shapeZYX[i] = q->shape[i];
}

void RQ_Delete(ROIQueue* q) {
    if (!q) return;
    pb200::context_detach(q->ctx, q);
    delete q;
}

void ImgProc_Flush(ImageProcessor* q) {
    if (q) q->Flush();
}

void ImgProc_AddFrameU16(ImageProcessor* q, const uint16_t* data) {
    fq_guarded(
        [&]() -> int {
            if (!q) throw FrameQueueError("ImgProc_AddFrameU16: null processor");
            q->AddFrameU16(data);
            return 0;
        },
        0);
}

void ImgProc_AddFrameF32(ImageProcessor* q, const float* data) {
    fq_guarded(
        [&]() -> int {
            if (!q) throw FrameQueueError("ImgProc_AddFrameF32: null processor");
            q->AddFrameF32(data);
            return 0;
        },
        0);
}

int ImgProc_GetQueueLength(ImageProcessor* q) { return q ? q->GetQueueLength() : 0; }

int ImgProc_ReadFrame(ImageProcessor* q, float* image, float* processed) {
    return q ? q->ReadFrame(image, processed) : 0;
}

int ImgProc_NumFinishedFrames(ImageProcessor* q) { return q ? q->NumFinishedFrames() : 0; }

bool ImgProc_IsIdle(ImageProcessor* q) { return q ? q->IsIdle() : true; }

void ImgProc_Destroy(ImageProcessor* q) {
    if (!q) return;
    pb200::context_detach(q->ctx, q);
    delete q;
}

ImageProcessor* SpotExtractionQueue_Create(int width, int height, ROIQueue* roilist, SpotDetectorFactory* sdf,
                                           CameraCalibration* calib, int numDetectionThreads, int sumframes,
                                           Context* ctx) {
    (void)numDetectionThreads;
    (void)sumframes;  // the ROI queue's z size sets the group size (ImgFilterQueue.cu:283)
    return fq_guarded(
        [&]() -> ImageProcessor* {
            if (!roilist || !sdf) throw FrameQueueError("SpotExtractionQueue_Create: null ROI queue or detector");
            const SpotDetectorConfig* cfg = pb200::spot_factory_config(sdf);
            auto* q = new SpotExtractionQueue(width, height, roilist, *cfg, calib);
            q->ctx = ctx;
            pb200::context_attach(ctx, q, destroy_imgproc);
            return q;
        },
        (ImageProcessor*)nullptr);
}

ImageProcessor* ROIExtractor_Create(int imgWidth, int imgHeight, const ExtractionROI* rois, int numrois, int roiframes,
                                    int roisize, CameraCalibration* calib, Context* ctx) {
    return fq_guarded(
        [&]() -> ImageProcessor* {
            auto* q = new ROIExtractorQueue(imgWidth, imgHeight, rois, numrois, roiframes, roisize, calib);
            q->ctx = ctx;
            pb200::context_attach(ctx, q, destroy_imgproc);
            return q;
        },
        (ImageProcessor*)nullptr);
}

int ROIExtractor_GetResultCount(ImageProcessor* re) {
    auto* q = dynamic_cast<ROIExtractorQueue*>(re);
    return q ? q->result_count() : 0;
}

int ROIExtractor_GetResults(ImageProcessor* re, int numrois, ExtractionROI* rois, float* framedata) {
    return fq_guarded(
        [&]() -> int {
            auto* q = dynamic_cast<ROIExtractorQueue*>(re);
            if (!q) throw FrameQueueError("ROIExtractor_GetResults: not a ROI extractor");
            return q->results(numrois, rois, framedata);
        },
        0);
}

}  // extern "C"
