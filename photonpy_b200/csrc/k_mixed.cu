// Instantiation and launcher of the mixed-model persistent fit kernel.
#include "launch.cuh"
#include "mixed.cuh"

namespace pb200 {

// Lanes per ROI of the mixed kernel: 4 (ROI sizes up to 16 pixels).
constexpr int kMixedLanes = 4;

int mixed_lanes() { return kMixedLanes; }

void launch_mixed(const MixedTask* d_tasks, int ntasks, int totalTiles, int tileRois, int* d_counter,
                  int strideFloats, int variant, cudaStream_t s) {
    auto kern = mixed_fit_kernel<kMixedLanes, 128, 3, false>;
    int threads = 128;
    if (variant == 1) {
        kern = mixed_fit_kernel<kMixedLanes, 256, 2, true>;
        threads = 256;
    } else if (variant == 2) {
        kern = mixed_fit_kernel<kMixedLanes, 128, 4, true>;
    }
    const int gpb = threads / kMixedLanes;
    const size_t smem = (size_t)gpb * strideFloats * sizeof(float);
    if (smem > (size_t)kMaxSmemPerBlock) throw std::runtime_error("mixed kernel: shared memory per block too large");
    set_smem_attr(kern, smem);
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, threads, smem) != cudaSuccess || perSM < 1)
        throw std::runtime_error("mixed kernel: occupancy query failed");
    const int warpsPerBlock = threads / 32;
    const long long needBlocks = ((long long)totalTiles + warpsPerBlock - 1) / warpsPerBlock;
    const long long cap = (long long)num_sms() * perSM;
    const int grid = (int)(needBlocks < cap ? needBlocks : cap);
    if (grid <= 0) return;
    kern<<<grid, threads, smem, s>>>(d_tasks, ntasks, totalTiles, tileRois, d_counter, strideFloats);
    check_launch("mixed kernel launch");
    count_launch();
}

}  // namespace pb200
