// Instantiation and launcher of the mixed-model persistent fit kernel.
#include "launch.cuh"
#include "mixed.cuh"

namespace pb200 {

// Lanes per ROI of the mixed kernel: 4 (ROI sizes up to 16 pixels).
constexpr int kMixedLanes = 4;

int mixed_lanes() { return kMixedLanes; }

template <int PASS>
const void* mixed_kernel_for(int variant, int* threads) {
    *threads = variant == 1 ? 256 : 128;
    if (variant == 1) return (const void*)mixed_fit_kernel<kMixedLanes, 256, 2, true, PASS>;
    if (variant == 2) return (const void*)mixed_fit_kernel<kMixedLanes, 128, 4, true, PASS>;
    return (const void*)mixed_fit_kernel<kMixedLanes, 128, 3, false, PASS>;
}

// Persistent launch: at most one block per resident slot, fewer when the batch has fewer claims
// (totalClaims = sum over buckets of ceil(n / chunk)) than groups.
void launch_mixed(const MixedTask* d_tasks, int ntasks, int totalClaims, int chunk, int* d_counters,
                  int strideFloats, int variant, bool fisherPass, cudaStream_t s) {
    int threads = 128;
    const void* kern = fisherPass ? mixed_kernel_for<PASS_FISHER>(variant, &threads)
                                  : mixed_kernel_for<PASS_LM>(variant, &threads);
    const int gpb = threads / kMixedLanes;
    const size_t smem = (size_t)gpb * strideFloats * sizeof(float);
    if (smem > (size_t)kMaxSmemPerBlock) throw std::runtime_error("mixed kernel: shared memory per block too large");
    set_smem_attr(kern, smem);
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kern, threads, smem) != cudaSuccess || perSM < 1)
        throw std::runtime_error("mixed kernel: occupancy query failed");
    const long long needBlocks = ((long long)totalClaims + gpb - 1) / gpb;
    const long long cap = (long long)num_sms() * perSM;
    const int grid = (int)(needBlocks < cap ? needBlocks : cap);
    if (grid <= 0) return;
    void* args[] = {(void*)&d_tasks, (void*)&ntasks, (void*)&d_counters, (void*)&chunk, (void*)&strideFloats};
    if (cudaLaunchKernel(kern, dim3(grid), dim3(threads), args, smem, s) != cudaSuccess)
        throw std::runtime_error("mixed kernel launch failed");
    check_launch("mixed kernel launch");
    count_launch();
}

}  // namespace pb200
