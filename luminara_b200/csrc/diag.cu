// diag.cu -- diagnostic microbenchmark (sm_100a): the L1 load throughput that bounds the
// megakernel's node and primitive fetches.
//
// The megakernel's algorithmic bytes (64-byte BVH nodes, 16-48-byte primitive records) are
// served from L1 and L2 -- on the sphere field the scene is a few tens of kilobytes and DRAM
// sees almost none of it -- so the HBM copy rate is not the roof those bytes run against.  This
// kernel measures the roof instead: 128-bit __ldg loads from a 32 KiB table (L1-resident after
// the first touch) by every SM at full occupancy, independent loads only (no dependence chain),
//   pattern 0  coalesced: a warp reads 512 contiguous bytes per load instruction;
//   pattern 1  gather: each lane reads one 64-byte record (four float4) at a hashed index, the
//              access pattern of a BVH node visit.
// No counterpart in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>

#include "../../include/luminara_gpu.h"
#include "scene_access.h"

namespace {

constexpr int kProbeThreads = 256;
constexpr uint32_t kTableVec = 2048;          // 32 KiB of float4

template <int PATTERN>
__global__ void __launch_bounds__(kProbeThreads) k_l1_probe(const float4* __restrict__ tab, uint32_t iters,
                                                            float* __restrict__ out) {
    const uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t h = tid * 0x9E3779B9u + 0x7f4a7c15u;
    float acc = 0.0f;
#pragma unroll 4
    for (uint32_t it = 0; it < iters; ++it) {
        float4 v0, v1, v2, v3;
        if constexpr (PATTERN == 0) {
            const uint32_t base = it * 128u + warp * 512u + lane;
            v0 = __ldg(tab + ((base + 0u) & (kTableVec - 1)));
            v1 = __ldg(tab + ((base + 32u) & (kTableVec - 1)));
            v2 = __ldg(tab + ((base + 64u) & (kTableVec - 1)));
            v3 = __ldg(tab + ((base + 96u) & (kTableVec - 1)));
        } else {
            h = h * 1664525u + 1013904223u;                   // independent of the loaded data
            const uint32_t node = (h >> 9) & (kTableVec / 4 - 1);
            v0 = __ldg(tab + 4 * node + 0);
            v1 = __ldg(tab + 4 * node + 1);
            v2 = __ldg(tab + 4 * node + 2);
            v3 = __ldg(tab + 4 * node + 3);
        }
        acc += (v0.x + v1.y) + (v2.z + v3.w);
    }
    out[tid] = acc;
}

}  // namespace

extern "C" lum_status lum_diag_l1_throughput(int32_t pattern, double* gbs) {
    if (!gbs || pattern < 0 || pattern > 1) return lum::set_error(LUM_ERR_INVALID_ARGUMENT, "bad argument");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = 0;
    auto fn = pattern == 0 ? k_l1_probe<0> : k_l1_probe<1>;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kProbeThreads, 0);
    const int grid = std::max(1, sms) * std::max(1, per_sm);
    float4* tab = nullptr;
    float* out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e;
    char msg[256];
    const uint32_t iters = 8192;
    float best = 1e30f;
    if ((e = cudaMalloc(&tab, kTableVec * sizeof(float4))) != cudaSuccess ||
        (e = cudaMalloc(&out, (size_t)grid * kProbeThreads * sizeof(float))) != cudaSuccess ||
        (e = cudaMemset(tab, 0, kTableVec * sizeof(float4))) != cudaSuccess ||
        (e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess)
        goto done;
    for (int rep = 0; rep < 4; ++rep) {     // the first launch warms the table into L1
        cudaEventRecord(e0, 0);
        fn<<<grid, kProbeThreads>>>(tab, iters, out);
        cudaEventRecord(e1, 0);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess || (e = cudaGetLastError()) != cudaSuccess) goto done;
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best = std::min(best, ms);
    }
    *gbs = (double)grid * kProbeThreads * iters * 64.0 / (best * 1e-3) / 1e9;
done:
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (tab) cudaFree(tab);
    if (out) cudaFree(out);
    if (e != cudaSuccess) {
        snprintf(msg, sizeof msg, "lum_diag_l1_throughput: %s", cudaGetErrorString(e));
        return lum::set_error(LUM_ERR_CUDA, msg);
    }
    return LUM_OK;
}
