// aov.cu -- the AOV passes (render.rs:3508-3568): depth, normal and albedo of the closest hit
// of one ray per pixel through the pixel centre.
//
// One thread per pixel (grid-stride).  The ray is the time limit's centre sample
// (start_path_centre: stratum 0's lens and time draws); albedo is the hit material's scatter
// attenuation with that pixel's bounce-0 scatter draws (Blends resolved as in the
// integrator), or, for a surface that does not scatter, its emission scaled by
// 1 / max(max component, 1).  Bytes follow Rust's `as u8` (saturating, NaN -> 0).
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "tracer.cuh"

namespace lum {
namespace {

constexpr int kAovThreads = 128;

__device__ __forceinline__ uint8_t as_u8(float x) {
    if (!(x > 0.0f)) return 0;
    if (x >= 255.0f) return 255;
    return (uint8_t)x;
}

__device__ __forceinline__ uint8_t unit_byte(float x) { return as_u8(fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f); }
__device__ __forceinline__ uint8_t clamp_byte(float x) { return as_u8(fminf(fmaxf(x, 0.0f), 255.0f)); }

__global__ void __launch_bounds__(kAovThreads) k_aov(SceneDev S, RenderDev R, float* __restrict__ depth,
                                                     uint8_t* __restrict__ normals, uint8_t* __restrict__ albedo,
                                                     WorkCounters* wc) {
    extern __shared__ int s_stack[];
    int* stack = s_stack + threadIdx.x;
    uint32_t err = 0;
    const size_t n = (size_t)R.w * R.h;
    for (size_t o = (size_t)blockIdx.x * blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(o % R.w), j = (uint32_t)(o / R.w);
        const uint32_t gi = i + R.crop_x, gj = j + R.crop_y;
        const uint32_t pixel = gj * R.full_w + gi;
        Path P;
        start_path_centre(S, R, gi, gj, pixel, P);
        Hit h;
        h.t = CUDART_INF_F;
        h.prim = -1;
        h.b1 = h.b2 = 0.0f;
        float dv = 0.0f;
        uint8_t nb[3] = {0, 0, 0}, ab[3] = {0, 0, 0};
        if (trace<false>(S, P.ray, 0.001f, false, h, stack, err)) {
            dv = h.t;
            const Surface sf = surface_of(S, P.ray, h);
            nb[0] = clamp_byte((sf.n.x * 0.5f + 0.5f) * 255.0f);
            nb[1] = clamp_byte((sf.n.y * 0.5f + 0.5f) * 255.0f);
            nb[2] = clamp_byte((sf.n.z * 0.5f + 0.5f) * 255.0f);
            if (albedo) {
                const MatDev& m = S.mats[sf.mat];
                const float4 su = draw4(R.key0, R.key1, pixel, 0, 0, CALL_SCATTER);
                const MatDev& ms = blend_leaf(S, m, R, pixel, 0, 0);
                Scatter sc;
                sc.org = sf.p;
                if (scatter<-1>(ms, P.ray, sf, h.t, su, R, pixel, 0, 0, sc)) {
                    ab[0] = unit_byte(sc.att.x);
                    ab[1] = unit_byte(sc.att.y);
                    ab[2] = unit_byte(sc.att.z);
                } else {
                    const V e = emitted_at(S, sf.mat, m, sf.p);
                    const float me = fmaxf(fmaxf(e.x, fmaxf(e.y, e.z)), 1.0f);
                    ab[0] = clamp_byte(e.x / me * 255.0f);
                    ab[1] = clamp_byte(e.y / me * 255.0f);
                    ab[2] = clamp_byte(e.z / me * 255.0f);
                }
            }
        }
        if (depth) depth[o] = dv;
        for (int c = 0; c < 3; ++c) {
            if (normals) normals[3 * o + c] = nb[c];
            if (albedo) albedo[3 * o + c] = ab[c];
        }
    }
    if (err) atomicOr(&wc->error_flags, err);
}

}  // namespace

cudaError_t launch_aov(const SceneDev& S, const RenderDev& R, float* depth, uint8_t* normals, uint8_t* albedo,
                       WorkCounters* wc, cudaStream_t stream) {
    const size_t stack = (size_t)kStackDepth * kAovThreads * sizeof(int);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_aov, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)stack);
        attr = true;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const size_t n = (size_t)R.w * R.h;
    const int grid = (int)std::max<size_t>(1, std::min<size_t>((n + kAovThreads - 1) / kAovThreads, (size_t)sms * 8));
    k_aov<<<grid, kAovThreads, stack, stream>>>(S, R, depth, normals, albedo, wc);
    return cudaGetLastError();
}

}  // namespace lum
