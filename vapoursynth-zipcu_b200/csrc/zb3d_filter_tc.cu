// Precision form of the collaborative filter (zb3d_args.filter_form = 1): the same
// algorithm as the plain 16-lane filter (vszipcu src/bm3d.cu:457-546), with the 2D
// transforms of the group's patches on the tensor cores (zb3d_dct_tc.cu: TF32 with the
// hi/lo split, FP32 accumulation) instead of the FP32 SIMT codelets.  The result agrees
// with the plain form and the FP64 oracle to FP32 rounding, but not bit for bit: the
// contraction sums in another order, so a coefficient that sits within rounding of the
// hard threshold can be kept by one form and dropped by the other.
//
// Per plane of an entry, over a stack S[group][patch][64] in global memory:
//   1. gather:     S = the 8 matched 8x8 patches of every group (noisy; with Wiener also
//                  the basic estimate's patches into a second stack B)
//   2. forward 2D: S = (T (x) T) S per patch on tcgen05 (and B)
//   3. shrink:     per group and 2D coefficient, the 1D transform T along the 8 patches,
//                  hard threshold at sigma (the 3D DC kept) or the Wiener gain from B,
//                  the 1/4096 of the unnormalised 3D pair, the inverse 1D transform T^T;
//                  the group's weight 1 / (kept count) or 1 / (sum of squared gains)
//   4. inverse 2D: S = (T^T (x) T^T) S per patch on tcgen05
//   5. aggregate:  the weighted patches into the fixed-point accumulators of the plain
//                  form (same extractor rounding), weights at the patch origins
// so finish, the stacked output and the temporal aggregation read the same accumulators.
// T is the unnormalised DCT-II of the plain form (the orthonormal one scaled by 4).
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "zb3d_args.h"

namespace zb {

int dct2d_tf32_run(const float *d_x, float *d_y, long long npatches, int split, int inverse, int *d_status,
                   cudaStream_t stream);
cudaError_t dct_tc_init(int dev);

namespace {

__constant__ float c_t8[8][8];  // T[k][m]: coefficient k of sample m

__device__ __forceinline__ unsigned long long pf_to_fix(float v) {
    return (unsigned long long)__float2ll_rn(v * kFixScale);
}

// S[g][p][row * 8 + j] = plane[z][y + row][x + j] of patch p of group g: one thread per
// patch column j, so that consecutive lanes read and write consecutive pixels
__global__ void pf_gather(const float *__restrict__ plane, long long frame_stride, int pitch,
                          const int2 *__restrict__ list, long long nblocks, float *__restrict__ stack) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nblocks * 64) return;
    const long long gp = i >> 3;  // group * 8 + patch
    const int j = (int)(i & 7);
    const int2 v = list[gp];
    const float *s = plane + ((unsigned)v.y >> 24) * frame_stride + (long long)(v.y & 0xffffff) * pitch + v.x + j;
    float *d = stack + gp * 64 + j;
#pragma unroll
    for (int row = 0; row < 8; ++row) d[row * 8] = __ldg(s + (long long)row * pitch);
}

// One warp per group; lane handles 2D coefficients lane and lane + 32 across the 8 patches.
template <bool FINAL>
__global__ void pf_shrink(float *__restrict__ stack, const float *__restrict__ basic, long long nblocks, float sigma,
                          float *__restrict__ weight) {
    const long long g = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (g >= nblocks) return;
    float acc = 0.0f;  // kept coefficients, or the sum of squared Wiener gains
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        const int c = lane + 32 * half;
        float v[8], s[8];
#pragma unroll
        for (int p = 0; p < 8; ++p) v[p] = stack[(g * 8 + p) * 64 + c];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float t = 0.0f;
#pragma unroll
            for (int p = 0; p < 8; ++p) t = __fmaf_rn(c_t8[k][p], v[p], t);
            s[k] = t;
        }
        if constexpr (FINAL) {
            float b[8];
#pragma unroll
            for (int p = 0; p < 8; ++p) b[p] = basic[(g * 8 + p) * 64 + c];
            const float s2 = sigma * sigma;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                float r = 0.0f;
#pragma unroll
                for (int p = 0; p < 8; ++p) r = __fmaf_rn(c_t8[k][p], b[p], r);
                const float r2 = r * r;
                const float gain = (c == 0 && k == 0) ? 1.0f : r2 / (r2 + s2);
                acc = __fmaf_rn(gain, gain, acc);
                s[k] = s[k] * gain * (1.0f / 4096.0f);
            }
        } else {
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const bool keep = (c == 0 && k == 0) || fabsf(s[k]) >= sigma;
                acc += keep ? 1.0f : 0.0f;
                s[k] = keep ? s[k] * (1.0f / 4096.0f) : 0.0f;
            }
        }
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            float t = 0.0f;
#pragma unroll
            for (int k = 0; k < 8; ++k) t = __fmaf_rn(c_t8[k][p], s[k], t);
            stack[(g * 8 + p) * 64 + c] = t;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) weight[g] = 1.0f / acc;
}

// num[z][y + row][x + j] += w * S[g][p][row * 8 + j] (extractor rounding of the plain form);
// den at the patch origin += w.  One thread per patch column j: a warp's atomics fall on
// 4 patch rows of 8 consecutive pixels each.
__global__ void pf_aggregate(const float *__restrict__ stack, const float *__restrict__ weight,
                             const int2 *__restrict__ list, long long nblocks, unsigned long long *num,
                             unsigned long long *den, long long frame_stride, int pitch, float E) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nblocks * 64) return;
    const long long gp = i >> 3;
    const int j = (int)(i & 7);
    const float w = weight[gp >> 3];
    const int2 v = list[gp];
    const long long o = ((unsigned)v.y >> 24) * frame_stride + (long long)(v.y & 0xffffff) * pitch + v.x;
    const float *d = stack + gp * 64 + j;
    unsigned long long *q = num + o + j;
#pragma unroll
    for (int row = 0; row < 8; ++row)
        atomicAdd(q + (long long)row * pitch, pf_to_fix(__fmaf_rn(w, d[row * 8], E) - E));
    if (j == 0) atomicAdd(den + o, pf_to_fix((w + E) - E));
}

std::once_flag g_t8_host;
float g_t8[8][8];
std::once_flag g_t8_dev[64];
cudaError_t g_t8_err[64];

}  // namespace

// The constants of the precision filter on device `dev` (the 1D matrix and the 2D
// transform's matrices); synchronous, so call it before any stream capture.
cudaError_t filter_precision_init(int dev) {
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    std::call_once(g_t8_host, [] {
        const double pi = 3.14159265358979323846264338327950288;
        for (int k = 0; k < 8; ++k)
            for (int m = 0; m < 8; ++m)
                g_t8[k][m] = (float)(4.0 * (k == 0 ? std::sqrt(1.0 / 8.0) : std::sqrt(2.0 / 8.0)) *
                                     std::cos(pi * (2 * m + 1) * k / 16.0));
    });
    std::call_once(g_t8_dev[dev], [dev] {
        g_t8_err[dev] = cudaMemcpyToSymbol(c_t8, g_t8, sizeof(g_t8));
        if (g_t8_err[dev] == cudaSuccess) g_t8_err[dev] = dct_tc_init(dev);
    });
    return g_t8_err[dev];
}

// Stack floats the precision filter needs per group and stack.
size_t filter_precision_stack_floats(long long nblocks) { return (size_t)nblocks * 8 * 64; }

// The precision filter of one entry: every plane of `a` into its accumulators.  stack /
// basic: filter_precision_stack_floats(a.nblocks) floats each (basic only for final_),
// 16-byte aligned; weight: a.nblocks floats; status: the transform's wait status.
cudaError_t launch_filter_precision(const FilterArgs &a, bool final_, float *stack, float *basic, float *weight,
                                    int *status, cudaStream_t st) {
    const long long nb = a.nblocks;
    if (nb <= 0) return cudaSuccess;
    const unsigned grid_rows = (unsigned)((nb * 64 + 255) / 256);
    const unsigned grid_groups = (unsigned)((nb * 32 + 255) / 256);
    for (int pl = 0; pl < a.nplanes; ++pl) {
        const float sigma = a.sigma[pl];
        if (a.chroma && sigma < 1.19209290e-7f) continue;
        const float *noisy = a.src + (final_ ? a.clip_stride : 0) + pl * a.plane_stride;
        pf_gather<<<grid_rows, 256, 0, st>>>(noisy, a.frame_stride, a.pitch, a.list, nb, stack);
        if (final_) pf_gather<<<grid_rows, 256, 0, st>>>(a.src + pl * a.plane_stride, a.frame_stride, a.pitch, a.list,
                                                         nb, basic);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (dct2d_tf32_run(stack, stack, nb * 8, 1, 0, status, st) != 0) return cudaErrorLaunchFailure;
        if (final_ && dct2d_tf32_run(basic, basic, nb * 8, 1, 0, status, st) != 0) return cudaErrorLaunchFailure;
        if (final_)
            pf_shrink<true><<<grid_groups, 256, 0, st>>>(stack, basic, nb, sigma, weight);
        else
            pf_shrink<false><<<grid_groups, 256, 0, st>>>(stack, nullptr, nb, sigma, weight);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        if (dct2d_tf32_run(stack, stack, nb * 8, 1, 1, status, st) != 0) return cudaErrorLaunchFailure;
        pf_aggregate<<<grid_rows, 256, 0, st>>>(stack, weight, a.list, nb, a.num + pl * a.acc_plane_stride,
                                                a.den + pl * a.acc_plane_stride, a.acc_frame_stride, a.pitch,
                                                a.extractor);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace zb
