// Precision form of the patch transform: the 2D DCT of 8x8 patches as a tcgen05
// TF32 contraction with FP32 accumulation in tensor memory, with the accuracy won
// back by splitting both operands into a TF32 high part and an FP32 remainder.
//
// The 2D transform of a patch is one 64x64 matrix: vec(Y) = (T (x) T) vec(X), T the
// unnormalised DCT-II that every transform here and in the reference uses (orthonormal
// DCT-II scaled by 4 per axis, vszipcu src/bm3d.cu:32-110).  A tile of 128 patches is
// the M = 128 side of the MMA, the 64 output coefficients the N = 64 side, the 64
// pixels the K side (8 MMAs of K = 8).  With X = Xh + Xl and K = Kh + Kl (h = TF32
// truncation, l = the exact FP32 remainder, itself read as TF32), the product is
// Xl.Kh + Xh.Kl + Xh.Kh, small terms first; only Xl.Kl (about 2^-22 relative) is
// dropped.  The plain form keeps the FP32 SIMT transforms, which are bitwise equal
// to the reference's; this form is a measured alternative, not on the plain path.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "zb3d_tcgen05.cuh"

namespace zb {
namespace {
using namespace tc05;

constexpr int TILE = 128;                        // patches per tile (M)
constexpr int A_BYTES = TILE * 64 * 4;           // one A operand copy: 32 KB
constexpr int B_BYTES = 64 * 64 * 4;             // one B operand copy: 16 KB
constexpr int SMEM = 2 * A_BYTES + 2 * B_BYTES + 64;
constexpr unsigned WAIT_LIMIT = 1u << 22;
constexpr int THREADS = 256;                     // 8 warps: all stage, two per tensor-memory lane quarter drain
// kind::tf32: FP32 accumulator (bit 4), TF32 A (bits 7-9 = 2) and B (bits 10-12 = 2),
// both K-major, N = 64 (bits 17-22 = N >> 3), M = 128 (bits 24-28 = M >> 4)
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);

// (T (x) T) as [output coefficient r * 8 + c][input pixel i * 8 + j]: TF32 high parts, remainders
__device__ float g_kron[2][64 * 64];

// Byte offset of element (row, k) in a K-major operand without swizzle: core matrices
// of 8 rows x 16 bytes (4 elements), 8-row groups 128 bytes apart, 4-element K chunks
// rows * 16 bytes apart.
__host__ __device__ constexpr uint32_t kmaj(int row, int k, int rows) {
    return (uint32_t)((k >> 2) * rows * 16 + (row >> 3) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

__host__ __device__ inline float tf32_high(float x) {
#ifdef __CUDA_ARCH__
    return __uint_as_float(__float_as_uint(x) & 0xffffe000u);
#else
    uint32_t u;
    std::memcpy(&u, &x, 4);
    u &= 0xffffe000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
#endif
}

// shared-memory matrix descriptor, K-major without swizzle: start, LBO (K chunks), SBO (8-row groups)
__device__ __forceinline__ uint64_t desc_k(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
        : "memory");
}

// each CTA stages the matrix once and walks tiles of 128 patches
__global__ void __launch_bounds__(THREADS) dct2d_tf32(const float *__restrict__ x, float *__restrict__ y, long long n,
                                                  int split, int *status) {
    extern __shared__ __align__(1024) uint8_t sm[];
    uint8_t *a_hi = sm, *a_lo = sm + A_BYTES, *b_hi = sm + 2 * A_BYTES, *b_lo = b_hi + B_BYTES;
    uint64_t *bar = reinterpret_cast<uint64_t *>(b_lo + B_BYTES);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int i = tid; i < 64 * 64; i += THREADS) {
        const int row = i >> 6, k = i & 63;
        *reinterpret_cast<float *>(b_hi + kmaj(row, k, 64)) = g_kron[0][i];
        *reinterpret_cast<float *>(b_lo + kmaj(row, k, 64)) = g_kron[1][i];
    }
    if (tid == 0) {
        mbar_init(smem_u32(bar), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) tmem_alloc(smem_u32(tslot), 64);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo), bh = smem_u32(b_hi), bl = smem_u32(b_lo);

    const long long ntiles = (n + TILE - 1) / TILE;
    uint32_t phase = 0;
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const long long p0 = t * TILE;
        // the tile's patches, split into TF32 high parts and FP32 remainders, written in
        // shared-memory order: a warp fills 128 contiguous bytes (8 patches x one 4-pixel
        // chunk) per store, conflict-free, and reads 8 runs of 16 bytes from global memory
        for (int s = tid; s < TILE * 64; s += THREADS) {
            const int kk = s & 3, row = (s >> 2) & (TILE - 1), kc = s >> 9;  // s = kmaj(row, 4 kc + kk) / 4
            const long long p = p0 + row;
            const float v = p < n ? __ldg(x + p * 64 + kc * 4 + kk) : 0.0f;
            const float hi = tf32_high(v);
            reinterpret_cast<float *>(a_hi)[s] = hi;
            reinterpret_cast<float *>(a_lo)[s] = v - hi;
        }
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        fence_after_sync();
        if (tid == 0) {
            uint32_t acc = 0;
            for (int part = split ? 0 : 2; part < 3; ++part) {  // Xl.Kh, Xh.Kl, then Xh.Kh
                const uint32_t a = part == 0 ? al : ah, b = part == 1 ? bl : bh;
                for (int ks = 0; ks < 8; ++ks) {
                    mma_tf32(tmem, desc_k(a + ks * 2 * TILE * 16, TILE * 16, 128),
                             desc_k(b + ks * 2 * 64 * 16, 64 * 16, 128), acc);
                    acc = 1;
                }
            }
            mma_commit(smem_u32(bar));
        }
        bool done = false;
        for (unsigned i = 0; i < WAIT_LIMIT && !done; ++i) done = mbar_try(smem_u32(bar), phase);
        phase ^= 1u;
        if (!__syncthreads_and(done)) {
            // the products did not complete in time: record it (1), let them land, stop.  If
            // they still have not landed, the status is 2: tensor memory is freed while an MMA
            // may still write it, so the caller must treat the device as unhealthy and not retry.
            if (tid == 0) {
                atomicExch(status, 1);
                bool landed = false;
                for (unsigned i = 0; i < WAIT_LIMIT && !landed; ++i) landed = mbar_try(smem_u32(bar), phase ^ 1u);
                if (!landed) atomicExch(status, 2);
            }
            __syncthreads();
            break;
        }
        fence_after_sync();
        // warp w reads tensor-memory lanes 32 (w % 4) .. + 31 (one patch per thread), columns
        // 32 (w / 4) .. + 31 (half of its coefficients)
        {
            const int quarter = warp & 3, half = warp >> 2;
            const long long p = p0 + quarter * 32 + lane;
            float v[32];
            tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(half * 32), v);
            if (p < n) {
                float4 *dst = reinterpret_cast<float4 *>(y + p * 64 + half * 32);
#pragma unroll
                for (int q = 0; q < 8; ++q) dst[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        }
        fence_before_sync();
        __syncthreads();  // A staging and the accumulator are reused by the next tile
        fence_after_sync();
    }
    __syncthreads();
    if (warp == 0) {
        __syncwarp();  // lane 0 issued the MMAs alone; tcgen05.dealloc is .sync.aligned
        tmem_dealloc(tmem, 64);
    }
}

std::once_flag g_host_once;
float g_host_kron[2][64 * 64];
std::once_flag g_dev_once[64];
cudaError_t g_dev_err[64];

// (T (x) T) from the closed form of T in double on the host, split into float parts:
// built once per process, then copied once per device
cudaError_t init_matrix(int dev) {
    std::call_once(g_host_once, [] {
        const double pi = 3.14159265358979323846264338327950288;
        double T[8][8];
        for (int k = 0; k < 8; ++k)
            for (int m = 0; m < 8; ++m)
                T[k][m] = 4.0 * (k == 0 ? std::sqrt(1.0 / 8.0) : std::sqrt(2.0 / 8.0)) *
                          std::cos(pi * (2 * m + 1) * k / 16.0);
        for (int r = 0; r < 8; ++r)
            for (int c = 0; c < 8; ++c)
                for (int i = 0; i < 8; ++i)
                    for (int j = 0; j < 8; ++j) {
                        const float v = (float)(T[r][i] * T[c][j]);
                        const float hi = tf32_high(v);
                        g_host_kron[0][(r * 8 + c) * 64 + i * 8 + j] = hi;
                        g_host_kron[1][(r * 8 + c) * 64 + i * 8 + j] = v - hi;
                    }
    });
    std::call_once(g_dev_once[dev], [dev] {
        g_dev_err[dev] = cudaMemcpyToSymbol(g_kron, g_host_kron, sizeof(g_host_kron));
        if (g_dev_err[dev] == cudaSuccess) g_dev_err[dev] = cudaFuncSetAttribute(dct2d_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    });
    return g_dev_err[dev];
}

}  // namespace
}  // namespace zb

extern "C" int zb3d_dct2d_tf32(const float *d_x, float *d_y, long long npatches, int split, int *d_status,
                               void *stream) {
    using namespace zb;
    if (npatches < 0 || (npatches > 0 && (!d_x || !d_y || !d_status))) return 1;
    if (((uintptr_t)d_y & 15) != 0) return 1;
    if (npatches == 0) return 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 2;
    if (init_matrix(dev) != cudaSuccess) return 2;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long ntiles = (npatches + TILE - 1) / TILE;
    const int grid = (int)(ntiles < 2LL * sms ? ntiles : 2LL * sms);
    dct2d_tf32<<<grid, THREADS, SMEM, (cudaStream_t)stream>>>(d_x, d_y, npatches, split, d_status);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}
