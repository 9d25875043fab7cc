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
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "zb3d_tcgen05.cuh"

namespace zb {
namespace {
using namespace tc05;

// Pipeline (one CTA per SM, persistent over tiles of 128 patches, STAGES stages):
//   warp 8 (lane 0)  TMA: the tile's [128][64] FP32 patches as two 128-byte-swizzled boxes
//                    of 32 columns (the canonical K-major SW128 operand layout)
//   warps 4-7        split each element in place into its TF32 high part (kept in the
//                    stage) and the FP32 remainder (written beside it, same layout)
//   warp 9 (lane 0)  24 tcgen05.mma kind::tf32 (3 products x 8 K-steps) into the stage's
//                    64-column accumulator in tensor memory, committed to an mbarrier
//   warps 0-3        drain: tcgen05.ld of lane quarter `warp`, rows written back into the
//                    stage's remainder area (SW128 layout, conflict-free), TMA store
// so the loads of later tiles, the products of one and the stores of earlier ones overlap.
constexpr int TILE = 128;                        // patches per tile (M)
constexpr int HALF_BYTES = TILE * 32 * 4;        // one SW128 box: 128 rows x 128 bytes
constexpr int STAGE_BYTES = 4 * HALF_BYTES;      // high parts (2 boxes) + remainders (2 boxes)
constexpr int B_BYTES = 64 * 64 * 4;             // one B operand copy: 16 KB
constexpr int STAGES = 3;
constexpr int OFF_B = STAGES * STAGE_BYTES;
constexpr int OFF_BAR = OFF_B + 2 * B_BYTES;
constexpr int NBAR = 6 * STAGES;                 // full, split, acc_full, acc_empty, rows_written, stage_free
constexpr int SMEM = OFF_BAR + NBAR * 8 + 16 + 1024;  // + tensor-memory slot, abort flag; + alignment slack
constexpr uint32_t TMEM_COLS = STAGES <= 2 ? 128 : 256;  // a 64-column accumulator per stage, power of two
constexpr unsigned WAIT_LIMIT = 1u << 22;
constexpr int THREADS = 320;                     // 10 warps
static_assert(SMEM <= 227 * 1024, "DCT pipeline exceeds shared memory");
static_assert(STAGES * 64 <= (int)TMEM_COLS, "accumulators exceed the tensor-memory allocation");
// kind::tf32: FP32 accumulator (bit 4), TF32 A (bits 7-9 = 2) and B (bits 10-12 = 2),
// both K-major, N = 64 (bits 17-22 = N >> 3), M = 128 (bits 24-28 = M >> 4)
constexpr uint32_t IDESC = (1u << 4) | (2u << 7) | (2u << 10) | ((64u >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);

// [direction][hi, lo][output index][input index]: direction 0 is (T (x) T) as [coefficient
// r * 8 + c][pixel i * 8 + j], direction 1 its transpose (the inverse transform, up to the
// factor 256 of the unnormalised pair); TF32 high parts and remainders
__device__ float g_kron[2][2][64 * 64];

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

// K-major, 128-byte swizzle (layout type 2 at bits 61-63): rows of 128 bytes, 8-row groups
// 1024 bytes apart (SBO), LBO 16 bytes (unused within one swizzle row); the atom is
// 1024-byte aligned and a K-step inside it only moves the start address
__device__ __forceinline__ uint64_t desc_sw128(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3fff) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
        : "memory");
}

// one [128 rows][32 columns] box of the [n][64] patch matrix: load (zero fill past n) / store (clipped)
__device__ __forceinline__ void tma_load_box(uint32_t dst, const CUtensorMap *map, int col, int row, uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
        "[%4];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(col), "r"(row), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ void tma_store_box(const CUtensorMap *map, int col, int row, uint32_t src) {
    asm volatile("cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];\n" ::"l"(
                     reinterpret_cast<uint64_t>(map)),
                 "r"(col), "r"(row), "r"(src)
                 : "memory");
}

// Bounded wait on an mbarrier phase; gives up at once when another role has aborted.  On
// timeout it sets the abort flag and status 1.
__device__ __forceinline__ bool wait_phase(uint32_t mbar, uint32_t parity, volatile int *abort_flag, int *status) {
    for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try(mbar, parity)) return true;
        if (*abort_flag) return false;
    }
    *abort_flag = 1;
    atomicCAS(status, 0, 1);
    return false;
}

__global__ void __launch_bounds__(THREADS, 1) dct2d_tf32(const __grid_constant__ CUtensorMap map_x,
                                                       const __grid_constant__ CUtensorMap map_y, long long n,
                                                       int split, int inverse, int *status) {
    extern __shared__ uint8_t sm_raw[];
    // 1024-byte aligned base: the SW128 boxes and the swizzle phase of the MMA operands need it
    const uint32_t raw_u32 = smem_u32(sm_raw);
    uint8_t *sm = sm_raw + (((raw_u32 + 1023u) & ~1023u) - raw_u32);
    const uint32_t base = smem_u32(sm);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t bar0 = base + OFF_BAR;
    auto full = [&](int s) { return bar0 + 8u * s; };
    auto splitb = [&](int s) { return bar0 + 8u * (STAGES + s); };
    auto accf = [&](int s) { return bar0 + 8u * (2 * STAGES + s); };
    auto acce = [&](int s) { return bar0 + 8u * (3 * STAGES + s); };
    auto rows = [&](int s) { return bar0 + 8u * (4 * STAGES + s); };
    auto sfree = [&](int s) { return bar0 + 8u * (5 * STAGES + s); };
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + OFF_BAR + NBAR * 8);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(sm + OFF_BAR + NBAR * 8 + 4);
    uint8_t *b_hi = sm + OFF_B, *b_lo = sm + OFF_B + B_BYTES;

    for (int i = tid; i < 64 * 64; i += THREADS) {
        const int row = i >> 6, k = i & 63;
        *reinterpret_cast<float *>(b_hi + kmaj(row, k, 64)) = g_kron[inverse][0][i];
        *reinterpret_cast<float *>(b_lo + kmaj(row, k, 64)) = g_kron[inverse][1][i];
    }
    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            mbar_init(full(s), 1);
            mbar_init(splitb(s), 4);
            mbar_init(accf(s), 1);
            mbar_init(acce(s), 4);
            mbar_init(rows(s), 4);
            mbar_init(sfree(s), 1);
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    fence_async_smem();  // the B operands, written by threads, are read by the tensor cores
    if (warp == 9) tmem_alloc(smem_u32(tslot), TMEM_COLS);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;
    const long long ntiles = (n + TILE - 1) / TILE;
    auto stage_hi = [&](int s) { return base + (uint32_t)(s * STAGE_BYTES); };
    auto stage_lo = [&](int s) { return base + (uint32_t)(s * STAGE_BYTES + 2 * HALF_BYTES); };

    if (warp == 8) {
        // ---- TMA producer ----
        if (lane == 0) {
            long long li = 0, last_use[STAGES];
            for (int s = 0; s < STAGES; ++s) last_use[s] = -1;
            for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++li) {
                const int s = (int)(li % STAGES);
                const uint32_t u = (uint32_t)(li / STAGES);
                if (!wait_phase(sfree(s), (u & 1u) ^ 1u, abort_flag, status)) break;
                mbar_arrive_tx(full(s), 2 * HALF_BYTES);
                tma_load_box(stage_hi(s), &map_x, 0, (int)(t * TILE), full(s));
                tma_load_box(stage_hi(s) + HALF_BYTES, &map_x, 32, (int)(t * TILE), full(s));
                last_use[s] = u;
            }
            if (*abort_flag) {
                // the last load issued into each stage must land before the CTA's shared
                // memory goes away (its phase stays complete once it has completed)
                for (int s = 0; s < STAGES; ++s) {
                    if (last_use[s] < 0) continue;
                    bool landed = false;
                    for (unsigned i = 0; i < WAIT_LIMIT && !landed; ++i)
                        landed = mbar_test(full(s), (uint32_t)(last_use[s] & 1));
                    if (!landed) atomicExch(status, 2);
                }
            }
        }
    } else if (warp >= 4 && warp < 8) {
        // ---- split: X = Xh + Xl in place ----
        const int j = tid - 128;
        long long li = 0;
        for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++li) {
            const int s = (int)(li % STAGES);
            const uint32_t u = (uint32_t)(li / STAGES);
            if (!wait_phase(full(s), u & 1u, abort_flag, status)) break;
            float4 *hi = reinterpret_cast<float4 *>(sm + s * STAGE_BYTES);
            float4 *lo = reinterpret_cast<float4 *>(sm + s * STAGE_BYTES + 2 * HALF_BYTES);
#pragma unroll 4
            for (int v = 0; v < 2 * HALF_BYTES / 16; v += 128) {
                const float4 x = hi[v + j];
                const float4 h = make_float4(tf32_high(x.x), tf32_high(x.y), tf32_high(x.z), tf32_high(x.w));
                hi[v + j] = h;
                lo[v + j] = make_float4(x.x - h.x, x.y - h.y, x.z - h.z, x.w - h.w);
            }
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(splitb(s));
        }
    } else if (warp == 9) {
        // ---- MMA issuer ----
        if (lane == 0) {
            long long issued = 0;
            const uint32_t bh = base + OFF_B, bl = base + OFF_B + B_BYTES;
            long long li = 0;
            for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++li) {
                const int s = (int)(li % STAGES);
                const uint32_t u = (uint32_t)(li / STAGES);
                if (!wait_phase(splitb(s), u & 1u, abort_flag, status)) break;
                if (!wait_phase(acce(s), (u & 1u) ^ 1u, abort_flag, status)) break;
                fence_after_sync();
                const uint32_t d = tmem + (uint32_t)(s * 64);
                uint32_t acc = 0;
                for (int part = split ? 0 : 2; part < 3; ++part) {  // Xl.Kh, Xh.Kl, then Xh.Kh
                    const uint32_t a = part == 0 ? stage_lo(s) : stage_hi(s), b = part == 1 ? bl : bh;
                    for (int ks = 0; ks < 8; ++ks) {
                        mma_tf32(d, desc_sw128(a + (uint32_t)((ks >> 2) * HALF_BYTES + (ks & 3) * 32)),
                                 desc_k(b + ks * 2 * 64 * 16, 64 * 16, 128), acc);
                        acc = 1;
                    }
                }
                mma_commit(accf(s));
                ++issued;
            }
            if (*abort_flag && issued > 0) {
                // the last commit covers every product issued: wait for it before tensor
                // memory is released
                const long long last = issued - 1;
                const int s = (int)(last % STAGES);
                bool landed = false;
                for (unsigned i = 0; i < WAIT_LIMIT && !landed; ++i)
                    landed = mbar_test(accf(s), (uint32_t)((last / STAGES) & 1));
                if (!landed) atomicExch(status, 2);
            }
        }
        __syncwarp();
    } else {
        // ---- drain (warps 0-3): accumulator -> rows in the stage -> TMA store ----
        const int quarter = warp, r = quarter * 32 + lane;
        long long li = 0;
        for (long long t = blockIdx.x; t < ntiles; t += gridDim.x, ++li) {
            const int s = (int)(li % STAGES);
            const uint32_t u = (uint32_t)(li / STAGES);
            const bool ok = wait_phase(accf(s), u & 1u, abort_flag, status);
            if (!__all_sync(0xffffffffu, ok)) break;
            fence_after_sync();
            float v[32], w[32];
            const uint32_t ta = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(s * 64);
            tmem_ld32(ta, v);
            tmem_ld32(ta + 32, w);
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(acce(s));
            // row r of the tile, columns 0-31 then 32-63, in the SW128 layout of the output boxes
            uint8_t *out = sm + s * STAGE_BYTES + 2 * HALF_BYTES;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const uint32_t off = (uint32_t)(r * 128 + ((c ^ (r & 7)) * 16));
                *reinterpret_cast<float4 *>(out + off) = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
                *reinterpret_cast<float4 *>(out + HALF_BYTES + off) =
                    make_float4(w[4 * c], w[4 * c + 1], w[4 * c + 2], w[4 * c + 3]);
            }
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(rows(s));
            // thread 0 stores the tile once the four warps' rows are written (a bounded wait,
            // not a barrier: a warp that gave up must not hold the others)
            if (warp == 0) {
                bool stored = true;
                if (lane == 0) {
                    stored = wait_phase(rows(s), u & 1u, abort_flag, status);
                    if (stored) {
                        tma_store_box(&map_y, 0, (int)(t * TILE), stage_lo(s));
                        tma_store_box(&map_y, 32, (int)(t * TILE), stage_lo(s) + HALF_BYTES);
                        asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
                        asm volatile("cp.async.bulk.wait_group.read 0;\n" ::: "memory");
                        mbar_arrive(sfree(s));
                    }
                }
                // the warp leaves together (its tensor-memory loads are .sync.aligned)
                if (!__shfl_sync(0xffffffffu, stored, 0)) break;
            }
        }
        if (tid == 0) asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 9) {
        __syncwarp();  // tcgen05.dealloc is .sync.aligned
        tmem_dealloc(tmem, TMEM_COLS);
    }
}

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<EncodeTiledFn>(f);
        return (EncodeTiledFn) nullptr;
    }();
    return fn;
}

// [n][64] FP32 as a 2-D tensor (64 columns, n rows), boxes of 32 columns x 128 rows, 128-byte swizzle
bool patch_map(CUtensorMap *map, const float *p, long long n) {
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return false;
    const cuuint64_t dims[2] = {64, (cuuint64_t)n};
    const cuuint64_t strides[1] = {64 * 4};
    const cuuint32_t box[2] = {32, TILE};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(p), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

std::once_flag g_host_once;
float g_host_kron[2][2][64 * 64];
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
                        g_host_kron[0][0][(r * 8 + c) * 64 + i * 8 + j] = hi;
                        g_host_kron[0][1][(r * 8 + c) * 64 + i * 8 + j] = v - hi;
                        g_host_kron[1][0][(i * 8 + j) * 64 + r * 8 + c] = hi;
                        g_host_kron[1][1][(i * 8 + j) * 64 + r * 8 + c] = v - hi;
                    }
    });
    std::call_once(g_dev_once[dev], [dev] {
        g_dev_err[dev] = cudaMemcpyToSymbol(g_kron, g_host_kron, sizeof(g_host_kron));
        if (g_dev_err[dev] == cudaSuccess) g_dev_err[dev] = cudaFuncSetAttribute(dct2d_tf32, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM);
    });
    return g_dev_err[dev];
}

}  // namespace

// The matrices on device `dev` (once per process and device; synchronous, so call it
// before any stream capture).
cudaError_t dct_tc_init(int dev) {
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    return init_matrix(dev);
}

// y = (T (x) T) x per patch, or with inverse the transposed matrix (T^T (x) T^T); x == y is
// allowed (each tile is loaded before it is stored, and tiles do not overlap).  Returns 0,
// 1 for bad arguments, 2 for a CUDA error.
int dct2d_tf32_run(const float *d_x, float *d_y, long long npatches, int split, int inverse, int *d_status,
                   cudaStream_t stream) {
    if (npatches < 0 || (npatches > 0 && (!d_x || !d_y || !d_status))) return 1;
    // TMA: both matrices 16-byte aligned (rows are 256 bytes apart)
    if (((uintptr_t)d_y & 15) != 0 || ((uintptr_t)d_x & 15) != 0) return 1;
    if (npatches == 0) return 0;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 2;
    if (init_matrix(dev) != cudaSuccess) return 2;
    CUtensorMap mx, my;
    if (!patch_map(&mx, d_x, npatches) || !patch_map(&my, d_y, npatches)) return 2;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long ntiles = (npatches + TILE - 1) / TILE;
    const int grid = (int)(ntiles < sms ? ntiles : sms);
    dct2d_tf32<<<grid, THREADS, SMEM, stream>>>(mx, my, npatches, split, inverse ? 1 : 0, d_status);
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

}  // namespace zb

extern "C" int zb3d_dct2d_tf32(const float *d_x, float *d_y, long long npatches, int split, int *d_status,
                               void *stream) {
    return zb::dct2d_tf32_run(d_x, d_y, npatches, split, 0, d_status, (cudaStream_t)stream);
}
