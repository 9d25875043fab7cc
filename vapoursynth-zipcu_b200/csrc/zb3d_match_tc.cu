// Block matching on the 5th-generation tensor cores (tcgen05), SSD, spatial search.
//
// The plain matcher evaluates every candidate's SSD in the reference's FP32
// operation order (vszipcu src/bm3d.cu:282-302, 614-660).  This form gets the
// same lists with far less FP32 work:
//
//  1. Per tile of 8 x 16 reference blocks (M = 128 rows), the candidate
//     positions of the union of their search windows are streamed through
//     tcgen05.mma (kind::f16, FP32 accumulation in tensor memory) in chunks of
//     N = 256 candidates.  Row m of the product is, for block m and candidate c,
//         d(m, c) = |b_c - c0|^2 - 2 (mu_m - c0) S_c - 2 (a_m - mu_m) . (b_c - c0)
//     (c0 a tile constant, mu_m the block mean, S_c the candidate sum), which
//     equals SSD(a_m, b_c) - |a_m - c0|^2.  The pixel cross term runs on FP16
//     operands; the norm terms enter as FP16 hi/lo pairs; candidates outside
//     block m's window get +16384 through one-hot window terms.  K = 96.
//  2. Pass 1 keeps, per block, the minimum of d over 16 groups of candidates.
//     The eighth smallest group minimum U comes from eight distinct window
//     candidates, so the reference's eighth-best FP32 error is at most
//     U + |a - c0|^2 + eps, where eps bounds |d - (SSD_ref - |a - c0|^2)|.
//  3. Pass 2 recomputes the chunks and collects every candidate with
//     d <= U + 2 eps: a superset of the exact top 8 (ties included).
//  4. The collected candidates (in scan order) get the exact FP32 SSD in the
//     reference's order and go through the reference's insertion rule and self
//     inclusion, so the list is bit-identical to the plain matcher's.
//
// A block whose collection overflows, or a tile whose pixels leave the range
// the FP16 terms are sized for (|x| <= 4), is listed for the exact matcher
// (zb_match_global, gen_mode 2), so the result never depends on the bound
// being tight.
//
// Compiled with -use_fast_math like the other matching kernels: the exact
// re-rank uses explicit __fmul_rn / __fmaf_rn, so its arithmetic is fixed.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "zb3d_args.h"
#include "zb3d_match.cuh"

namespace zb {
namespace tc {

constexpr int BX = 8, BY = 16, M = BX * BY;  // reference blocks per tile
constexpr int N = 256;                       // candidates per MMA chunk
constexpr int K = 96;                        // 64 pixels + 5 norm terms + 8 + 16 window one-hots + 3 zero
constexpr int KSTEPS = K / 16;
constexpr int MAX_UC = 56, MAX_UR = 88;      // candidate union of a tile: columns, rows
constexpr int REG_ROWS = MAX_UR + 7;
constexpr int REG_COLS = 64;                 // staged region columns (union + 7, padded)
constexpr int R16_PITCH = 33;                // 32-bit words per FP16 region row (+1 against bank conflicts)
constexpr int CAP = 96;                      // collected candidates per block
constexpr int THREADS = 256;                 // warps 0-3: one block per thread; warps 4-7: operand builders
constexpr float BIG = 16384.0f;              // window penalty (exact in FP16)
constexpr float RANGE = 4.0f;                // pixel magnitude the FP16 terms are sized for
constexpr unsigned WAIT_LIMIT = 1u << 22;    // polls of an mbarrier before giving up (~0.5 s)

// shared memory plan (bytes); core-matrix layouts need 16-byte alignment
constexpr int SZ_A = M * K * 2;                              // operand A: 128 x 96 FP16
constexpr int SZ_B = N * K * 2;                              // one operand-B slab: 256 x 96 FP16
constexpr int OFF_A = 0;
constexpr int OFF_B = OFF_A + SZ_A;                          // two slabs
constexpr int OFF_R16E = OFF_B + 2 * SZ_B;                   // FP16 region, pairs from even columns
constexpr int SZ_R16 = ((REG_ROWS * R16_PITCH * 4 + 15) / 16) * 16;
constexpr int OFF_R16O = OFF_R16E + SZ_R16 + 64;             // pairs from odd columns (16 banks apart)
constexpr int OFF_SP = OFF_R16O + SZ_R16;                    // per candidate: S hi, S lo, p hi, p lo (FP16)
constexpr int SZ_SP = MAX_UR * MAX_UC * 8;
constexpr int OFF_XP = OFF_SP + SZ_SP;                       // per union column: 8 x-window penalties
constexpr int SZ_XP = (MAX_UC + 1) * 16;
constexpr int OFF_YP = OFF_XP + SZ_XP;                       // per union row: 16 y-window penalties
constexpr int SZ_YP = MAX_UR * 32;
constexpr int OFF_BUF = OFF_YP + SZ_YP;                      // [CAP][128] collected flat indices
constexpr int SZ_BUF = CAP * M * 2;
constexpr int OFF_ROWMAX = OFF_BUF + SZ_BUF;                 // per union row: max candidate |b - c0|^2
constexpr int OFF_MISC = OFF_ROWMAX + MAX_UR * 4;             // mbarriers, TMEM address, reductions
constexpr int SMEM_BYTES = OFF_MISC + 128;
static_assert(SMEM_BYTES <= 227 * 1024, "tensor-core matcher exceeds shared memory");
// during setup the slab area holds the FP32 region and the horizontal sums
constexpr int OFF_REG32 = OFF_B;
constexpr int OFF_HS = OFF_B + REG_ROWS * REG_COLS * 4;
static_assert(REG_ROWS * REG_COLS * 4 + 2 * REG_ROWS * MAX_UC * 4 <= 2 * SZ_B, "setup scratch exceeds slabs");

// core-matrix (no swizzle, K-major) byte offset of element (row, k) in a 96-wide operand
__device__ __forceinline__ int core_off(int row, int kc) { return (row >> 3) * 1536 + kc * 128 + (row & 7) * 16; }

// ---------------------------------------------------------------------------
// PTX wrappers (tcgen05, mbarrier), PTX ISA 8.6+ for sm_100a.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: no swizzle, K-major, start / LBO / SBO in
// 16-byte units, version 1 (bits 46-47) as tcgen05 requires.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP16 A and B (both the same type), FP32
// accumulator, both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t IDESC = (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.u32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar)
                 : "memory");
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint32_t mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t mbar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    return done != 0;
}

// Waits for phase `parity` of an mbarrier, at most WAIT_LIMIT polls; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
    for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_test(mbar, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void tmem_alloc(uint32_t slot_saddr, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(slot_saddr), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(taddr), "r"(ncols) : "memory");
}

// 32 consecutive FP32 columns of this warp's 32 lanes.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
        "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ uint32_t h2u(__half a, __half b) {
    return (uint32_t)__half_as_ushort(a) | ((uint32_t)__half_as_ushort(b) << 16);
}

// FP32 -> FP16 hi/lo pair: x ~= hi + lo to about 22 bits.
__device__ __forceinline__ void split_h(float x, __half &hi, __half &lo) {
    hi = __float2half_rn(x);
    lo = __float2half_rn(x - __half2float(hi));
}

// ---------------------------------------------------------------------------
// Tile geometry.  Tile (blockIdx.x, blockIdx.y) holds reference blocks
// kx0 + [0, 8) x ky0 + [0, 16); block m = 8 * row + column is TMEM lane m.
// The candidate union is [ux0, ux0 + nuc) x [uy0, uy0 + nur), enumerated
// row-major with an odd row stride (flat index f = row * stride + column), so
// that the 16 groups f mod 16 mix rows and columns; an even nuc gets one padded
// column.  Chunk c of the MMA stream is the flat range [256 c, 256 c + 256).
// ---------------------------------------------------------------------------
struct Geom {
    int kx0, ky0, nvx, nvy;
    int ux0, uy0, nuc, nur, stride, flat, nch;
};

__device__ __forceinline__ int block_x(const MatchArgs &a, int kx) { return min(a.bs * kx, a.w - 8); }
__device__ __forceinline__ int block_y(const MatchArgs &a, int ky) { return min(a.bs * ky, a.h - 8); }

__device__ __forceinline__ Geom tile_geom(const MatchArgs &a) {
    Geom g;
    g.kx0 = blockIdx.x * BX;
    g.ky0 = blockIdx.y * BY;
    g.nvx = min(BX, a.nbx - g.kx0);
    g.nvy = min(BY, a.nby - g.ky0);
    const int R = a.range;
    g.ux0 = max(block_x(a, g.kx0) - R, 0);
    g.uy0 = max(block_y(a, g.ky0) - R, 0);
    g.nuc = min(block_x(a, g.kx0 + g.nvx - 1) + R, a.w - 8) - g.ux0 + 1;
    g.nur = min(block_y(a, g.ky0 + g.nvy - 1) + R, a.h - 8) - g.uy0 + 1;
    g.stride = g.nuc | 1;
    g.flat = g.nur * g.stride;
    g.nch = (g.flat + N - 1) / N;
    return g;
}

// Exact SSD in the reference's order (vszipcu src/bm3d.cu:282-302): per column
// even and odd rows accumulate separately, columns join as
// ((s0+s1)+(s2+s3)) + ((s4+s5)+(s6+s7)).  c = reference patch, n = candidate.
__device__ __forceinline__ float exact_ssd(const float (&c)[64], const float *__restrict__ n, int pitch) {
    float s[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float d[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) d[i] = c[i * 8 + j] - __ldg(n + (long long)i * pitch + j);
        float e0 = __fmul_rn(d[0], d[0]);
        float e1 = __fmul_rn(d[1], d[1]);
        e0 = __fmaf_rn(d[2], d[2], e0);
        e1 = __fmaf_rn(d[3], d[3], e1);
        e0 = __fmaf_rn(d[4], d[4], e0);
        e1 = __fmaf_rn(d[5], d[5], e1);
        e0 = __fmaf_rn(d[6], d[6], e0);
        e1 = __fmaf_rn(d[7], d[7], e1);
        s[j] = e0 + e1;
    }
    return ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
}

// Eighth smallest of 16 values (bitonic sort of a register copy).
__device__ __forceinline__ float eighth_smallest(const float (&g)[16]) {
    float v[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = g[i];
#pragma unroll
    for (int k = 2; k <= 16; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const int l = i ^ j;
                if (l > i) {
                    const float lo = fminf(v[i], v[l]), hi = fmaxf(v[i], v[l]);
                    const bool up = (i & k) == 0;
                    v[i] = up ? lo : hi;
                    v[l] = up ? hi : lo;
                }
            }
    return v[7];
}

__device__ __forceinline__ uint32_t fsh(uint32_t lo, uint32_t hi) { return __funnelshift_r(lo, hi, 16); }

// Operand-B slab of chunk c: candidate n of the chunk is row n; its 96 K entries
// are the 64 centred FP16 pixels (patch row i = K core matrix i), then
// [S hi, S lo, S hi, p hi, p lo], the 8 x-window and 16 y-window penalties, 0.
// Run by the 128 builder threads (b = 0..127).
__device__ __forceinline__ void build_slab(unsigned char *smem, const Geom &g, int c, int slab, int b) {
    unsigned char *S = smem + OFF_B + slab * SZ_B;
    const uint32_t *r16e = reinterpret_cast<const uint32_t *>(smem + OFF_R16E);
    const uint32_t *r16o = reinterpret_cast<const uint32_t *>(smem + OFF_R16O);
    const uint2 *sp = reinterpret_cast<const uint2 *>(smem + OFF_SP);
    const uint4 *xpt = reinterpret_cast<const uint4 *>(smem + OFF_XP);
    const uint4 *ypt = reinterpret_cast<const uint4 *>(smem + OFF_YP);
    const uint32_t hb = (uint32_t)__half_as_ushort(__float2half_rn(BIG));
#pragma unroll 1
    for (int n = b; n < N; n += 128) {
        const int f = c * N + n;
        uint4 pc[12];
        bool pad = f >= g.flat;
        int r = 0, cc = 0;
        if (!pad) {
            r = f / g.stride;
            cc = f - r * g.stride;
            pad = cc >= g.nuc;
        }
        if (pad) {  // not a candidate: every x penalty set
#pragma unroll
            for (int i = 0; i < 8; ++i) pc[i] = make_uint4(0, 0, 0, 0);
            pc[8] = make_uint4(0, 0, hb << 16, hb | (hb << 16));
            pc[9] = make_uint4(hb | (hb << 16), hb | (hb << 16), hb, 0);
            pc[10] = make_uint4(0, 0, 0, 0);
            pc[11] = make_uint4(0, 0, 0, 0);
        } else {
            const uint32_t *src = (cc & 1) ? r16o : r16e;
            const int w0 = cc >> 1;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint32_t *rp = src + (r + i) * R16_PITCH + w0;
                pc[i] = make_uint4(rp[0], rp[1], rp[2], rp[3]);
            }
            const uint2 s = sp[r * MAX_UC + cc];
            const uint4 x = xpt[cc];
            const uint4 y0 = ypt[2 * r], y1 = ypt[2 * r + 1];
            pc[8] = make_uint4(s.x, (s.x & 0xffffu) | (s.y << 16), (s.y >> 16) | (x.x << 16), fsh(x.x, x.y));
            pc[9] = make_uint4(fsh(x.y, x.z), fsh(x.z, x.w), fsh(x.w, y0.x), fsh(y0.x, y0.y));
            pc[10] = make_uint4(fsh(y0.y, y0.z), fsh(y0.z, y0.w), fsh(y0.w, y1.x), fsh(y1.x, y1.y));
            pc[11] = make_uint4(fsh(y1.y, y1.z), fsh(y1.z, y1.w), y1.w >> 16, 0);
        }
#pragma unroll
        for (int kc = 0; kc < 12; ++kc) *reinterpret_cast<uint4 *>(S + core_off(n, kc)) = pc[kc];
    }
}

static_assert(OFF_MISC % 16 == 0 && OFF_B % 1024 == 0 && OFF_SP % 16 == 0 && OFF_XP % 16 == 0 &&
                  OFF_YP % 16 == 0 && OFF_R16O % 16 == 0,
              "shared-memory regions must stay 16-byte aligned");

__device__ __forceinline__ void list_fallback(const MatchArgs &a, int bi) {
    const int k = atomicAdd(a.tc_ws, 1);
    a.tc_ws[kTcWsList + k] = bi;
}

// One CTA per tile of 8 x 16 reference blocks.  Warps 0-3 own the blocks (one
// per thread, TMEM lanes 0-127); warps 4-7 build the operand-B slabs; thread
// 128 issues the MMAs.  Jobs j = 0 .. 2 nch - 1 are (pass j / nch, chunk
// j mod nch); job j accumulates into TMEM columns [256 (j & 1), +256) from slab
// j & 1 and completes phase j >> 1 of mbarrier j & 1.  Iteration j builds slab
// j + 1, reads job j - 1 out of TMEM while job j runs, and issues job j + 1.
__global__ void __launch_bounds__(THREADS, 1) zb_match_tc(MatchArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Geom g = tile_geom(a);
    const int H = a.h, R = a.range, P = a.pitch;
    const float *plane = a.frames + (long long)a.radius * a.fstride;

    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + OFF_MISC);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + OFF_MISC + 16);
    int *last_job = reinterpret_cast<int *>(smem + OFF_MISC + 20);
    int *oor = reinterpret_cast<int *>(smem + OFF_MISC + 24);
    float *red = reinterpret_cast<float *>(smem + OFF_MISC + 32);      // [0..3] mean sums, [4..7] counts
    int *tmax = reinterpret_cast<int *>(smem + OFF_MISC + 64);         // [0] max |S|, bits of a non-negative float
    float *rowmax = reinterpret_cast<float *>(smem + OFF_ROWMAX);
    float *reg = reinterpret_cast<float *>(smem + OFF_REG32);
    float *hs = reinterpret_cast<float *>(smem + OFF_HS);
    float *hp = hs + REG_ROWS * MAX_UC;
    uint16_t *buf = reinterpret_cast<uint16_t *>(smem + OFF_BUF);

    if (warp == 0) tmem_alloc(smem_u32(tslot), 512);
    if (tid == 0) {
        mbar_init(smem_u32(&mbar[0]), 1);
        mbar_init(smem_u32(&mbar[1]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        *last_job = -1;
        *oor = 0;
        tmax[0] = 0;
    }
    for (int r = tid; r < MAX_UR; r += THREADS) rowmax[r] = 0.0f;

    // ---- stage the FP32 region: union rows + 7, union columns + 7 -------------
    const int rr = g.nur + 7, rc = g.nuc + 7;
    for (int i = tid; i < rr * REG_COLS; i += THREADS) {
        const int row = i >> 6, col = i & 63;
        reg[i] = col < rc ? __ldg(plane + (long long)(g.uy0 + row) * P + g.ux0 + col) : 0.0f;
    }
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *tslot;

    // ---- per-block means; c0 = mean of the tile's block means -----------------
    const int bxl = tid & 7, byl = (tid >> 3) & 15;
    const bool valid = tid < M && bxl < g.nvx && byl < g.nvy;
    const int xb = block_x(a, g.kx0 + bxl), yb = block_y(a, g.ky0 + byl);
    const float *ra = reg + (yb - g.uy0) * REG_COLS + (xb - g.ux0);  // dereferenced only when valid
    float mu = 0.0f;
    if (valid) {
        float s = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) s += ra[i * REG_COLS + j];
        mu = s * (1.0f / 64.0f);
    }
    if (warp < 4) {
        float s = valid ? mu : 0.0f, n = valid ? 1.0f : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            n += __shfl_xor_sync(0xffffffffu, n, o);
        }
        if (lane == 0) {
            red[warp] = s;
            red[4 + warp] = n;
        }
    }
    __syncthreads();
    const float c0 = ((red[0] + red[1]) + (red[2] + red[3])) / fmaxf((red[4] + red[5]) + (red[6] + red[7]), 1.0f);

    // ---- FP16 centred region (even / odd pair copies), range check, row sums --
    uint32_t *r16e = reinterpret_cast<uint32_t *>(smem + OFF_R16E);
    uint32_t *r16o = reinterpret_cast<uint32_t *>(smem + OFF_R16O);
    bool bad = false;
    for (int i = tid; i < rr * 32; i += THREADS) {
        const int row = i >> 5, w = i & 31, c = 2 * w;
        const float *rp = reg + row * REG_COLS;
        const float x0 = rp[c], x1 = rp[c + 1], x2 = c + 2 < REG_COLS ? rp[c + 2] : 0.0f;
        const __half h0 = __float2half_rn(c < rc ? x0 - c0 : 0.0f);
        const __half h1 = __float2half_rn(c + 1 < rc ? x1 - c0 : 0.0f);
        const __half h2 = __float2half_rn(c + 2 < rc ? x2 - c0 : 0.0f);
        r16e[row * R16_PITCH + w] = h2u(h0, h1);
        r16o[row * R16_PITCH + w] = h2u(h1, h2);
        bad |= (c < rc && !(fabsf(x0) <= RANGE)) || (c + 1 < rc && !(fabsf(x1) <= RANGE));
    }
    if (bad) *oor = 1;
    for (int i = tid; i < rr * g.nuc; i += THREADS) {
        const int row = i / g.nuc, c = i - row * g.nuc;
        const float *rp = reg + row * REG_COLS + c;
        float s = 0.0f, q = 0.0f;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const float d = rp[j] - c0;
            s += d;
            q = fmaf(d, d, q);
        }
        hs[row * MAX_UC + c] = s;
        hp[row * MAX_UC + c] = q;
    }
    __syncthreads();

    // ---- per-candidate S, p as FP16 hi/lo; window penalty tables; maxima -----
    uint2 *sp = reinterpret_cast<uint2 *>(smem + OFF_SP);
    float smax = 0.0f;
    for (int i = tid; i < g.nur * g.nuc; i += THREADS) {
        const int r = i / g.nuc, c = i - r * g.nuc;
        float s = 0.0f, q = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            s += hs[(r + k) * MAX_UC + c];
            q += hp[(r + k) * MAX_UC + c];
        }
        __half sh, sl, ph, pl;
        split_h(s, sh, sl);
        split_h(q, ph, pl);
        sp[r * MAX_UC + c] = make_uint2(h2u(sh, sl), h2u(ph, pl));
        smax = fmaxf(smax, fabsf(s));
        atomicMax(reinterpret_cast<int *>(rowmax) + r, __float_as_int(q));  // q >= 0: int order = float order
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) smax = fmaxf(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    if (lane == 0) atomicMax(tmax, __float_as_int(smax));
    const __half hbig = __float2half_rn(BIG), hzero = __float2half_rn(0.0f);
    for (int c = tid; c < g.stride; c += THREADS) {
        __half p[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const bool out = c >= g.nuc || (j < g.nvx && abs(g.ux0 + c - block_x(a, g.kx0 + j)) > R);
            p[j] = out ? hbig : hzero;
        }
        reinterpret_cast<uint4 *>(smem + OFF_XP)[c] = make_uint4(h2u(p[0], p[1]), h2u(p[2], p[3]), h2u(p[4], p[5]),
                                                                 h2u(p[6], p[7]));
    }
    for (int r = tid; r < g.nur; r += THREADS) {
        __half p[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            const bool out = i < g.nvy && abs(g.uy0 + r - block_y(a, g.ky0 + i)) > R;
            p[i] = out ? hbig : hzero;
        }
        uint4 *yp = reinterpret_cast<uint4 *>(smem + OFF_YP) + 2 * r;
        yp[0] = make_uint4(h2u(p[0], p[1]), h2u(p[2], p[3]), h2u(p[4], p[5]), h2u(p[6], p[7]));
        yp[1] = make_uint4(h2u(p[8], p[9]), h2u(p[10], p[11]), h2u(p[12], p[13]), h2u(p[14], p[15]));
    }
    __syncthreads();

    // ---- operand A (one row per block) and the block's error bound ------------
    float eps = 0.0f;
    if (tid < M) {
        uint4 pa[12];
        if (valid) {
            float an2 = 0.0f, ah2 = 0.0f;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                __half h[8];
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const float x = ra[i * REG_COLS + j];
                    const float d = x - mu, e = x - c0;
                    an2 = fmaf(d, d, an2);
                    ah2 = fmaf(e, e, ah2);
                    h[j] = __float2half_rn(-2.0f * d);
                }
                pa[i] = make_uint4(h2u(h[0], h[1]), h2u(h[2], h[3]), h2u(h[4], h[5]), h2u(h[6], h[7]));
            }
            const float nu = mu - c0;
            __half nh, nl;
            split_h(nu, nh, nl);
            __half e[32];
            e[0] = __float2half_rn(-2.0f * __half2float(nh));
            e[1] = e[0];
            e[2] = __float2half_rn(-2.0f * __half2float(nl));
            e[3] = e[4] = __float2half_rn(1.0f);
#pragma unroll
            for (int j = 0; j < 8; ++j) e[5 + j] = j == bxl ? __float2half_rn(1.0f) : hzero;
#pragma unroll
            for (int i = 0; i < 16; ++i) e[13 + i] = i == byl ? __float2half_rn(1.0f) : hzero;
            e[29] = e[30] = e[31] = hzero;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                pa[8 + k] = make_uint4(h2u(e[8 * k], e[8 * k + 1]), h2u(e[8 * k + 2], e[8 * k + 3]),
                                       h2u(e[8 * k + 4], e[8 * k + 5]), h2u(e[8 * k + 6], e[8 * k + 7]));
            // eps bounds |d - (SSD_ref - |a - c0|^2)| over the block's window:
            // FP16 rounding of both cross-term operands (2^-11 each, x2 for the factor 2),
            // FP32 accumulation of 96 terms and the hi/lo splits (2^-15 of the term sizes).
            const int r0 = max(yb - R, 0) - g.uy0, r1 = min(yb + R, H - 8) - g.uy0;
            float pm = 0.0f;
            for (int r = r0; r <= r1; ++r) pm = fmaxf(pm, rowmax[r]);
            const float an = sqrtf(an2), bm = sqrtf(pm);
            const float sm = __int_as_float(tmax[0]);
            eps = 1.01f * 0.001953125f * an * bm +
                  3.0517578125e-05f * (2.0f * an * bm + 2.0f * fabsf(nu) * sm + pm + ah2 + 1.0f);
        } else {
#pragma unroll
            for (int k = 0; k < 12; ++k) pa[k] = make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int kc = 0; kc < 12; ++kc) *reinterpret_cast<uint4 *>(smem + OFF_A + core_off(tid, kc)) = pa[kc];
    }
    __syncthreads();  // region scratch (slab area) is dead from here on

    // ---- the MMA stream ----------------------------------------------------------
    const int nch = g.nch, J = 2 * nch;
    const uint32_t a_saddr = smem_u32(smem + OFF_A), b_saddr = smem_u32(smem + OFF_B);
    const uint32_t mb0 = smem_u32(&mbar[0]);
    int flo = 0, fhi = 0;  // flat range the warp's blocks need (warp-uniform)
    if (warp < 4) {
        const int by0 = 4 * warp, nr = min(4, g.nvy - by0);
        if (nr > 0) {
            flo = (max(block_y(a, g.ky0 + by0) - R, 0) - g.uy0) * g.stride;
            fhi = (min(block_y(a, g.ky0 + by0 + nr - 1) + R, H - 8) - g.uy0 + 1) * g.stride;
        }
    }
    const float kInf = __int_as_float(0x7f800000);
    float gm[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) gm[i] = kInf;
    float T = -kInf;  // collection threshold, set after the last pass-1 job (stays -inf for idle lanes)
    int cnt = 0;
    const bool dbg = a.tc_dbg != nullptr && blockIdx.x == 0 && blockIdx.y == 0;

    auto issue = [&](int job) {
        const int s = job & 1;
        const uint32_t d = tbase + (uint32_t)(s * N);
        const uint32_t bsa = b_saddr + s * SZ_B;
#pragma unroll
        for (int kk = 0; kk < KSTEPS; ++kk)
            mma_f16(d, make_desc(a_saddr + kk * 256, 128, 1536), make_desc(bsa + kk * 256, 128, 1536), kk);
        mma_commit(mb0 + 8 * s);
        *last_job = job;
    };

    if (warp >= 4) build_slab(smem, g, 0, 0, tid - 128);
    fence_async_smem();
    __syncthreads();
    if (tid == 128) {
        fence_after_sync();
        issue(0);
    }
    int timeout = 0, stop = 0;
    for (int j = 0; j <= J; ++j) {
        if (warp >= 4) {
            if (j + 1 < J) {
                // slab (j + 1) & 1 was last read by job j - 1
                if (j >= 1 && !mbar_wait(mb0 + 8 * ((j - 1) & 1), ((j - 1) >> 1) & 1)) timeout = 1;
                build_slab(smem, g, (j + 1) % nch, (j + 1) & 1, tid - 128);
                fence_async_smem();
            }
        } else if (j >= 1) {
            const int jj = j - 1, base = (jj % nch) * N;
            if (!mbar_wait(mb0 + 8 * (jj & 1), (jj >> 1) & 1)) timeout = 1;
            fence_after_sync();
            const bool pass2 = jj >= nch;
            const int s0 = max(flo - base, 0) >> 5;
            const int s1 = (min(fhi - base, N) + 31) >> 5;
            const uint32_t tl = tbase + ((uint32_t)(32 * warp) << 16) + (uint32_t)((jj & 1) * N);
            for (int sc = s0; sc < s1; ++sc) {
                float v[32];
                __syncwarp();  // tcgen05.ld is warp-collective: reconverge after the collection loop
                tmem_ld32(tl + 32 * sc, v);
                if (!pass2) {
#pragma unroll
                    for (int r = 0; r < 32; ++r) gm[r & 15] = fminf(gm[r & 15], v[r]);
                    if (dbg) {
                        float *o = a.tc_dbg + (size_t)tid * (nch * N) + base + 32 * sc;
#pragma unroll
                        for (int r = 0; r < 32; ++r) o[r] = v[r];
                    }
                } else {
                    unsigned hit = 0;
#pragma unroll
                    for (int r = 0; r < 32; ++r) hit |= v[r] <= T ? (1u << r) : 0u;
                    while (hit) {
                        const int r = __ffs(hit) - 1;
                        hit &= hit - 1;
                        if (cnt < CAP) buf[cnt * M + tid] = (uint16_t)(base + 32 * sc + r);
                        ++cnt;
                    }
                }
            }
            if (jj == nch - 1 && valid) T = eighth_smallest(gm) + 2.0f * eps;
            fence_before_sync();
        }
        stop = __syncthreads_or(timeout);
        if (stop) break;
        if (tid == 128 && j + 1 < J) {
            fence_after_sync();
            issue(j + 1);
        }
    }
    // ---- drain and release tensor memory -------------------------------------------
    if (stop && tid == 128) {
        const int L = *last_job;  // its completion implies every earlier MMA's
        if (L >= 0) mbar_wait(mb0 + 8 * (L & 1), (L >> 1) & 1);
    }
    if (stop && tid == 0) a.tc_ws[1] = 1;
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tbase, 512);
    }

    // ---- exact re-rank of the collected candidates --------------------------------
    if (warp >= 4) return;
    const bool fb = valid && (stop || *oor || cnt > CAP || !(T < 0.5f * BIG));
    if (valid) {
        const int bi = (g.ky0 + byl) * a.nbx + (g.kx0 + bxl);
        if (fb) {
            list_fallback(a, bi);
        } else {
            float c[64];
            const float *pa = plane + (long long)yb * P + xb;
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 8; ++j) c[i * 8 + j] = __ldg(pa + (long long)i * P + j);
            float e[8];
            int q[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                e[i] = ZB_FLT_MAX;
                q[i] = 0;
            }
            for (int s = 0; s < cnt; ++s) {  // flat order = the reference's scan order
                const int f = buf[s * M + tid];
                const int r = f / g.stride, cc = f - r * g.stride;
                if (r >= g.nur || cc >= g.nuc) continue;  // penalised positions are never collected
                const int cx = g.ux0 + cc, cy = g.uy0 + r;
                const float err = exact_ssd(c, plane + (long long)cy * P + cx, P);
                if (err < e[7]) top8_insert(e, q, err, pack_pos(cx, cy));
            }
            store_list(a, bi, xb, yb, e, q);
        }
    }
    if (a.tc_stats) {
        const unsigned nval = __popc(__ballot_sync(0xffffffffu, valid));
        const unsigned nfb = __popc(__ballot_sync(0xffffffffu, fb));
        const unsigned ns = __reduce_add_sync(0xffffffffu, valid && !fb ? (unsigned)cnt : 0u);
        if (lane == 0) {
            atomicAdd(a.tc_stats + 1, (unsigned long long)nval);
            atomicAdd(a.tc_stats + 2, (unsigned long long)ns);
            atomicAdd(a.tc_stats + 3, (unsigned long long)nfb);
        }
        if (tid == 0) atomicAdd(a.tc_stats, 1ull);
    }
}

}  // namespace tc

// The tensor-core form covers SSD spatial matching when a tile's candidate
// union fits the shared-memory plan (block_step 4 with bm_range <= 13, for
// example); everything else stays on the plain kernels.
bool tc_eligible(const MatchArgs &a) {
    return a.range >= 3 && a.w >= 16 && a.h >= 16 && 7 * a.bs + 2 * a.range + 1 <= tc::MAX_UC &&
           15 * a.bs + 2 * a.range + 1 <= tc::MAX_UR;
}

cudaError_t launch_match_tc(const MatchArgs &a, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(a.tc_ws, 0, kTcWsList * sizeof(int), st);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(tc::zb_match_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM_BYTES);
    if (e != cudaSuccess) return e;
    const dim3 grid((a.nbx + tc::BX - 1) / tc::BX, (a.nby + tc::BY - 1) / tc::BY);
    tc::zb_match_tc<<<grid, tc::THREADS, tc::SMEM_BYTES, st>>>(a);
    return cudaGetLastError();
}

// Flat candidates per tile row of the debug dump (tile (0, 0)): nch * 256.
int tc_debug_cols(const MatchArgs &a) {
    const int R = a.range;
    const int nvx = a.nbx < tc::BX ? a.nbx : tc::BX, nvy = a.nby < tc::BY ? a.nby : tc::BY;
    const int x1 = std::min(std::min(a.bs * (nvx - 1), a.w - 8) + R, a.w - 8);
    const int y1 = std::min(std::min(a.bs * (nvy - 1), a.h - 8) + R, a.h - 8);
    const int nuc = x1 + 1, nur = y1 + 1;
    const int flat = nur * (nuc | 1);
    return (flat + tc::N - 1) / tc::N * tc::N;
}

}  // namespace zb
