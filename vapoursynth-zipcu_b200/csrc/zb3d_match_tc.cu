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
#include "zb3d_tcgen05.cuh"

namespace zb {
namespace tc {

using namespace tc05;

constexpr int BX = 8, BY = 16, M = BX * BY;  // reference blocks per tile
constexpr int N = 128;                       // candidates per MMA chunk
constexpr int NSLOT = 4;                     // chunks in flight: slabs, TMEM accumulators (NSLOT * N = 512 columns)
constexpr int K = 96;                        // 64 pixels + 5 norm terms + 8 + 16 window one-hots + 3 zero
constexpr int KSTEPS = K / 16;
constexpr int MAX_UC = 56, MAX_UR = 88;      // candidate union of a tile: columns, rows
constexpr int REG_ROWS = MAX_UR + 7;
constexpr int REG_COLS = 64;                 // staged region columns (union + 7, padded)
constexpr int R16_PITCH = 33;                // 32-bit words per FP16 region row (+1 against bank conflicts)
constexpr int CAP = 48;                      // collected candidates per block and job parity
constexpr int THREADS = 416;                 // warps 0-7: blocks (two per block: even / odd jobs), 8-11: operand
                                             // builders, 12: MMA issuer
constexpr int NWARPS = THREADS / 32;
constexpr float BIG = 16384.0f;              // window penalty (exact in FP16)
constexpr float RANGE = 4.0f;                // pixel magnitude the FP16 terms are sized for
constexpr unsigned WAIT_LIMIT = 1u << 22;    // polls of an mbarrier before giving up (~0.5 s)

// shared memory plan (bytes); core-matrix layouts need 16-byte alignment
constexpr int SZ_A = M * K * 2;                              // operand A: 128 x 96 FP16
constexpr int SZ_B = N * K * 2;                              // one operand-B slab: 128 x 96 FP16
constexpr int OFF_A = 0;
constexpr int OFF_B = OFF_A + SZ_A;                          // NSLOT slabs
constexpr int OFF_R16E = OFF_B + NSLOT * SZ_B;               // FP16 region, pairs from even columns
constexpr int SZ_R16 = ((REG_ROWS * R16_PITCH * 4 + 15) / 16) * 16;
constexpr int OFF_R16O = OFF_R16E + SZ_R16 + 64;             // pairs from odd columns (16 banks apart)
constexpr int OFF_SP = OFF_R16O + SZ_R16;                    // per candidate: S hi, S lo, p hi, p lo (FP16)
constexpr int SZ_SP = MAX_UR * MAX_UC * 8;
constexpr int OFF_XP = OFF_SP + SZ_SP;                       // per union column: 8 x-window penalties
constexpr int SZ_XP = (MAX_UC + 1) * 16;
constexpr int OFF_YP = OFF_XP + SZ_XP;                       // per union row: 16 y-window penalties
constexpr int SZ_YP = MAX_UR * 32;
constexpr int OFF_BUF = OFF_YP + SZ_YP;                      // [2][CAP][128] collected flat indices per job parity
constexpr int SZ_BUF = 2 * CAP * M * 2;
constexpr int OFF_ROWMAX = OFF_BUF + SZ_BUF;                 // per union row: max candidate |b - c0|^2
constexpr int OFF_XCH = OFF_ROWMAX + MAX_UR * 4;              // pass-boundary exchange: minima [128][17], T, eps, counts
constexpr int SZ_XCH = (M * 17 + 5 * M) * 4;
constexpr int OFF_MISC = OFF_XCH + SZ_XCH;                    // mbarriers, TMEM address, reductions
constexpr int SMEM_BYTES = OFF_MISC + 160;  // 3 x NSLOT mbarriers, TMEM address, flags, reductions
static_assert(SMEM_BYTES <= 227 * 1024, "tensor-core matcher exceeds shared memory");
// during setup the slab area holds the FP32 region and the horizontal sums
constexpr int OFF_REG32 = OFF_B;
constexpr int OFF_HS = OFF_B + REG_ROWS * REG_COLS * 4;
static_assert(REG_ROWS * REG_COLS * 4 + 2 * REG_ROWS * MAX_UC * 4 <= NSLOT * SZ_B, "setup scratch exceeds slabs");

// Operands are K-major with the 64-byte swizzle: per 8-row group, K = 96 is three
// 512-byte atoms of 8 rows x 32 elements; in row r of an atom the 16-byte chunk
// c (8 elements) sits at chunk c ^ ((r >> 1) & 3).  core_off = byte offset of the
// 16-byte piece kc (K elements 8 kc .. 8 kc + 7) of a row.
__device__ __forceinline__ int core_off(int row, int kc) {
    return (row >> 3) * 1536 + (kc >> 2) * 512 + (row & 7) * 64 + (((kc & 3) ^ ((row >> 1) & 3)) << 4);
}

// ---------------------------------------------------------------------------
// Operand descriptors and waits of this kernel (the generic tcgen05 / mbarrier
// wrappers are in zb3d_tcgen05.cuh).
// ---------------------------------------------------------------------------

// Shared-memory matrix descriptor, K-major with the 64-byte swizzle (layout type 4
// at bits 61-63): start address and SBO (stride of 8-row groups, 1536 bytes) in
// 16-byte units, LBO 1 (unused by swizzled K-major layouts), version 1 at bits
// 46-47 as tcgen05 requires, base offset 0 (atoms are 512-byte aligned).  K step
// kk (16 elements) starts at atom kk / 2, byte 32 (kk % 2).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3fff) | (1ull << 16) | ((uint64_t)(1536 >> 4) << 32) | (1ull << 46) |
           (4ull << 61);
}
__device__ __forceinline__ uint32_t kstep_off(int kk) { return (uint32_t)((kk >> 1) * 512 + (kk & 1) * 32); }

// Instruction descriptor of kind::f16: FP16 A and B (both the same type), FP32
// accumulator, both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t IDESC = (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    mma_kind_f16(tmem_d, adesc, bdesc, IDESC, accumulate);
}

// Waits for phase `parity` of an mbarrier, at most WAIT_LIMIT polls; false on
// timeout.  `polls` counts the unsuccessful polls.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, unsigned &polls) {
    for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_test(mbar, parity)) {
            polls += i;
            return true;
        }
        if (i > 64) __nanosleep(64);
    }
    return false;
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
// ((s0+s1)+(s2+s3)) + ((s4+s5)+(s6+s7)).  Two columns go through each packed
// FP32x2 instruction; each lane keeps its own chain and rounding, so the value is
// the scalar one.  nc = the reference patch negated (n + (-c) == -(c - n)
// exactly), column pairs (2p, 2p + 1) per row; n = the candidate.
__device__ __forceinline__ float exact_ssd2(const float2 (&nc)[8][4], const float *n, int pitch) {
    float s[8];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        float2 d[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) d[i] = __fadd2_rn(make_float2(n[i * pitch + 2 * p], n[i * pitch + 2 * p + 1]), nc[i][p]);
        float2 e0 = __fmul2_rn(d[0], d[0]);
        float2 e1 = __fmul2_rn(d[1], d[1]);
        e0 = __ffma2_rn(d[2], d[2], e0);
        e1 = __ffma2_rn(d[3], d[3], e1);
        e0 = __ffma2_rn(d[4], d[4], e0);
        e1 = __ffma2_rn(d[5], d[5], e1);
        e0 = __ffma2_rn(d[6], d[6], e0);
        e1 = __ffma2_rn(d[7], d[7], e1);
        const float2 t = __fadd2_rn(e0, e1);
        s[2 * p] = t.x;
        s[2 * p + 1] = t.y;
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

// three-operand minimum (sm_100)
__device__ __forceinline__ float min3(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// floor(f / s) for f < 2^16, s < 2^10: multiply by 2^32 / s rounded up (error < 2^-16)
__device__ __forceinline__ int div_small(unsigned f, unsigned long long inv) { return (int)((f * inv) >> 32); }

// Operand-B slab of chunk c: candidate n of the chunk is row n; its 96 K entries
// are the 64 centred FP16 pixels (patch row i = K core matrix i), then
// [S hi, S lo, S hi, p hi, p lo], the 8 x-window and 16 y-window penalties, 0.
// Run by the 128 builder threads (b = 0..127), one candidate each.
__device__ __forceinline__ void build_slab(unsigned char *smem, const Geom &g, int c, int slab, int b) {
    unsigned char *S = smem + OFF_B + slab * SZ_B;
    const uint32_t *r16e = reinterpret_cast<const uint32_t *>(smem + OFF_R16E);
    const uint32_t *r16o = reinterpret_cast<const uint32_t *>(smem + OFF_R16O);
    const uint2 *sp = reinterpret_cast<const uint2 *>(smem + OFF_SP);
    const uint4 *xpt = reinterpret_cast<const uint4 *>(smem + OFF_XP);
    const uint4 *ypt = reinterpret_cast<const uint4 *>(smem + OFF_YP);
    const uint32_t hb = (uint32_t)__half_as_ushort(__float2half_rn(BIG));
    const unsigned long long inv = (0x100000000ull + g.stride - 1) / g.stride;
#pragma unroll 2
    for (int n = b; n < N; n += 128) {
        const int f = c * N + n;
        uint4 pc[12];
        bool pad = f >= g.flat;
        int r = 0, cc = 0;
        if (!pad) {
            r = div_small((unsigned)f, inv);
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

static_assert(OFF_MISC % 16 == 0 && OFF_B % 512 == 0 && SZ_B % 512 == 0 && OFF_SP % 16 == 0 && OFF_XP % 16 == 0 &&
                  OFF_YP % 16 == 0 && OFF_R16O % 16 == 0,
              "shared-memory regions must stay 16-byte aligned");

__device__ __forceinline__ void list_fallback(const MatchArgs &a, int bi) {
    const int k = atomicAdd(a.tc_ws, 1);
    a.tc_ws[kTcWsList + k] = bi;
}


// Asynchronous copy of the tile's FP32 region (union rows + 7, columns + 7) into
// shared memory at pitch REG_COLS; columns beyond it are zero-filled.
__device__ __forceinline__ void stage_region(float *reg, const float *plane, int P, const Geom &g, int tid) {
    const int rr = g.nur + 7, rc = g.nuc + 7;
    for (int i = tid; i < rr * REG_COLS; i += THREADS) {
        const int row = i >> 6, col = i & 63;
        const bool ok = col < rc;
        const float *src = plane + (long long)(g.uy0 + row) * P + g.ux0 + (ok ? col : 0);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_u32(reg + i)), "l"(src),
                     "r"(ok ? 4 : 0)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// One CTA per tile of 8 x 16 reference blocks.  Warps 0-7 own the blocks: warp w
// reads TMEM lanes 32 (w mod 4) .. + 31 (block m = lane index) for the jobs of
// parity w / 4.  Warps 8-11 build the operand-B slabs, lane 0 of warp 12 issues
// the MMAs.  Jobs j = 0 .. 2 nch - 1 are (pass j / nch, chunk
// j mod nch) and use slot s = j mod NSLOT: slab s, TMEM columns [128 s, 128 s + 128).
// The roles meet only at mbarriers: full[s] (slab built, 4 builder warps),
// done[s] (MMAs of the job complete, tcgen05.commit) and free[s] (TMEM slot read,
// the 4 warps of the job's parity); job j waits for phase j / NSLOT, and every producer of
// phase u + 1 first waits for a consumer of phase u, so parities never alias.
__global__ void __launch_bounds__(THREADS, 1) zb_match_tc(MatchArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Geom g = tile_geom(a);
    const int H = a.h, R = a.range, P = a.pitch;
    const float *plane = a.frames + (long long)a.radius * a.fstride;

    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + OFF_MISC);    // full[NSLOT], done[NSLOT], free[NSLOT]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + OFF_MISC + 96);
    int *oor = reinterpret_cast<int *>(smem + OFF_MISC + 100);
    int *tmax = reinterpret_cast<int *>(smem + OFF_MISC + 104);        // max |S|, bits of a non-negative float
    float *red = reinterpret_cast<float *>(smem + OFF_MISC + 112);     // [0..3] mean sums, [4..7] counts
    float *rowmax = reinterpret_cast<float *>(smem + OFF_ROWMAX);
    float *reg = reinterpret_cast<float *>(smem + OFF_REG32);
    float *hs = reinterpret_cast<float *>(smem + OFF_HS);
    float *hp = hs + REG_ROWS * MAX_UC;
    uint16_t *buf = reinterpret_cast<uint16_t *>(smem + OFF_BUF);
    const uint32_t mb = smem_u32(mbar);
    const uint32_t full0 = mb, done0 = mb + 8 * NSLOT, free0 = mb + 16 * NSLOT;  // slot s at +8 s

    unsigned long long *prof = a.tc_prof ? a.tc_prof + 16 * (blockIdx.y * gridDim.x + blockIdx.x) : nullptr;
    unsigned polls = 0;
    if (prof && tid == 0) prof[0] = clock64();
    if (warp == 0) tmem_alloc(smem_u32(tslot), 512);
    if (tid == 0) {
        for (int k = 0; k < NSLOT; ++k) {
            mbar_init(full0 + 8 * k, 4);
            mbar_init(done0 + 8 * k, 1);
            mbar_init(free0 + 8 * k, 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        *oor = 0;
        *tmax = 0;
    }
    stage_region(reg, plane, P, g, tid);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *tslot;
    if (prof && tid == 0) prof[1] = clock64();

    // ---- per-block means; c0 = mean of the tile's block means -----------------
    const int bxl = tid & 7, byl = (tid >> 3) & 15;
    const bool valid = tid < M && bxl < g.nvx && byl < g.nvy;
    const int xb = block_x(a, g.kx0 + bxl), yb = block_y(a, g.ky0 + byl);
    const int ra_off = (yb - g.uy0) * REG_COLS + (xb - g.ux0);  // used only when valid
    float mu = 0.0f;
    if (valid) {
        float s = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) s += reg[ra_off + i * REG_COLS + j];
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
    // one warp per region row: lane = 32-bit word of the FP16 copies / union column
    const int rr = g.nur + 7, rc = g.nuc + 7;
    uint32_t *r16e = reinterpret_cast<uint32_t *>(smem + OFF_R16E);
    uint32_t *r16o = reinterpret_cast<uint32_t *>(smem + OFF_R16O);
    bool bad = false;
    for (int row = warp; row < rr; row += NWARPS) {
        const float *rp = reg + row * REG_COLS;
        const int c = 2 * lane;
        const float x0 = rp[c], x1 = rp[c + 1], x2 = lane < 31 ? rp[c + 2] : 0.0f;
        const __half h0 = __float2half_rn(c < rc ? x0 - c0 : 0.0f);
        const __half h1 = __float2half_rn(c + 1 < rc ? x1 - c0 : 0.0f);
        const __half h2 = __float2half_rn(c + 2 < rc ? x2 - c0 : 0.0f);
        r16e[row * R16_PITCH + lane] = h2u(h0, h1);
        r16o[row * R16_PITCH + lane] = h2u(h1, h2);
        bad |= (c < rc && !(fabsf(x0) <= RANGE)) || (c + 1 < rc && !(fabsf(x1) <= RANGE));
        for (int cc = lane; cc < g.nuc; cc += 32) {
            float s = 0.0f, q = 0.0f;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float d = rp[cc + j] - c0;
                s += d;
                q = fmaf(d, d, q);
            }
            hs[row * MAX_UC + cc] = s;
            hp[row * MAX_UC + cc] = q;
        }
    }
    if (bad) *oor = 1;
    __syncthreads();
    if (prof && tid == 0) prof[2] = clock64();

    // ---- per-candidate S, p as FP16 hi/lo, row maxima of p; penalty tables ----
    uint2 *sp = reinterpret_cast<uint2 *>(smem + OFF_SP);
    float smax = 0.0f;
    for (int r = warp; r < g.nur; r += NWARPS) {
        float mx = 0.0f;
        for (int c = lane; c < g.nuc; c += 32) {
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
            mx = fmaxf(mx, q);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0) rowmax[r] = mx;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) smax = fmaxf(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    if (lane == 0) atomicMax(tmax, __float_as_int(smax));
    const __half hbig = __float2half_rn(BIG), hzero = __float2half_rn(0.0f), hone = __float2half_rn(1.0f);
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
    if (prof && tid == 0) prof[3] = clock64();

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
                    const float x = reg[ra_off + i * REG_COLS + j];
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
            e[3] = e[4] = hone;
#pragma unroll
            for (int j = 0; j < 8; ++j) e[5 + j] = j == bxl ? hone : hzero;
#pragma unroll
            for (int i = 0; i < 16; ++i) e[13 + i] = i == byl ? hone : hzero;
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
            const float sm = __int_as_float(*tmax);
            eps = 1.01f * 0.001953125f * an * bm +
                  3.0517578125e-05f * (2.0f * an * bm + 2.0f * fabsf(nu) * sm + pm + ah2 + 1.0f);
        } else {
#pragma unroll
            for (int k = 0; k < 12; ++k) pa[k] = make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int kc = 0; kc < 12; ++kc) *reinterpret_cast<uint4 *>(smem + OFF_A + core_off(tid, kc)) = pa[kc];
        fence_async_smem();
    }
    __syncthreads();  // the FP32 region in the slab area is dead from here on

    // ---- the MMA stream ------------------------------------------------------------
    const int nch = g.nch, J = 2 * nch;
    float *gmx = reinterpret_cast<float *>(smem + OFF_XCH);  // [128][17] odd-parity minima
    float *Tx = gmx + M * 17, *epsx = Tx + M;
    int *cntx = reinterpret_cast<int *>(epsx + M);           // [2][128] collection counts per job parity
    int *okx = cntx + 2 * M;                                 // [128] bound usable
    if (tid < M) epsx[tid] = eps;
    __syncthreads();
    if (prof && tid == 0) prof[4] = clock64();
    int timeout = 0, last = -1;
    long long t_ld = 0;  // profiling: cycles in TMEM loads (block warps) or slab builds (builders)
    int n_ld = 0;
    if (warp < 8) {
        const int q = warp & 3, par = warp >> 2, m = 32 * q + lane;
        const int mbx = m & 7, mby = m >> 3;
        const bool mvalid = mbx < g.nvx && mby < g.nvy;
        uint16_t *mybuf = buf + par * CAP * M;
        // the quarter's blocks need the flat range [flo, fhi)
        int flo = 0, fhi = 0;
        const int by0 = 4 * q, nr = min(4, g.nvy - by0);
        if (nr > 0) {
            flo = (max(block_y(a, g.ky0 + by0) - R, 0) - g.uy0) * g.stride;
            fhi = (min(block_y(a, g.ky0 + by0 + nr - 1) + R, H - 8) - g.uy0 + 1) * g.stride;
        }
        float gm[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) gm[i] = __int_as_float(0x7f800000);
        float T = -__int_as_float(0x7f800000);  // collection threshold (stays -inf for idle lanes)
        int cnt = 0;
        bool have_t = false;
        // pass boundary: the pair (warps q, q + 4) merges its minima and agrees on T
        auto exchange = [&]() {
            if (par == 1) {
#pragma unroll
                for (int i = 0; i < 16; ++i) gmx[m * 17 + i] = gm[i];
            }
            asm volatile("bar.sync %0, 64;\n" ::"r"(1 + q) : "memory");
            if (par == 0) {
#pragma unroll
                for (int i = 0; i < 16; ++i) gm[i] = fminf(gm[i], gmx[m * 17 + i]);
                if (mvalid) T = eighth_smallest(gm) + 2.0f * epsx[m];
                Tx[m] = T;
            }
            asm volatile("bar.sync %0, 64;\n" ::"r"(1 + q) : "memory");
            if (par == 1) T = Tx[m];
            have_t = true;
        };
        const bool dbg = a.tc_dbg != nullptr && blockIdx.x == 0 && blockIdx.y == 0;
        for (int j = par; j < J; j += 2) {
            if (j >= nch && !have_t) exchange();
            const int s = j % NSLOT, base = (j % nch) * N;
            if (!mbar_wait(done0 + 8 * s, (j / NSLOT) & 1, polls)) {
                timeout = 1;
                break;
            }
            fence_after_sync();
            const bool pass2 = j >= nch;
            const int s0 = max(flo - base, 0) >> 5;
            const int s1 = (min(fhi - base, N) + 31) >> 5;
            const uint32_t tl = tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)(s * N);
            for (int sc = s0; sc < s1; ++sc) {
                float v[32];
                __syncwarp();  // tcgen05.ld is warp-collective: reconverge after the collection loop
                const long long t0 = prof ? clock64() : 0;
                tmem_ld32(tl + 32 * sc, v);
                if (prof) {
                    t_ld += clock64() - t0;
                    ++n_ld;
                }
                if (!pass2) {
#pragma unroll
                    for (int r = 0; r < 16; ++r) gm[r] = min3(gm[r], v[r], v[r + 16]);
                    if (dbg) {
                        float *o = a.tc_dbg + (size_t)m * (nch * N) + base + 32 * sc;
#pragma unroll
                        for (int r = 0; r < 32; ++r) o[r] = v[r];
                    }
                } else {
                    unsigned h0 = 0, h1 = 0, h2 = 0, h3 = 0;  // four independent chains
#pragma unroll
                    for (int r = 0; r < 8; ++r) {
                        h0 |= (v[r] <= T ? 1u : 0u) << r;
                        h1 |= (v[r + 8] <= T ? 1u : 0u) << r;
                        h2 |= (v[r + 16] <= T ? 1u : 0u) << r;
                        h3 |= (v[r + 24] <= T ? 1u : 0u) << r;
                    }
                    unsigned hit = h0 | (h1 << 8) | (h2 << 16) | (h3 << 24);
                    while (hit) {
                        const int r = __ffs(hit) - 1;
                        hit &= hit - 1;
                        if (cnt < CAP) mybuf[cnt * M + m] = (uint16_t)(base + 32 * sc + r);
                        ++cnt;
                    }
                }
            }
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(free0 + 8 * s);
        }
        if (!have_t) exchange();  // both warps of a pair pass the boundary exactly once
        cntx[par * M + m] = cnt;
        if (par == 0) okx[m] = T < 0.5f * BIG;  // a bound at penalty level: the window was not covered
    } else if (warp < 12) {
        const int b = tid - 256;
        for (int j = 0; j < J; ++j) {
            const int s = j % NSLOT;
            // slab s was last read by job j - NSLOT
            if (j >= NSLOT && !mbar_wait(done0 + 8 * s, ((j - NSLOT) / NSLOT) & 1, polls)) {
                timeout = 1;
                break;
            }
            const long long t0 = prof ? clock64() : 0;
            build_slab(smem, g, j % nch, s, b);
            if (prof) t_ld += clock64() - t0;
            fence_async_smem();
            __syncwarp();
            if (lane == 0) mbar_arrive(full0 + 8 * s);
        }
    } else if (lane == 0) {
        const uint32_t a_saddr = smem_u32(smem + OFF_A), b_saddr = smem_u32(smem + OFF_B);
        for (int j = 0; j < J; ++j) {
            const int s = j % NSLOT;
            if (!mbar_wait(full0 + 8 * s, (j / NSLOT) & 1, polls) ||
                (j >= NSLOT && !mbar_wait(free0 + 8 * s, ((j - NSLOT) / NSLOT) & 1, polls))) {
                timeout = 1;
                break;
            }
            fence_after_sync();
            const uint32_t d = tbase + (uint32_t)(s * N), bsa = b_saddr + s * SZ_B;
#pragma unroll
            for (int kk = 0; kk < KSTEPS; ++kk)
                mma_f16(d, make_desc(a_saddr + kstep_off(kk)), make_desc(bsa + kstep_off(kk)), kk);
            mma_commit(done0 + 8 * s);
            last = j;
        }
    }
    const int stop = __syncthreads_or(timeout);
    if (prof) {
        const unsigned wp = __reduce_add_sync(0xffffffffu, polls);
        if (lane == 0) {
            atomicAdd(prof + (warp < 8 ? 8 : warp < 12 ? 9 : 10), (unsigned long long)wp);
            if (warp < 12) atomicAdd(prof + (warp < 8 ? 11 : 12), (unsigned long long)t_ld);
            if (warp < 8) atomicAdd(prof + 13, (unsigned long long)n_ld);
        }
    }
    // ---- drain and release tensor memory -------------------------------------------
    if (stop && warp == 12 && lane == 0 && last >= 0)
        mbar_wait(done0 + 8 * (last % NSLOT), (last / NSLOT) & 1, polls);
    if (stop && tid == 0) a.tc_ws[1] = 1;
    fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        fence_after_sync();
        tmem_dealloc(tbase, 512);
    }

    // ---- exact re-rank of the collected candidates from the FP32 region ------------
    // Three threads per block compute the exact errors of its collected candidates
    // (entries k = grp, grp + 3, ... of [even-job list, odd-job list]); then the
    // block's thread merges both lists in flat order (= the reference's scan order)
    // into the reference's insertion rule.
    stage_region(reg, plane, P, g, tid);
    __syncthreads();
    if (prof && tid == 0) prof[5] = clock64();
    float *errs = reg + REG_ROWS * REG_COLS;  // [2][CAP][128], after the region in the slab area
    const bool bad_tile = stop || *oor;
    const unsigned long long inv = (0x100000000ull + g.stride - 1) / g.stride;
    if (tid < 3 * M && !bad_tile) {
        const int m = tid & 127, grp = tid >> 7;
        const int mbx = m & 7, mby = m >> 3;
        const int c0n = cntx[m], c1n = cntx[M + m];
        if (mbx < g.nvx && mby < g.nvy && okx[m] && c0n <= CAP && c1n <= CAP) {
            const int moff = (block_y(a, g.ky0 + mby) - g.uy0) * REG_COLS + (block_x(a, g.kx0 + mbx) - g.ux0);
            float2 nc[8][4];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int p = 0; p < 4; ++p)
                    nc[i][p] = make_float2(-reg[moff + i * REG_COLS + 2 * p], -reg[moff + i * REG_COLS + 2 * p + 1]);
            for (int k = grp; k < c0n + c1n; k += 3) {
                const int p = k < c0n ? 0 : 1, idx = (p * CAP + (p ? k - c0n : k)) * M + m;
                const unsigned f = buf[idx];
                const int r = div_small(f, inv), cc = (int)f - r * g.stride;
                // penalised positions are never collected; keep the guard for the index arithmetic
                errs[idx] = (r < g.nur && cc < g.nuc) ? exact_ssd2(nc, reg + r * REG_COLS + cc, REG_COLS) : ZB_FLT_MAX;
            }
        }
    }
    __syncthreads();
    if (prof && tid == 0) prof[6] = clock64();
    if (tid >= M) return;
    const int c0n = cntx[tid], c1n = cntx[M + tid];
    const bool fb = valid && (bad_tile || !okx[tid] || c0n > CAP || c1n > CAP);
    if (valid) {
        const int bi = (g.ky0 + byl) * a.nbx + (g.kx0 + bxl);
        if (fb) {
            list_fallback(a, bi);
        } else {
            float e[8];
            int q[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                e[i] = ZB_FLT_MAX;
                q[i] = 0;
            }
            int i0 = 0, i1 = 0;
            while (i0 < c0n || i1 < c1n) {
                const unsigned f0 = i0 < c0n ? buf[i0 * M + tid] : 0xffffffffu;
                const unsigned f1 = i1 < c1n ? buf[(CAP + i1) * M + tid] : 0xffffffffu;
                const bool take0 = f0 < f1;  // a flat index belongs to one chunk, so to one list
                const unsigned f = take0 ? f0 : f1;
                const float err = take0 ? errs[i0 * M + tid] : errs[(CAP + i1) * M + tid];
                i0 += take0;
                i1 += !take0;
                const int r = div_small(f, inv), cc = (int)f - r * g.stride;
                if (err < e[7]) top8_insert(e, q, err, pack_pos(g.ux0 + cc, g.uy0 + r));
            }
            store_list(a, bi, xb, yb, e, q);
        }
    }
    if (prof && tid == 0) prof[7] = clock64();
    if (a.tc_stats) {
        const unsigned nval = __popc(__ballot_sync(0xffffffffu, valid));
        const unsigned nfb = __popc(__ballot_sync(0xffffffffu, fb));
        const unsigned ns = __reduce_add_sync(0xffffffffu, valid && !fb ? (unsigned)(c0n + c1n) : 0u);
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
