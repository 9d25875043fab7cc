// Block matching on the 5th-generation tensor cores (tcgen05), SSD, spatial search.
//
// The plain matcher evaluates every candidate's SSD in the reference's FP32
// operation order (vszipcu src/bm3d.cu:282-302, 614-660).  This form gets the
// same lists with the distances bounded on the tensor cores:
//
//  1. A tile is 8 x 16 reference blocks (M = 128 rows of the MMA, TMEM lane m =
//     block m).  The candidate positions of the union of their search windows,
//     nur rows x nuc columns (nuc <= 56), are numbered row-major at a fixed row
//     pitch of 56: flat f = r * 56 + c.  They stream through tcgen05.mma
//     (kind::f16, FP32 accumulation in tensor memory) in chunks of N = 224
//     consecutive f, i.e. 4 whole rows.  Row m of the product is, for block m and
//     a candidate f inside block m's columns,
//         d(m, f) = |b_f - c0|^2 - 2 (mu_m - c0) S_f - 2 (a_m - mu_m) . (b_f - c0)
//     (c0 a tile constant, mu_m the block mean, S_f the candidate sum), which
//     equals SSD(a_m, b_f) - |a_m - c0|^2.  The pixel cross term runs on FP16
//     operands; the norm terms enter as FP16 hi/lo pairs in a fifth K step, whose
//     second half adds 16384 where the candidate's column lies outside block m's
//     window (a one-hot of the block column in A against a per-column penalty row
//     in B; the penalty rows repeat every 56 candidates, so one 224-row table
//     serves every chunk).
//  2. Operand B needs no per-chunk build: the tile's region is expanded once into
//     E[y][x] = the 8 FP16 pixels (y, x .. x + 7) - c0, 16 bytes per position, at
//     the row pitch of 56 positions.  Patch row i of candidate f is then E entry
//     f + 56 i, so one shared-memory descriptor (8-row core matrices 128 bytes
//     apart, K chunks one E row apart) walks 224 consecutive candidates and the
//     8 patch rows.  The norm terms sit in a per-candidate table read the same way.
//     A 32-column group of a chunk spans at most two rows, so the window's rows
//     are two compares per block and group.
//  3. Pass 1 keeps, per block, the minimum of d over 16 groups of its window
//     candidates by flat index mod 16, and over 16 groups by union row mod 16 (good
//     matches along a vertical edge share few column residues but many rows).  The
//     smaller of the two eighth smallest group minima, U, comes from eight distinct
//     window candidates, so the reference's eighth-best FP32 error is at most
//     U + |a - c0|^2 + eps, where eps bounds |d - (SSD_ref - |a - c0|^2)|.  Pass 2 recomputes the chunks and collects
//     every window candidate with d <= U + 2 eps: a superset of the exact top 8,
//     ties included.
//  4. The collected candidates get the exact FP32 SSD in the reference's order
//     and the eight smallest by (error, scan position) are kept, which is the list
//     the reference's strict-less insertion builds in scan order; then self
//     inclusion.  The list is bit-identical to the plain matcher's.
//
// A block whose collection overflows, or a tile whose pixels leave the range the
// FP16 terms are sized for (|x| <= 4), is listed for the exact matcher
// (zb_match_global, gen_mode 2), so the result never depends on the bound being
// tight.
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
constexpr int WX = 56;                       // flat row pitch: candidate columns per union row (nuc <= WX)
constexpr int ROWS_PER_CHUNK = 4;
constexpr int N = ROWS_PER_CHUNK * WX;       // candidates per MMA chunk = TMEM columns of one slot (224)
constexpr int KSTEPS = 5;                    // patch rows (0,1) (2,3) (4,5) (6,7), then norms + column penalties
constexpr int MAX_UC = WX, MAX_UR = 88;      // candidate union of a tile: columns, rows
constexpr int REG_ROWS = MAX_UR + 7;
constexpr int REG_COLS = 64;                 // staged FP32 region: columns (union + 7, padded)
constexpr int E_ROWS = MAX_UR + ROWS_PER_CHUNK - 1 + 7;  // candidate rows of the last chunk + 7 patch rows
constexpr int T_ROWS = MAX_UR + ROWS_PER_CHUNK - 1;
constexpr int NLIST = 4;                     // block warps per lane quarter: job parity (x chunk row half
                                             // when 4); each keeps its own collection list
constexpr int CAP = NLIST == 4 ? 16 : 32;    // collected candidates per block and list
constexpr int MMA_WARP = 4 * NLIST;          // TMEM owner and MMA issuer (lane 0); the warps above it help
                                             // in setup and the re-rank
constexpr int THREADS = NLIST == 4 ? 544 : 384;
constexpr int NWARPS = THREADS / 32;
constexpr float BIG = 16384.0f;              // column-window penalty (exact in FP16)
constexpr float RANGE = 4.0f;                // pixel magnitude the FP16 terms are sized for
constexpr unsigned WAIT_LIMIT = 1u << 16;    // suspended waits on an mbarrier before giving up

// shared memory plan (bytes)
constexpr int OFF_E = 0;                                     // expanded region, FP16 x 8 per position
constexpr int SZ_E = E_ROWS * WX * 16;
constexpr int OFF_T = OFF_E + SZ_E;                          // per candidate: S hi, S lo, S hi, p hi, p lo, 0, 0, 0
constexpr int SZ_T = T_ROWS * WX * 16;
constexpr int OFF_XP = OFF_T + SZ_T;                         // per chunk column: 8 block-column penalties (FP16)
constexpr int SZ_XP = N * 16;
constexpr int OFF_A = OFF_XP + SZ_XP;                        // operand A: 10 K chunks x 128 rows x 16 bytes
constexpr int A_KCHUNK = M * 16;
constexpr int SZ_A = 10 * A_KCHUNK;
constexpr int OFF_BUF = OFF_A + SZ_A;                        // setup: FP32 region; stream: lists + group minima
constexpr int SZ_REG = REG_ROWS * REG_COLS * 4;
constexpr int SZ_LIST = NLIST * CAP * M * 2;                 // [4][CAP][128] flat indices (16 bits)
constexpr int OFF_GMX = OFF_BUF + SZ_LIST;                   // [16][128] group minima (order-preserving keys)
constexpr int SZ_BUF = SZ_REG > SZ_LIST + 16 * M * 4 ? SZ_REG : SZ_LIST + 16 * M * 4;
constexpr int OFF_GMR = OFF_BUF + SZ_BUF;                    // [16][128] minima per union row mod 16 (pass 1)
constexpr int OFF_EPS = OFF_GMR + 16 * M * 4;                // [128] 2 eps
constexpr int OFF_TX = OFF_EPS + M * 4;                      // [128] collection bound U + 2 eps
constexpr int OFF_CNT = OFF_TX + M * 4;                      // [4][128] collection counts
constexpr int OFF_ROWMAX = OFF_CNT + NLIST * M * 4;          // [MAX_UR] max |b - c0|^2 per union row
constexpr int OFF_MISC = OFF_ROWMAX + MAX_UR * 4;            // mbarriers, TMEM address, flags, reductions
constexpr int SMEM_BYTES = OFF_MISC + 96;
static_assert(SMEM_BYTES <= 227 * 1024, "tensor-core matcher exceeds shared memory");
static_assert(OFF_T % 16 == 0 && OFF_XP % 16 == 0 && OFF_A % 128 == 0 && OFF_BUF % 16 == 0 && OFF_MISC % 16 == 0,
              "shared-memory regions must stay aligned");
static_assert(N % 16 == 0 && N <= 256 && 2 * N <= 512 && N % 32 == 0, "chunk shape");
// during setup the E area holds the horizontal sums; during the re-rank the FP32 region
// (E area) and the exact errors (T area)
static_assert(2 * REG_ROWS * MAX_UC * 4 <= SZ_E && SZ_REG <= SZ_E && NLIST * CAP * M * 4 <= SZ_T, "scratch reuse");
static_assert(N == 4 * 56, "the row-half load table below assumes 4 rows of 56 candidates per chunk");

// Shared-memory matrix descriptor, K-major without swizzle (layout type 0): start
// address, LBO (distance of K-adjacent core matrices) and SBO (distance of 8-row
// groups) in 16-byte units, version 1 at bits 46-47 as tcgen05 requires.
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP16 A and B (both the same type), FP32
// accumulator, both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28.
constexpr uint32_t IDESC = (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);

// Waits for phase `parity` of an mbarrier: try_wait suspends the thread until the
// phase completes or a hardware time limit passes, so waiting warps take no issue
// slots from the working ones.  At most WAIT_LIMIT such waits; false on timeout.
// `polls` counts the waits that ran out.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, unsigned &polls) {
    for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try(mbar, parity)) {
            polls += i;
            return true;
        }
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
// The candidate union is [ux0, ux0 + nuc) x [uy0, uy0 + nur), flat f = r * 56 + c;
// chunk k is the flat range [224 k, 224 k + 224), union rows 4 k .. 4 k + 3.
// ---------------------------------------------------------------------------
struct Geom {
    int kx0, ky0, nvx, nvy;
    int ux0, uy0, nuc, nur, flat, nch;
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
    g.flat = g.nur * WX;
    g.nch = (g.nur + ROWS_PER_CHUNK - 1) / ROWS_PER_CHUNK;
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

// The same exact SSD with the reference patch c read from shared memory as well:
// n + (-c) is computed as -(c - n) exactly, so the value is the one above.
__device__ __forceinline__ float exact_ssd2_s(const float *c, const float *n, int pitch) {
    float s[8];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        float2 d[8];
#pragma unroll
        for (int i = 0; i < 8; ++i)
            d[i] = __fadd2_rn(make_float2(n[i * pitch + 2 * p], n[i * pitch + 2 * p + 1]),
                              make_float2(-c[i * pitch + 2 * p], -c[i * pitch + 2 * p + 1]));
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

// minimum of three (two two-operand minima: the three-operand PTX form costs more)
__device__ __forceinline__ float min3(float a, float b, float c) { return fminf(fminf(a, b), c); }

// minimum of 32 values, depth 4
__device__ __forceinline__ float min32(const float (&v)[32]) {
    float a[11];
#pragma unroll
    for (int k = 0; k < 10; ++k) a[k] = min3(v[3 * k], v[3 * k + 1], v[3 * k + 2]);
    a[10] = fminf(v[30], v[31]);
    const float b0 = min3(a[0], a[1], a[2]), b1 = min3(a[3], a[4], a[5]), b2 = min3(a[6], a[7], a[8]);
    return fminf(min3(b0, b1, b2), fminf(a[9], a[10]));
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

// Bits [0, b) set (b in 0..32).
__device__ __forceinline__ uint32_t low_bits(int b) { return b >= 32 ? 0xffffffffu : ((1u << b) - 1u); }

// Order-preserving integer key of a float (no NaN): a < b  <=>  key(a) < key(b), so that
// shared-memory atomicMin can merge minima of any sign.
__device__ __forceinline__ int fkey(float f) {
    const int k = __float_as_int(f);
    return k >= 0 ? k : k ^ 0x7fffffff;
}
__device__ __forceinline__ float fkey_inv(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7fffffff); }

// The TMEM loads of one chunk row half (chunk columns, width 32 or 16): rows 0-1 are
// columns 0-111, rows 2-3 columns 112-223.  Half 0 loads columns 0, 32, 64 and 96 (16
// wide), half 1 columns 112 (16 wide), 128, 160 and 192; a load's bits below bnd lie in
// its first row, the rest in the next one (bnd = 24 at column 32, 8 at column 160).

// (error, scan position) order: the reference's strict-less insertion over a
// row-major scan keeps, among equal errors, the one scanned first
__device__ __forceinline__ bool lex_less(float e1, int p1, float e2, int p2) { return e1 < e2 || (e1 == e2 && p1 < p2); }

__device__ __forceinline__ void top8_insert_lex(float (&e)[8], int (&q)[8], float err, int pos) {
#pragma unroll
    for (int i = 7; i > 0; --i) {
        const bool ci = lex_less(err, pos, e[i], q[i]);
        const bool cp = lex_less(err, pos, e[i - 1], q[i - 1]);
        e[i] = cp ? e[i - 1] : (ci ? err : e[i]);
        q[i] = cp ? q[i - 1] : (ci ? pos : q[i]);
    }
    if (lex_less(err, pos, e[0], q[0])) {
        e[0] = err;
        q[0] = pos;
    }
}

// Self-check of an index, address or descriptor range before it is used.  A failed
// check skips the access, records the first failure of the launch in tc_ws[2]
// (code) and tc_ws[3..6] (values, tile), and marks the tile (*tile_bad) so that all
// its blocks go to the exact matcher.
__device__ __forceinline__ bool guard(const MatchArgs &a, int *tile_bad, bool ok, int code, int v0, int v1, int v2) {
    if (!ok) {
        if (atomicCAS(a.tc_ws + 2, 0, code) == 0) {
            a.tc_ws[3] = v0;
            a.tc_ws[4] = v1;
            a.tc_ws[5] = v2;
            a.tc_ws[6] = (int)(blockIdx.y * 65536 + blockIdx.x);
        }
        *tile_bad = 1;
    }
    return ok;
}

__device__ __forceinline__ void list_fallback(const MatchArgs &a, int bi) {
    const int k = atomicAdd(a.tc_ws, 1);
    if (k < a.nbx * a.nby) a.tc_ws[kTcWsList + k] = bi;
}

// Asynchronous copy of the tile's FP32 region (union rows + 7, columns + 7) into
// shared memory, at pitch REG_COLS; columns beyond it are zero-filled.  `cap` is
// the floats the destination area holds.
__device__ __forceinline__ void stage_region(float *reg, int cap, const float *plane, int P, const Geom &g, int tid,
                                             const MatchArgs &a, int *tile_bad) {
    const int rr = g.nur + 7, rc = g.nuc + 7;
    for (int i = tid; i < rr * REG_COLS; i += THREADS) {
        const int row = i >> 6, col = i & 63;
        const bool ok = col < rc;
        if (!guard(a, tile_bad, i < cap && g.uy0 >= 0 && g.uy0 + row < a.h && g.ux0 >= 0 && g.ux0 + (ok ? col : 0) < a.w,
                   10, g.uy0 + row, g.ux0 + col, i))
            continue;
        const float *src = plane + (long long)(g.uy0 + row) * P + g.ux0 + (ok ? col : 0);
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(smem_u32(reg + i)), "l"(src),
                     "r"(ok ? 4 : 0)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// One CTA per tile of 8 x 16 reference blocks.  The block warps (4 NLIST) own the
// blocks: warp w reads TMEM lanes 32 (w mod 4) .. + 31 (block m = lane index), for the
// jobs of parity (w / 4) mod 2, which use TMEM slot (w / 4) mod 2 (columns
// [224 s, 224 s + 224)); with NLIST = 4 each takes one half of the chunk's rows.  Lane 0
// of warp MMA_WARP issues the MMAs.  The roles meet at mbarriers: done[s] (MMAs of the
// job complete, tcgen05.commit) and free[s] (the slot read by the block warps of its
// parity); job j waits for phase (j / 2) mod 2.
__global__ void __launch_bounds__(THREADS, 1) zb_match_tc(MatchArgs a) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const Geom g = tile_geom(a);
    const int H = a.h, W = a.w, R = a.range, P = a.pitch;
    const int nuc = g.nuc;
    const float *plane = a.frames + (long long)a.radius * a.fstride;

    uint64_t *mbar = reinterpret_cast<uint64_t *>(smem + OFF_MISC);  // done[2], free[2]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(smem + OFF_MISC + 32);
    int *oor = reinterpret_cast<int *>(smem + OFF_MISC + 36);
    int *tmax = reinterpret_cast<int *>(smem + OFF_MISC + 40);        // max |S|, bits of a non-negative float
    int *tile_bad = reinterpret_cast<int *>(smem + OFF_MISC + 44);    // a self-check failed in this tile
    float *red = reinterpret_cast<float *>(smem + OFF_MISC + 48);     // [0..3] mean sums, [4..7] counts
    float *rowmax = reinterpret_cast<float *>(smem + OFF_ROWMAX);
    float *reg = reinterpret_cast<float *>(smem + OFF_BUF);           // setup: FP32 region
    float *hs = reinterpret_cast<float *>(smem + OFF_E);              // setup: horizontal sums
    float *hp = hs + REG_ROWS * MAX_UC;
    uint16_t *lists = reinterpret_cast<uint16_t *>(smem + OFF_BUF);   // [2][CAP][128]
    float *gmx = reinterpret_cast<float *>(smem + OFF_GMX);           // [16][128]
    float *gmr = reinterpret_cast<float *>(smem + OFF_GMR);           // [16][128]
    float *eps2x = reinterpret_cast<float *>(smem + OFF_EPS);
    float *tx = reinterpret_cast<float *>(smem + OFF_TX);
    int *cntx = reinterpret_cast<int *>(smem + OFF_CNT);
    const uint32_t mb = smem_u32(mbar);
    const uint32_t done0 = mb, free0 = mb + 16;  // slot s at +8 s

    unsigned long long *prof = a.tc_prof ? a.tc_prof + 16 * (blockIdx.y * gridDim.x + blockIdx.x) : nullptr;
    // tile (1, 1) also traces every job after the per-tile blocks: [j][0] issued (MMA thread,
    // after its commit), [j][1] completion seen and [j][2] slot freed (warp 0 or 4, lane 0)
    unsigned long long *trace = (a.tc_prof && blockIdx.x == 1 && blockIdx.y == 1)
                                    ? a.tc_prof + 16 * (gridDim.x * gridDim.y) : nullptr;
    unsigned polls = 0;
    if (prof && tid == 0) prof[0] = clock64();
    if (warp == MMA_WARP) {
        __syncwarp();  // tcgen05.alloc is .sync.aligned
        tmem_alloc(smem_u32(tslot), 512);
    }
    if (tid == 0) {
        for (int k = 0; k < 2; ++k) {
            mbar_init(done0 + 8 * k, 1);
            mbar_init(free0 + 8 * k, 2 * NLIST);  // the block warps of the slot's job parity
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        *oor = 0;
        *tmax = 0;
        *tile_bad = 0;
    }
    __syncthreads();
    stage_region(reg, SZ_BUF / 4, plane, P, g, tid, a, tile_bad);
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *tslot;
    if (tid == 0) guard(a, tile_bad, tbase == 0u, 1, (int)tbase, 0, 0);  // all 512 columns: lane 0, column 0
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

    // ---- range check, horizontal 8-sums of (x - c0) and (x - c0)^2 ---------------
    const int rr = g.nur + 7, rc = nuc + 7;
    bool bad = false;
    for (int row = warp; row < rr; row += NWARPS) {
        const float *rp = reg + row * REG_COLS;
        const float x0 = rp[lane], x1 = rp[lane + 32];
        bad |= (lane < rc && !(fabsf(x0) <= RANGE)) || (lane + 32 < rc && !(fabsf(x1) <= RANGE));
        for (int cc = lane; cc < nuc; cc += 32) {
            float s = 0.0f, q = 0.0f;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const float d = rp[cc + j] - c0;
                s += d;
                q = fmaf(d, d, q);
            }
            if (guard(a, tile_bad, row * MAX_UC + cc < REG_ROWS * MAX_UC, 20, row, cc, 0)) {
                hs[row * MAX_UC + cc] = s;
                hp[row * MAX_UC + cc] = q;
            }
        }
    }
    if (bad) *oor = 1;
    __syncthreads();
    if (prof && tid == 0) prof[2] = clock64();

    // ---- norm table: per candidate S and p as FP16 hi/lo, row maxima of p ------
    // rows up to the last chunk's; columns nuc .. 55 and rows nur .. zero (never in a window)
    uint4 *tt = reinterpret_cast<uint4 *>(smem + OFF_T);
    const int trows = g.nch * ROWS_PER_CHUNK;
    float smax = 0.0f;
    for (int r = warp; r < trows; r += NWARPS) {
        float mx = 0.0f;
        for (int c = lane; c < WX; c += 32) {
            uint4 e = make_uint4(0, 0, 0, 0);
            if (r < g.nur && c < nuc) {
                float s = 0.0f, q = 0.0f;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    s += hs[(r + k) * MAX_UC + c];
                    q += hp[(r + k) * MAX_UC + c];
                }
                __half sh, sl, ph, pl;
                split_h(s, sh, sl);
                split_h(q, ph, pl);
                e = make_uint4(h2u(sh, sl), h2u(sh, ph), h2u(pl, __float2half_rn(0.0f)), 0u);
                smax = fmaxf(smax, fabsf(s));
                mx = fmaxf(mx, q);
            }
            if (guard(a, tile_bad, r < T_ROWS, 21, r, c, 0)) tt[r * WX + c] = e;
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        if (lane == 0 && r < g.nur) rowmax[r] = mx;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) smax = fmaxf(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    if (lane == 0) atomicMax(tmax, __float_as_int(smax));
    // column penalties: chunk column n is union column n mod 56; block column j's window
    // is [x_j - R, x_j + R]; columns at or beyond nuc are not candidates
    {
        const __half hbig = __float2half_rn(BIG), hzero = __float2half_rn(0.0f);
        uint4 *xp = reinterpret_cast<uint4 *>(smem + OFF_XP);
        for (int n = tid; n < N; n += THREADS) {
            const int c = n % WX;
            __half pnl[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const bool out = c >= nuc || (j < g.nvx && abs(g.ux0 + c - block_x(a, g.kx0 + j)) > R);
                pnl[j] = out ? hbig : hzero;
            }
            xp[n] = make_uint4(h2u(pnl[0], pnl[1]), h2u(pnl[2], pnl[3]), h2u(pnl[4], pnl[5]), h2u(pnl[6], pnl[7]));
        }
    }
    __syncthreads();  // the horizontal sums are dead from here on

    // ---- expanded region: E[y][x] = FP16 (x + j, j < 8) - c0 of region row y -----
    // rows beyond the region (read only by the last chunk's padding rows) are zero
    uint4 *ee = reinterpret_cast<uint4 *>(smem + OFF_E);
    const int erows = trows + 7;
    for (int i = tid; i < erows * WX; i += THREADS) {
        const int y = i / WX, x = i - y * WX;
        uint4 e = make_uint4(0, 0, 0, 0);
        if (y < rr) {
            const float *rp = reg + y * REG_COLS + x;
            __half h[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) h[j] = __float2half_rn(rp[j] - c0);
            e = make_uint4(h2u(h[0], h[1]), h2u(h[2], h[3]), h2u(h[4], h[5]), h2u(h[6], h[7]));
        }
        if (guard(a, tile_bad, y < E_ROWS && x + 7 < REG_COLS, 22, i, y, x)) ee[i] = e;
    }
    if (prof && tid == 0) prof[3] = clock64();

    // ---- operand A (one row per block) and the block's error bound ------------
    if (tid < M) {
        uint4 pa[10];
        float eps = 0.0f;
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
            const __half m2h = __float2half_rn(-2.0f * __half2float(nh));
            const __half m2l = __float2half_rn(-2.0f * __half2float(nl));
            const __half one = __float2half_rn(1.0f), zero = __float2half_rn(0.0f);
            // [S hi, S lo, S hi, p hi, p lo] . [-2 nh, -2 nh, -2 nl, 1, 1], then the block
            // column's one-hot against the column penalties
            pa[8] = make_uint4(h2u(m2h, m2h), h2u(m2l, one), h2u(one, zero), 0u);
            __half oh[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) oh[j] = j == bxl ? one : zero;
            pa[9] = make_uint4(h2u(oh[0], oh[1]), h2u(oh[2], oh[3]), h2u(oh[4], oh[5]), h2u(oh[6], oh[7]));
            // eps bounds |d - (SSD_ref - |a - c0|^2)| over the block's window:
            // FP16 rounding of both cross-term operands (2^-11 each, x2 for the factor 2),
            // FP32 accumulation and the hi/lo splits (2^-15 of the term sizes)
            const int r0 = max(yb - R, 0) - g.uy0, r1 = min(yb + R, H - 8) - g.uy0;
            float pm = 0.0f;
            for (int r = r0; r <= r1; ++r) pm = fmaxf(pm, rowmax[r]);
            const float an = sqrtf(an2), bm = sqrtf(pm);
            const float sm = __int_as_float(*tmax);
            eps = 1.01f * 0.001953125f * an * bm +
                  3.0517578125e-05f * (2.0f * an * bm + 2.0f * fabsf(nu) * sm + pm + ah2 + 1.0f);
        } else {
#pragma unroll
            for (int k = 0; k < 10; ++k) pa[k] = make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int kc = 0; kc < 10; ++kc)
            *reinterpret_cast<uint4 *>(smem + OFF_A + kc * A_KCHUNK + (tid >> 3) * 128 + (tid & 7) * 16) = pa[kc];
        eps2x[tid] = 2.0f * eps;
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            gmr[i * M + tid] = __int_as_float(0x7f800000);
            reinterpret_cast<int *>(gmx)[i * M + tid] = fkey(__int_as_float(0x7f800000));
        }
    }
    fence_async_smem();
    fence_before_sync();
    __syncthreads();  // the FP32 region in the list area is dead from here on
    fence_after_sync();
    const bool bad_tile = *oor != 0 || *tile_bad != 0;
    if (prof && tid == 0) prof[4] = clock64();

    // ---- the MMA stream ------------------------------------------------------------
    // jobs j = 0 .. 2 nch - 1 are (pass j / nch, chunk j mod nch) on TMEM slot j mod 2
    const int nch = g.nch, J = 2 * nch;
    int timeout = 0, last = -1;
    long long t_ld = 0, t_p1 = 0, t_p2 = 0, t_wait = 0;  // profiling: cycles in TMEM loads, passes, waits
    int n_ld = 0;
    if (bad_tile) {
        // pixels beyond the FP16 sizing: every block of the tile goes to the FP32 scan
    } else if (warp < MMA_WARP) {
        const int q = warp & 3, par = (warp >> 2) & 1, m = 32 * q + lane;
        const int half0 = NLIST == 4 ? warp >> 3 : 0, nhalf = NLIST == 4 ? 1 : 2;  // chunk row halves
        const int lid = NLIST == 4 ? 2 * par + half0 : par;  // this warp's collection list
        const int mbx = m & 7, mby = m >> 3;
        const bool mvalid = mbx < g.nvx && mby < g.nvy;
        uint16_t *mylist = lists + lid * CAP * M;
        int *gmk = reinterpret_cast<int *>(gmx);
        // the quarter's blocks need union rows [qr0, qr1]
        int qr0 = 1, qr1 = 0;
        const int by0 = 4 * q, nr = min(4, g.nvy - by0);
        if (nr > 0) {
            qr0 = max(block_y(a, g.ky0 + by0) - R, 0) - g.uy0;
            qr1 = min(block_y(a, g.ky0 + by0 + nr - 1) + R, H - 8) - g.uy0;
        }
        // the block's window rows (empty for idle lanes); its columns are handled by the
        // penalties inside the product
        const int my = block_y(a, g.ky0 + mby);
        const int wr0 = mvalid ? max(my - R, 0) - g.uy0 : 1, wr1 = mvalid ? min(my + R, H - 8) - g.uy0 : 0;
        float gm[16];
#pragma unroll
        for (int i = 0; i < 16; ++i) gm[i] = __int_as_float(0x7f800000);
        float T = -__int_as_float(0x7f800000);  // collection bound (stays -inf for idle lanes)
        int cnt = 0;
        bool have_t = false;
        // pass boundary: the quarter's four warps merge their minima and agree on T
        auto exchange = [&]() {
#pragma unroll
            for (int i = 0; i < 16; ++i) atomicMin(gmk + i * M + m, fkey(gm[i]));
            __syncwarp();
            asm volatile("barrier.sync %0, %1;\n" ::"r"(1 + q), "r"(32 * NLIST) : "memory");
            if (lid == 0) {
                float ge[16], rw[16];
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    ge[i] = fkey_inv(gmk[i * M + m]);
                    rw[i] = gmr[i * M + m];
                }
                if (mvalid) T = fminf(eighth_smallest(ge), eighth_smallest(rw)) + eps2x[m];
                tx[m] = T;
            }
            __syncwarp();
            asm volatile("barrier.sync %0, %1;\n" ::"r"(1 + q), "r"(32 * NLIST) : "memory");
            if (lid != 0) T = tx[m];
            have_t = true;
        };
        const bool dbg = a.tc_dbg != nullptr && blockIdx.x == 0 && blockIdx.y == 0;
        const int s = par;
        for (int j = par; j < J; j += 2) {
            const bool pass2 = j >= nch;
            if (pass2 && !have_t) exchange();
            const long long tw0 = prof ? clock64() : 0;
            if (!mbar_wait(done0 + 8 * s, (j >> 1) & 1, polls)) {
                timeout = 1;
                break;
            }
            if (prof) t_wait += clock64() - tw0;
            fence_after_sync();
            if (trace && q == 0 && lid == 0 && lane == 0) trace[3 * j + 1] = clock64();
            const int ck = pass2 ? j - nch : j;
            const int row0 = ROWS_PER_CHUNK * ck;
            const uint32_t tl = tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)(s * N);
            for (int li = 0; li < 4 * nhalf; ++li) {
                // load li of this warp's row halves: chunk columns col .. col + 31 (or + 15),
                // union rows ra (bits below bnd) and rb
                const int half = half0 + (li >> 2), l = li & 3;
                // half 0: columns 0, 32, 64, 96 (16 wide); half 1: 112 (16 wide), 128, 160, 192
                const int col = half == 0 ? 32 * l : (l == 0 ? 112 : 96 + 32 * l);
                const bool narrow = col == 96 || col == 112;
                const int ra = row0 + col / WX;
                const int bnd = col + 32 > (ra - row0 + 1) * WX && !narrow ? (ra - row0 + 1) * WX - col : 32;
                const int rb = bnd < 32 ? ra + 1 : ra;
                if (rb < qr0 || ra > qr1) continue;  // no block of this quarter looks at these rows
                float v[32];
                __syncwarp();  // tcgen05.ld is warp-collective: reconverge after the collection code
                if (!guard(a, tile_bad,
                           (tl >> 16) == (uint32_t)(32 * q) && (tl & 0xffffu) + (uint32_t)col + (narrow ? 16u : 32u) <= 512u,
                           40, col, (int)tl, j)) {
                    timeout = 1;
                    break;
                }
                const long long t0 = prof ? clock64() : 0;
                if (narrow) {
                    tmem_ld16(tl + col, v);
#pragma unroll
                    for (int r = 16; r < 32; ++r) v[r] = __int_as_float(0x7f800000);
                } else {
                    tmem_ld32(tl + col, v);
                }
                if (prof) {
                    t_ld += clock64() - t0;
                    ++n_ld;
                }
                const long long tp0 = prof ? clock64() : 0;
                const int g0 = ck * N + col;
                const bool ina = ra >= wr0 && ra <= wr1, inb = rb >= wr0 && rb <= wr1;
                // the row boundary is a multiple of 8, so the window's rows select whole
                // 8-element blocks: bit k of bsel = block k is in the window's rows
                const int nba = bnd >> 3;  // blocks in row ra
                const uint32_t bsel = ((ina ? (1u << nba) - 1u : 0u) | (inb ? (0xfu & ~((1u << nba) - 1u)) : 0u)) &
                                      (narrow ? 0x3u : 0xfu);
                if (!bsel) {
                    // no window row of this block
                } else {
                    float b8[4];
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        b8[k] = min3(min3(v[8 * k], v[8 * k + 1], v[8 * k + 2]),
                                     min3(v[8 * k + 3], v[8 * k + 4], v[8 * k + 5]), fminf(v[8 * k + 6], v[8 * k + 7]));
                    const float inf = __int_as_float(0x7f800000);
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (!((bsel >> k) & 1u)) b8[k] = inf;
                    if (!pass2) {
                        if (dbg && guard(a, tile_bad, g0 + (narrow ? 15 : 31) < nch * N, 41, g0, m, nch)) {
                            float *o = a.tc_dbg + (size_t)m * (nch * N) + g0;
#pragma unroll
                            for (int r = 0; r < 32; ++r)
                                if (r < 16 || !narrow) o[r] = v[r];
                        }
                        // group minima over the block's window rows (out-of-window columns carry
                        // the penalty): by flat index mod 16 (col is a multiple of 16), and by
                        // union row mod 16 (this warp's chunks own row residues 4 (k mod 4) + its
                        // row halves, so no two warps of a quarter write the same slot)
                        if (bsel != (narrow ? 0x3u : 0xfu)) {
#pragma unroll
                            for (int r = 0; r < 32; ++r)
                                if (!((bsel >> (r >> 3)) & 1u)) v[r] = inf;
                        }
#pragma unroll
                        for (int r = 0; r < 16; ++r) gm[r] = min3(gm[r], v[r], v[r + 16]);
                        const float sa = nba == 1 ? b8[0] : nba == 3 ? min3(b8[0], b8[1], b8[2])
                                                                      : fminf(fminf(b8[0], b8[1]), fminf(b8[2], b8[3]));
                        float *ga = gmr + (ra & 15) * M + m;
                        *ga = fminf(*ga, sa);
                        if (rb > ra) {
                            const float sb = nba == 1 ? min3(b8[1], b8[2], b8[3]) : b8[3];
                            float *gb = gmr + (rb & 15) * M + m;
                            *gb = fminf(*gb, sb);
                        }
                    } else if (fminf(fminf(b8[0], b8[1]), fminf(b8[2], b8[3])) <= T) {
                        // collect the window candidates at or below T, block by block
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            if (!(b8[k] <= T)) continue;
                            uint32_t hit = 0;
#pragma unroll
                            for (int r = 0; r < 8; ++r) hit |= (v[8 * k + r] <= T ? 1u : 0u) << r;
                            while (hit) {
                                const int r = 8 * k + __ffs(hit) - 1;
                                hit &= hit - 1;
                                if (cnt < CAP && guard(a, tile_bad, g0 + r < g.flat, 42, g0 + r, cnt, g.flat))
                                    mylist[cnt * M + m] = (uint16_t)(g0 + r);
                                ++cnt;
                            }
                        }
                    }
                }
                if (prof) (pass2 ? t_p2 : t_p1) += clock64() - tp0;
            }
            fence_before_sync();
            __syncwarp();
            if (lane == 0) mbar_arrive(free0 + 8 * s);
            if (trace && q == 0 && lid == 0 && lane == 0) trace[3 * j + 2] = clock64();
            if (timeout) break;
        }
        if (!have_t) exchange();  // every warp of a quarter passes the boundary exactly once
        cntx[lid * M + m] = cnt;
        if (lid == 0) tx[m] = T;
    } else if (warp == MMA_WARP && lane == 0) {
        const uint32_t a_saddr = smem_u32(smem + OFF_A), e_saddr = smem_u32(smem + OFF_E),
                       t_saddr = smem_u32(smem + OFF_T), xp_saddr = smem_u32(smem + OFF_XP);
        const uint32_t row_bytes = 16u * (uint32_t)WX;
        for (int j = 0; j < J; ++j) {
            const int s = j & 1, c = j < nch ? j : j - nch;
            if (j >= 2 && !mbar_wait(free0 + 8 * s, ((j - 2) >> 1) & 1, polls)) {
                timeout = 1;
                break;
            }
            fence_after_sync();
            const uint32_t d = tbase + (uint32_t)(s * N);
            const uint32_t eb = e_saddr + 16u * (uint32_t)(c * N);
            const uint32_t tb = t_saddr + 16u * (uint32_t)(c * N);
            // last byte each operand's descriptors reach: E (8 patch rows of N candidates),
            // the norm table (N rows), the penalties (N rows), A (10 K chunks)
            const uint32_t e_end = eb + 7u * row_bytes + (uint32_t)(N * 16 - 1);
            const uint32_t t_end = tb + (uint32_t)(N * 16 - 1);
            if (!guard(a, tile_bad,
                       e_end < e_saddr + (uint32_t)SZ_E && t_end < t_saddr + (uint32_t)SZ_T && xp_saddr > tb &&
                           xp_saddr - tb < (1u << 18) && (d >> 16) == 0u && (d & 0xffffu) + N <= 512u,
                       30, (int)(e_end - e_saddr), (int)(t_end - t_saddr), (int)d)) {
                timeout = 1;
                break;
            }
#pragma unroll
            for (int kk = 0; kk < KSTEPS - 1; ++kk)
                mma_kind_f16(d, desc(a_saddr + 2 * kk * A_KCHUNK, A_KCHUNK, 128),
                             desc(eb + 2 * kk * row_bytes, row_bytes, 128), IDESC, kk);
            // norm terms (the chunk's table rows) and, as the K step's second 8-element
            // chunk, the column penalties (the same 224-row table for every chunk)
            mma_kind_f16(d, desc(a_saddr + 8 * A_KCHUNK, A_KCHUNK, 128), desc(tb, xp_saddr - tb, 128), IDESC, 1);
            mma_commit(done0 + 8 * s);
            if (trace) trace[3 * j] = clock64();
            last = j;
        }
    }
    const int stop = __syncthreads_or(timeout);
    if (prof) {
        const unsigned wp = __reduce_add_sync(0xffffffffu, polls);
        if (lane == 0) {
            atomicAdd(prof + (warp < MMA_WARP ? 8 : 10), (unsigned long long)wp);
            if (warp < MMA_WARP) {
                atomicAdd(prof + 11, (unsigned long long)t_ld);
                atomicAdd(prof + 12, (unsigned long long)t_p1);
                atomicAdd(prof + 13, (unsigned long long)n_ld);
                atomicAdd(prof + 14, (unsigned long long)t_p2);
                atomicAdd(prof + 15, (unsigned long long)t_wait);
            }
        }
    }
    // ---- drain and release tensor memory -------------------------------------------
    if (stop && warp == MMA_WARP && lane == 0 && last >= 0)
        mbar_wait(done0 + 8 * (last & 1), (last >> 1) & 1, polls);
    if (stop && tid == 0) a.tc_ws[1] = 1;
    fence_before_sync();
    __syncthreads();
    if (warp == MMA_WARP) {
        // lane 0 of this warp ran the MMA loop alone: tcgen05.dealloc is .sync.aligned, so
        // the warp must be converged before it
        __syncwarp();
        fence_after_sync();
        tmem_dealloc(tbase, 512);
    }
    if (prof && tid == 0) prof[5] = clock64();

    // ---- exact re-rank of the collected candidates from the FP32 region ------------
    // RR threads per block compute the exact errors of its collected candidates
    // (entries grp, grp + RR, ... of each of its lists); then the block's thread keeps
    // the eight smallest by (error, scan position).
    const bool skip_tile = stop || bad_tile;
    float *reg2 = reinterpret_cast<float *>(smem + OFF_E);  // the FP32 region again
    float *errs = reinterpret_cast<float *>(smem + OFF_T);  // [2][CAP][128]
    if (!skip_tile) stage_region(reg2, SZ_E / 4, plane, P, g, tid, a, tile_bad);
    __syncthreads();
    constexpr int RR = THREADS / M;  // threads per block in the exact re-rank
    if (!skip_tile && tid < RR * M) {
        const int m = tid & 127, grp = tid >> 7;
        const int mbx = m & 7, mby = m >> 3;
        const int cn0 = cntx[m], cn1 = cntx[M + m];
        const int cn2 = NLIST == 4 ? cntx[2 * M + m] : 0, cn3 = NLIST == 4 ? cntx[3 * M + m] : 0;
        const bool over = cn0 > CAP || cn1 > CAP || cn2 > CAP || cn3 > CAP;
        if (mbx < g.nvx && mby < g.nvy && !over && tx[m] < __int_as_float(0x7f800000)) {
            const float *ref = reg2 + (block_y(a, g.ky0 + mby) - g.uy0) * REG_COLS + (block_x(a, g.kx0 + mbx) - g.ux0);
            // thread grp of the block takes the entries grp, grp + RR, ... of each list
            for (int li = 0; li < NLIST; ++li) {
                const int n = li == 0 ? cn0 : li == 1 ? cn1 : li == 2 ? cn2 : cn3;
                for (int k = grp; k < n; k += RR) {
                    const int idx = (li * CAP + k) * M + m;
                    const int f = lists[idx];
                    const int r = f / WX, cc = f - r * WX;
                    errs[idx] = guard(a, tile_bad, r < g.nur && cc < nuc, 50, f, r, cc)
                                    ? exact_ssd2_s(ref, reg2 + r * REG_COLS + cc, REG_COLS)
                                    : 0.0f;
                }
            }
        }
    }
    __syncthreads();
    if (prof && tid == 0) prof[6] = clock64();
    if (tid >= M) return;
    const int cn0 = cntx[tid], cn1 = cntx[M + tid];
    const int cn2 = NLIST == 4 ? cntx[2 * M + tid] : 0, cn3 = NLIST == 4 ? cntx[3 * M + tid] : 0;
    const bool over = cn0 > CAP || cn1 > CAP || cn2 > CAP || cn3 > CAP;
    const int total = cn0 + cn1 + cn2 + cn3;
    const bool fb = valid && (skip_tile || *tile_bad || over || !(tx[tid] < __int_as_float(0x7f800000)));
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
                q[i] = 0x7fffffff;
            }
            for (int li = 0; li < NLIST; ++li) {
                const int n = li == 0 ? cn0 : li == 1 ? cn1 : li == 2 ? cn2 : cn3;
                for (int kk = 0; kk < n; ++kk) {
                    const int idx = (li * CAP + kk) * M + tid;
                    const int f = lists[idx];
                    const int r = f / WX, cc = f - r * WX;
                    top8_insert_lex(e, q, errs[idx], pack_pos(g.ux0 + cc, g.uy0 + r));
                }
            }
            bool in_plane = true;
#pragma unroll
            for (int i = 0; i < 8; ++i) in_plane = in_plane && pos_x(q[i]) <= W - 8 && pos_y(q[i]) <= H - 8;
            if (guard(a, tile_bad, in_plane, 60, bi, q[7], total))
                store_list(a, bi, xb, yb, e, q);
            else
                list_fallback(a, bi);
        }
    }
    if (prof && tid == 0) prof[7] = clock64();
    if (a.tc_stats) {
        const unsigned nval = __popc(__ballot_sync(0xffffffffu, valid));
        const unsigned nfb = __popc(__ballot_sync(0xffffffffu, fb));
        const unsigned ns = __reduce_add_sync(0xffffffffu, valid && !fb ? (unsigned)total : 0u);
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

// Flat candidates per block row of the debug dump (tile (0, 0)): chunks * 224.
int tc_debug_cols(const MatchArgs &a) {
    const int R = a.range;
    const int nvx = a.nbx < tc::BX ? a.nbx : tc::BX, nvy = a.nby < tc::BY ? a.nby : tc::BY;
    (void)nvx;
    const int y1 = std::min(std::min(a.bs * (nvy - 1), a.h - 8) + R, a.h - 8);
    const int nur = y1 + 1;
    const int nch = (nur + tc::ROWS_PER_CHUNK - 1) / tc::ROWS_PER_CHUNK;
    return nch * tc::N;
}

}  // namespace zb
