// zb3d device kernels: block matching, collaborative filtering, aggregation.
//
// Compiled for sm_100a with -use_fast_math, the same floating-point mode as the
// reference kernel (vszipcu src/bm3d.zig:20-24): flush-to-zero, approximate
// division / square root, FMA contraction.  Where bit-exact agreement with the
// reference matters (patch distances, transforms, shrinkage) the operation order
// is the reference's; the distance chains are written with explicit
// __fmul_rn/__fmaf_rn so the contraction is fixed by the source, not the compiler.
//
// Design (B200):
//  * Matching: one lane owns 4 columns ("half block") of a reference block and
//    slides a 4x8 candidate window along each candidate row.  With block_step 4,
//    lane k's half is the first half of block k and the second half of block
//    k-1, so every column distance is computed once for two blocks.  Candidate
//    rows of a whole warp-row of blocks are staged in a shared-memory tile and
//    read as float4 (bank-conflict free, no shuffles in the inner loop except one
//    to join the two halves).  The top-8 list lives in registers and follows the
//    reference's insertion rule in scan order, so the lists are bit-identical.
//  * Filtering: 16 lanes per group (32 values each), the reference's transform order, FP32.
//  * Aggregation: signed 64-bit fixed point (2^32 = 1.0) with integer atomics,
//    which is exact and order independent; the weight sum is accumulated once
//    per patch at its origin and expanded by an 8x8 box sum in the finish pass.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "zb3d_args.h"
#include "zb3d_match.cuh"
#include "zb3d_transforms.cuh"

namespace zb {

static constexpr unsigned kFull = 0xffffffffu;

// ---------------------------------------------------------------------------
// Global -> shared staging with cp.async: no register round trip, every copy of
// the CTA in flight at once, one wait.  Columns outside [0, w) are zero-filled
// (src-size 0; the source address then stays a valid in-plane address).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async_f32(float *sdst, const float *gsrc, bool valid) {
    const unsigned saddr = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(saddr), "l"(gsrc), "r"(valid ? 4 : 0)
                 : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// rows [0, nrows) x cols [0, ncols) of the plane window at (gx0, gy0) -> smem rows of pitch sp
__device__ __forceinline__ void stage_window(float *smem, int sp, const float *plane, long long pitch, int gx0,
                                             int gy0, int nrows, int ncols, int w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = warp; r < nrows; r += nw) {
        const float *srow = plane + (long long)(gy0 + r) * pitch;
        float *drow = smem + r * sp;
        for (int c = lane; c < ncols; c += 32) {
            const int gx = gx0 + c;
            const bool ok = gx >= 0 && gx < w;
            cp_async_f32(drow + c, srow + (ok ? gx : 0), ok);
        }
    }
}

// ---------------------------------------------------------------------------
// Patch distances, per half block (4 columns x 8 rows), vszipcu src/bm3d.cu:282-390.
// Column j: even rows and odd rows accumulate separately, column = e0 + e1; the
// 8 columns join as ((s0+s1)+(s2+s3)) + ((s4+s5)+(s6+s7)): each half returns its
// bracket, the caller adds the two halves.  `st` is the reference patch's
// statistic (mean for zssd/zsad, norm for ssd/norm); `pm` the lane-pair mask.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float colsum8(const float (&n)[8][4], int j) {
    return ((n[0][j] + n[1][j]) + (n[2][j] + n[3][j])) + ((n[4][j] + n[5][j]) + (n[6][j] + n[7][j]));
}

template <int M>
__device__ __forceinline__ float half_distance(const float (&c)[8][4], const float (&n)[8][4], float st, unsigned pm) {
    float s[4] = {0.0f, 0.0f, 0.0f, 0.0f};
    if constexpr (M == M_SSD) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float d[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) d[i] = c[i][j] - n[i][j];
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
    } else if constexpr (M == M_SAD) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float e0 = 0.0f, e1 = 0.0f;
#pragma unroll
            for (int i = 0; i < 8; i += 2) {
                e0 += fabsf(c[i][j] - n[i][j]);
                e1 += fabsf(c[i + 1][j] - n[i + 1][j]);
            }
            s[j] = e0 + e1;
        }
    } else if constexpr (M == M_ZSSD || M == M_ZSAD) {
        float hsum = (colsum8(n, 0) + colsum8(n, 1)) + (colsum8(n, 2) + colsum8(n, 3));
        float tot = hsum + __shfl_xor_sync(pm, hsum, 1);
        const float dm = st - tot * (1.0f / 64.f);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float v[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) v[i] = (c[i][j] - n[i][j]) - dm;
            if constexpr (M == M_ZSSD) {
                float e0 = __fmul_rn(v[0], v[0]);
                float e1 = __fmul_rn(v[1], v[1]);
                e0 = __fmaf_rn(v[2], v[2], e0);
                e1 = __fmaf_rn(v[3], v[3], e1);
                e0 = __fmaf_rn(v[4], v[4], e0);
                e1 = __fmaf_rn(v[5], v[5], e1);
                e0 = __fmaf_rn(v[6], v[6], e0);
                e1 = __fmaf_rn(v[7], v[7], e1);
                s[j] = e0 + e1;
            } else {
                float e0 = 0.0f, e1 = 0.0f;
#pragma unroll
                for (int i = 0; i < 8; i += 2) {
                    e0 += fabsf(v[i]);
                    e1 += fabsf(v[i + 1]);
                }
                s[j] = e0 + e1;
            }
        }
    } else {  // M_SSD_NORM: 2 - 2 <a,b> / (|a| |b| + eps)
        float q[4], x[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float e0 = __fmul_rn(n[0][j], n[0][j]);
            float e1 = __fmul_rn(n[1][j], n[1][j]);
            float f0 = __fmul_rn(c[0][j], n[0][j]);
            float f1 = __fmul_rn(c[1][j], n[1][j]);
#pragma unroll
            for (int i = 2; i < 8; i += 2) {
                e0 = __fmaf_rn(n[i][j], n[i][j], e0);
                e1 = __fmaf_rn(n[i + 1][j], n[i + 1][j], e1);
                f0 = __fmaf_rn(c[i][j], n[i][j], f0);
                f1 = __fmaf_rn(c[i + 1][j], n[i + 1][j], f1);
            }
            q[j] = e0 + e1;
            x[j] = f0 + f1;
        }
        float hq = (q[0] + q[1]) + (q[2] + q[3]);
        float hx = (x[0] + x[1]) + (x[2] + x[3]);
        float nn = sqrtf(hq + __shfl_xor_sync(pm, hq, 1));
        float dot = hx + __shfl_xor_sync(pm, hx, 1);
        // full distance; the caller's half join is skipped for this metric.  The
        // reference's 2 - 2 dot / (|a| |b| + eps) under fast math is the approximate
        // reciprocal of the denominator with the subtraction fused into it; written out
        // so that no kernel's instruction selection can round it differently
        float r;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(__fmaf_rn(st, nn, ZB_FLT_EPS)));
        return __fmaf_rn(-2.0f * dot, r, 2.0f);
    }
    return (s[0] + s[1]) + (s[2] + s[3]);
}

// Joins the two half distances (pair lanes) into the block distance.
template <int M>
__device__ __forceinline__ float join_pair(float hd, unsigned pm) {
    if constexpr (M == M_SSD_NORM) return hd;
    return hd + __shfl_xor_sync(pm, hd, 1);
}

// Statistic of the reference patch needed by the mean- or norm-based metrics.
template <int M>
__device__ __forceinline__ float ref_stat(const float (&c)[8][4], unsigned pm) {
    if constexpr (M == M_ZSSD || M == M_ZSAD) {
        float h = (colsum8(c, 0) + colsum8(c, 1)) + (colsum8(c, 2) + colsum8(c, 3));
        return (h + __shfl_xor_sync(pm, h, 1)) * (1.0f / 64.f);
    } else if constexpr (M == M_SSD_NORM) {
        float q[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            float e0 = __fmul_rn(c[0][j], c[0][j]);
            float e1 = __fmul_rn(c[1][j], c[1][j]);
#pragma unroll
            for (int i = 2; i < 8; i += 2) {
                e0 = __fmaf_rn(c[i][j], c[i][j], e0);
                e1 = __fmaf_rn(c[i + 1][j], c[i + 1][j], e1);
            }
            q[j] = e0 + e1;
        }
        float h = (q[0] + q[1]) + (q[2] + q[3]);
        return sqrtf(h + __shfl_xor_sync(pm, h, 1));
    }
    return 0.0f;
}

// metrics whose column terms can be shared between neighbouring blocks
template <int M> struct Shareable { static constexpr bool value = (M == M_SSD || M == M_SAD); };

__device__ __forceinline__ float f4c(const float4 &v, int k) {
    return k == 0 ? v.x : k == 1 ? v.y : k == 2 ? v.z : v.w;
}

// ---------------------------------------------------------------------------
// Spatial matching, block_step 4 or 8, from a shared-memory tile.
// A warp covers one row of reference blocks; lane k's half starts at column
// x0 + 4k (SHARED: block k = lanes k, k+1) or, in PAIR mode, block b = lanes
// 2b, 2b+1.  The CTA's warps take consecutive block rows and share the tile,
// which is staged with cp.async.  Each candidate row is scanned in chunks of 4
// displacements; the two float4 window halves alternate roles between chunks so
// the sliding window never moves between registers.
// ---------------------------------------------------------------------------
template <int M, bool SHARED>
__device__ __forceinline__ void tiled_chunk(const float4 (&X)[8], const float4 (&Y)[8], int m, int R, int row, int xb,
                                            int lo, int hi, const float (&c)[8][4], float st, float (&e)[8],
                                            int (&q)[8]) {
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int dx = -R + 4 * m + s;
        if (dx > R) break;
        float n[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) n[i][j] = (j + s < 4) ? f4c(X[i], j + s) : f4c(Y[i], j + s - 4);
        const float hd = half_distance<M>(c, n, st, kFull);
        float err;
        if constexpr (SHARED)
            err = hd + __shfl_down_sync(kFull, hd, 1);
        else
            err = join_pair<M>(hd, kFull);
        if (dx >= lo && dx <= hi && err < e[7]) top8_insert(e, q, err, pack_pos(xb + dx, row));
    }
}

template <int M, bool SHARED, int BS>
__global__ void __launch_bounds__(128) zb_match_tiled(MatchArgs a) {
    extern __shared__ __align__(16) float tile[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    constexpr int NBW = SHARED ? 31 : 16;
    const int R = a.range, W = a.w, H = a.h, tp = a.tile_pitch;
    const int kx0 = blockIdx.x * NBW;
    const int x0 = kx0 * BS;
    const int by0 = blockIdx.y * nw;
    const int by_last = min(by0 + nw - 1, a.nby - 1);
    const int y_first = min(BS * by0, H - 8);
    const int y_last = min(BS * by_last, H - 8);
    const int r0 = max(y_first - R, 0);
    const int nrows = min(y_last + R, H - 8) + 8 - r0;
    const float *plane = a.frames + (long long)a.radius * a.fstride;
    stage_window(tile, tp, plane, a.pitch, x0 - R, r0, nrows, tp, W);
    cp_async_wait_all();
    __syncthreads();

    const int by = by0 + warp;
    if (by >= a.nby) return;
    const int y = min(BS * by, H - 8);
    const int b = SHARED ? lane : (lane >> 1);
    const int hh = SHARED ? 0 : (lane & 1);
    const int kx = kx0 + b;
    const int xb = BS * kx;
    const int uo = BS * b + 4 * hh;  // tile column of this half at dx = -R
    const bool blk = (SHARED ? lane < 31 : true) && kx < a.nbx_al;

    float c[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) c[i][j] = tile[(y - r0 + i) * tp + uo + R + j];
    const float st = ref_stat<M>(c, kFull);

    float e[8];
    int q[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        e[i] = ZB_FLT_MAX;
        q[i] = 0;
    }
    const int top = max(y - R, 0), bottom = min(y + R, H - 8);
    // valid displacements of this block: 0 <= xb + dx <= W - 8 (none for helper lanes)
    const int lo = blk ? -xb : 1, hi = blk ? W - 8 - xb : 0;
    const int chunks = a.chunks;

    for (int row = top; row <= bottom; ++row) {
        const float *tr = tile + (row - r0) * tp + uo;
        float4 A[8], B[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) A[i] = *reinterpret_cast<const float4 *>(tr + i * tp);
        for (int m = 0; m < chunks; m += 2) {
#pragma unroll
            for (int i = 0; i < 8; ++i) B[i] = *reinterpret_cast<const float4 *>(tr + i * tp + 4 * (m + 1));
            tiled_chunk<M, SHARED>(A, B, m, R, row, xb, lo, hi, c, st, e, q);
            if (m + 1 < chunks) {
#pragma unroll
                for (int i = 0; i < 8; ++i) A[i] = *reinterpret_cast<const float4 *>(tr + i * tp + 4 * (m + 2));
                tiled_chunk<M, SHARED>(B, A, m + 1, R, row, xb, lo, hi, c, st, e, q);
            }
        }
    }

    if (!blk || (!SHARED && hh)) return;
    store_list(a, (long long)by * a.nbx + kx, xb, y, e, q);
}

// ---------------------------------------------------------------------------
// SSD matching with packed FP32x2 arithmetic (sm_100 FADD2 / FMUL2 / FFMA2).
// The tile is stored twice with candidate rows interleaved in pairs, once with
// pairs starting at even tile rows and once at odd ones; a float2 then holds
// rows (2k, 2k+1) of one column of a window, exactly the operands of the even-
// and odd-row partial sums, which advance together: acc = fma2(d, d, acc)
// computes the reference's e0 and e1 chains in one instruction and acc.x + acc.y
// is their join.  d = n + (-c) = -(c - n) exactly, so d*d is the reference's
// square.  A pair row holds the tile's columns as 16-byte chunks of two columns
// each, in two half-planes of g chunks: columns 4u, 4u+1 form chunk u of the first,
// columns 4u+2, 4u+3 chunk u of the second.  A lane's block half starts at a column
// that is a multiple of 4, so at every step the lanes of a quarter warp read eight
// consecutive chunks of one half-plane (float4 loads free of bank conflicts), and a
// lane's address advances by one chunk per displacement chunk.  With g fixed at
// compile time (kTile2G, for up to 8 chunks of displacements: bm_range <= 15) every
// other offset is an immediate.
// ---------------------------------------------------------------------------
constexpr int kTile2G = 40;  // half-plane chunks of the fixed layout (tile pitch <= 160)

__host__ __device__ constexpr int tile2_g(int tile_pitch, bool fixed) {  // chunks per half-plane
    return fixed ? kTile2G : tile_pitch / 4;
}

__host__ __device__ constexpr bool tile2_fixed(int chunks) { return chunks <= (4 * kTile2G - 128) / 4; }

// float offset of column `col` in a pair row of half-plane size g
__device__ __forceinline__ int split_off(int col, int g) { return ((col >> 1) & 1) * 4 * g + 4 * (col >> 2) + 2 * (col & 1); }

__device__ __forceinline__ float2 f4lo(const float4 &v) { return make_float2(v.x, v.y); }
__device__ __forceinline__ float2 f4hi(const float4 &v) { return make_float2(v.z, v.w); }

// One chunk: displacements dx = -R + 4m + s (s = 0..3) of candidate row `row`.  The
// chunk reads window columns c0 .. c0 + 6 (c0 = the lane's tile column at dx = -R, plus
// 4m; a multiple of 4) of the four pair rows; pc points at column c0 of the first pair
// row.  GF: half-plane chunks when fixed at compile time, else 0 (pp_rt and g_rt give
// the pitch and half-plane size).  The columns are loaded one column pair at a time, just
// before the sums that use them: column col feeds the (s, j = col - s) chains, each
// of which runs over its pair rows k = 0..3 in order, so every sum is the reference's.
// Keeping no window in registers holds the kernel at 112-116 registers.  The four distances
// come first (no branch between their FMA chains), then the insertions in scan order;
// a displacement past R is computed from the tile's padding columns and discarded.
template <bool SHARED, int GF>
__device__ __forceinline__ void tiled2_chunk(const float *pc, int pp_rt, int g_rt, int m, int R, int row, int xb,
                                             int lo, int hi, const float2 (&nc)[4][4], float (&e)[8], int (&q)[8]) {
    const int pp = GF ? 8 * GF : pp_rt, g = GF ? GF : g_rt;
    float sj[4][4];
#pragma unroll
    for (int p = 0; p < 4; ++p) {
        float4 v[4];  // columns (2p, 2p + 1) of pair rows k: (row 2k, row 2k + 1) of each
#pragma unroll
        for (int k = 0; k < 4; ++k)
            v[k] = *reinterpret_cast<const float4 *>(pc + k * pp + (p & 1) * 4 * g + 4 * (p >> 1));
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int col = 2 * p + h;
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int j = col - s;
                if (j < 0 || j > 3) continue;
                float2 d = __fadd2_rn(h ? f4hi(v[0]) : f4lo(v[0]), nc[0][j]);
                float2 acc = __fmul2_rn(d, d);
#pragma unroll
                for (int k = 1; k < 4; ++k) {
                    d = __fadd2_rn(h ? f4hi(v[k]) : f4lo(v[k]), nc[k][j]);
                    acc = __ffma2_rn(d, d, acc);
                }
                sj[s][j] = acc.x + acc.y;
            }
        }
    }
    float err[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) err[s] = (sj[s][0] + sj[s][1]) + (sj[s][2] + sj[s][3]);
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        if constexpr (SHARED)
            err[s] += __shfl_down_sync(kFull, err[s], 1);
        else
            err[s] += __shfl_xor_sync(kFull, err[s], 1);
    }
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const int dx = -R + 4 * m + s;
        if (dx <= R && dx >= lo && dx <= hi && err[s] < e[7]) top8_insert(e, q, err[s], pack_pos(xb + dx, row));
    }
}

// One tile of the packed FP32x2 SSD matcher: block columns [31 bx, 31 bx + 31) (SHARED)
// or [16 bx, ...), block rows [nw by, nw by + nw), nw = the CTA's warps; `tile` is the
// dynamic shared-memory tile (match_tile2_bytes).
template <bool SHARED, int BS, bool FIXED>
__device__ __forceinline__ void match_tiled2_tile_g(const MatchArgs &a, int bx, int by_cta, float *tile) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    constexpr int NBW = SHARED ? 31 : 16;
    const int R = a.range, W = a.w, H = a.h, tp = a.tile_pitch;
    const int g = tile2_g(tp, FIXED), pp = 8 * g;
    const int kx0 = bx * NBW;
    const int x0 = kx0 * BS;
    const int by0 = by_cta * nw;
    const int by_last = min(by0 + nw - 1, a.nby - 1);
    const int y_first = min(BS * by0, H - 8);
    const int y_last = min(BS * by_last, H - 8);
    const int r0 = max(y_first - R, 0);
    const int nrows = min(y_last + R, H - 8) + 8 - r0;
    const int npe = (nrows + 1) >> 1;  // even-start pair rows
    float *tE = tile;
    float *tO = tile + npe * pp;
    const float *plane = a.frames + (long long)a.radius * a.fstride;
    {
        const int gx0 = x0 - R;
        for (int t = warp; t < nrows; t += nw) {
            const float *srow = plane + (long long)(r0 + t) * a.pitch;
            float *de = tE + (t >> 1) * pp + (t & 1);
            float *dq = t > 0 ? tO + ((t - 1) >> 1) * pp + ((t - 1) & 1) : nullptr;
            for (int c = lane; c < tp; c += 32) {
                const int gx = gx0 + c;
                const bool ok = gx >= 0 && gx < W;
                const float *gs = srow + (ok ? gx : 0);
                cp_async_f32(de + split_off(c, g), gs, ok);
                if (dq) cp_async_f32(dq + split_off(c, g), gs, ok);
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();

    const int by = by0 + warp;
    if (by >= a.nby) return;
    const int y = min(BS * by, H - 8);
    const int b = SHARED ? lane : (lane >> 1);
    const int hh = SHARED ? 0 : (lane & 1);
    const int kx = kx0 + b;
    const int xb = BS * kx;
    const int uo = BS * b + 4 * hh;  // tile column of this half at dx = -R (a multiple of 4)
    const bool blk = (SHARED ? lane < 31 : true) && kx < a.nbx_al;

    // negated reference half as row pairs (2k, 2k+1) of each of its 4 columns
    float2 nc[4][4];
    {
        const int t0 = y - r0;
        const float *base = (t0 & 1) ? tO + ((t0 - 1) >> 1) * pp : tE + (t0 >> 1) * pp;
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const float2 v = *reinterpret_cast<const float2 *>(base + k * pp + split_off(uo + R + j, g));
                nc[k][j] = make_float2(-v.x, -v.y);
            }
    }

    float e[8];
    int q[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        e[i] = ZB_FLT_MAX;
        q[i] = 0;
    }
    const int top = max(y - R, 0), bottom = min(y + R, H - 8);
    const int lo = blk ? -xb : 1, hi = blk ? W - 8 - xb : 0;
    const int chunks = a.chunks;

    for (int row = top; row <= bottom; ++row) {
        const int t0 = row - r0;
        const float *prow = (t0 & 1) ? tO + ((t0 - 1) >> 1) * pp : tE + (t0 >> 1) * pp;
        const float *pc = prow + uo;  // column uo: chunk uo / 4 of the first half-plane
        for (int m = 0; m < chunks; ++m, pc += 4)
            tiled2_chunk<SHARED, FIXED ? kTile2G : 0>(pc, pp, g, m, R, row, xb, lo, hi, nc, e, q);
    }

    if (!blk || (!SHARED && hh)) return;
    store_list(a, (long long)by * a.nbx + kx, xb, y, e, q);
}

// The tile with the fixed half-plane size where the displacements allow it.
template <bool SHARED, int BS>
__device__ __forceinline__ void match_tiled2_tile(const MatchArgs &a, int bx, int by_cta, float *tile) {
    if (tile2_fixed(a.chunks))
        match_tiled2_tile_g<SHARED, BS, true>(a, bx, by_cta, tile);
    else
        match_tiled2_tile_g<SHARED, BS, false>(a, bx, by_cta, tile);
}

// Up to 8 block rows (warps) per CTA; 2 CTAs of 8 warps fit the register file.
template <bool SHARED, int BS>
__global__ void __launch_bounds__(256, 2) zb_match_tiled2(MatchArgs a) {
    extern __shared__ __align__(16) float tile[];
    match_tiled2_tile<SHARED, BS>(a, blockIdx.x, blockIdx.y, tile);
}

// ---------------------------------------------------------------------------
// Scan of one rectangular candidate window from global memory by a lane pair
// (row-major, the reference's order).  `plane` is already offset by this
// lane's half (4*hh columns).  A 4-column ring holds the sliding window.
// ---------------------------------------------------------------------------
template <int M, int K = 8>
__device__ __forceinline__ void scan_window(const float *__restrict__ plane, int pitch, int left, int right, int top,
                                            int bottom, const float (&c)[8][4], float st, unsigned pm,
                                            float (&e)[K], int (&q)[K]) {
    for (int row = top; row <= bottom; ++row) {
        const float *rp = plane + (long long)row * pitch;
        float w[8][4];
#pragma unroll
        for (int i = 0; i < 8; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) w[i][j] = __ldg(rp + i * pitch + left + j);
        for (int col = left; col <= right; col += 4) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int cc = col + s;
                if (cc > right) break;
                float n[8][4];
#pragma unroll
                for (int i = 0; i < 8; ++i)
#pragma unroll
                    for (int j = 0; j < 4; ++j) n[i][j] = w[i][(s + j) & 3];
                const float hd = half_distance<M>(c, n, st, pm);
                const float err = join_pair<M>(hd, pm);
                if (err < e[K - 1]) topk_insert<K>(e, q, err, pack_pos(cc, row));
                if (cc + 1 <= right) {
#pragma unroll
                    for (int i = 0; i < 8; ++i) w[i][s] = __ldg(rp + i * pitch + cc + 4);
                }
            }
        }
    }
}

// The same scan for SSD on packed FP32x2 arithmetic: the ring holds rows (2k, 2k+1) of
// each of its 4 columns as a float2, nc the negated reference half in the same pairs, and
// one __ffma2_rn advances the even-row and the odd-row chain of a column together (each
// with its own rounding), so every distance is half_distance<M_SSD>'s; n + (-c) is
// exactly -(c - n), so the squares are the same.
template <int K = 8>
__device__ __forceinline__ void scan_window_ssd2(const float *__restrict__ plane, int pitch, int left, int right,
                                                 int top, int bottom, const float2 (&nc)[4][4], unsigned pm,
                                                 float (&e)[K], int (&q)[K]) {
    for (int row = top; row <= bottom; ++row) {
        const float *rp = plane + (long long)row * pitch;
        float2 w[4][4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int j = 0; j < 4; ++j)
                w[k][j] = make_float2(__ldg(rp + 2 * k * pitch + left + j), __ldg(rp + (2 * k + 1) * pitch + left + j));
        for (int col = left; col <= right; col += 4) {
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                const int cc = col + s;
                if (cc > right) break;
                float sj[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    float2 d = __fadd2_rn(w[0][(s + j) & 3], nc[0][j]);
                    float2 acc = __fmul2_rn(d, d);
#pragma unroll
                    for (int k = 1; k < 4; ++k) {
                        d = __fadd2_rn(w[k][(s + j) & 3], nc[k][j]);
                        acc = __ffma2_rn(d, d, acc);
                    }
                    sj[j] = acc.x + acc.y;
                }
                const float hd = (sj[0] + sj[1]) + (sj[2] + sj[3]);
                const float err = hd + __shfl_xor_sync(pm, hd, 1);
                if (err < e[K - 1]) topk_insert<K>(e, q, err, pack_pos(cc, row));
                if (cc + 1 <= right) {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        w[k][s] = make_float2(__ldg(rp + 2 * k * pitch + cc + 4), __ldg(rp + (2 * k + 1) * pitch + cc + 4));
                }
            }
        }
    }
}

// The negated reference half as row pairs (2k, 2k+1) of each of its 4 columns.
__device__ __forceinline__ void neg_pairs(const float (&c)[8][4], float2 (&nc)[4][4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int j = 0; j < 4; ++j) nc[k][j] = make_float2(-c[2 * k][j], -c[2 * k + 1][j]);
}

// Spatial matching for block steps the tiled kernels do not take (and the blocks the
// tensor-core form lists), reading candidates through the L1/L2 path.  Lane pair per block.
template <int M>
__global__ void __launch_bounds__(128) zb_match_global(MatchArgs a) {
    const int lane = threadIdx.x & 31;
    const long long pair = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 1;
    const int hh = lane & 1;
    const long long nb = a.gen_mode == 2 ? (long long)a.tc_ws[0] : (long long)a.nby * a.nbx;
    if (pair >= nb) return;
    int kx, by;
    if (a.gen_mode == 2) {
        const int bi = a.tc_ws[kTcWsList + pair];
        by = bi / a.nbx;
        kx = bi - by * a.nbx;
    } else {
        by = (int)(pair / a.nbx);
        kx = (int)(pair - (long long)by * a.nbx);
    }
    const int W = a.w, H = a.h, R = a.range;
    const int x = min(a.bs * kx, W - 8), y = min(a.bs * by, H - 8);
    const unsigned pm = 3u << (lane & 30);
    const float *plane = a.frames + (long long)a.radius * a.fstride + 4 * hh;

    float c[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) c[i][j] = __ldg(plane + (long long)(y + i) * a.pitch + x + j);
    const float st = ref_stat<M>(c, pm);
    float e[8];
    int q[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        e[i] = ZB_FLT_MAX;
        q[i] = 0;
    }
    if constexpr (M == M_SSD) {
        float2 nc[4][4];
        neg_pairs(c, nc);
        scan_window_ssd2(plane, a.pitch, max(x - R, 0), min(x + R, W - 8), max(y - R, 0), min(y + R, H - 8), nc, pm,
                         e, q);
    } else {
        scan_window<M>(plane, a.pitch, max(x - R, 0), min(x + R, W - 8), max(y - R, 0), min(y + R, H - 8), c, st, pm,
                       e, q);
    }
    if (hh) return;
    const long long bi = (long long)by * a.nbx + kx;
    const int self = pack_pos(x, y);
    if (a.self_incl) {
        bool found = false;
#pragma unroll
        for (int i = 0; i < 8; ++i) found |= (q[i] == self);
        if (!found) {
#pragma unroll
            for (int i = 7; i > 0; --i) {
                e[i] = e[i - 1];
                q[i] = q[i - 1];
            }
            e[0] = 0.0f;
            q[0] = self;
        }
    }
    const int zr = a.radius << 24;
#pragma unroll
    for (int i = 0; i < 8; ++i) a.list[bi * 8 + i] = make_int2(pos_x(q[i]), pos_y(q[i]) | zr);
    if (a.errs) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a.errs[bi * 8 + i] = e[i];
    }
}

// The clamped last block column (x = W - 8) that the tiled kernels leave out: one warp per
// block.  Its candidate rows are split into 16 consecutive ranges in order, one per lane
// pair, each scanned in the reference's order into a list of its own; the lists are then
// merged in row order, a later range's entries inserted (strict less) after the earlier
// ranges', which is the list of one scan over all the rows.
template <int M>
__global__ void __launch_bounds__(128) zb_match_column(MatchArgs a) {
    const int lane = threadIdx.x & 31;
    const int by = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (by >= a.nby) return;  // whole warps
    const int hh = lane & 1, pr = lane >> 1;
    const int W = a.w, H = a.h, R = a.range;
    const int kx = a.nbx - 1;
    const int x = min(a.bs * kx, W - 8), y = min(a.bs * by, H - 8);
    const unsigned pm = 3u << (lane & 30);
    const float *plane = a.frames + (long long)a.radius * a.fstride + 4 * hh;

    float c[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) c[i][j] = __ldg(plane + (long long)(y + i) * a.pitch + x + j);
    const float st = ref_stat<M>(c, pm);
    float e[8];
    int q[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        e[i] = ZB_FLT_MAX;
        q[i] = 0;
    }
    const int top = max(y - R, 0), bottom = min(y + R, H - 8);
    const int per = (bottom - top + 16) / 16;
    const int r0 = top + pr * per, r1 = min(r0 + per - 1, bottom);
    if (r0 <= r1) {
        if constexpr (M == M_SSD) {
            float2 nc[4][4];
            neg_pairs(c, nc);
            scan_window_ssd2(plane, a.pitch, max(x - R, 0), min(x + R, W - 8), r0, r1, nc, pm, e, q);
        } else {
            scan_window<M>(plane, a.pitch, max(x - R, 0), min(x + R, W - 8), r0, r1, c, st, pm, e, q);
        }
    }
#pragma unroll
    for (int k = 1; k < 16; k <<= 1) {
        float oe[8];
        int oq[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            oe[i] = __shfl_down_sync(kFull, e[i], 2 * k);
            oq[i] = __shfl_down_sync(kFull, q[i], 2 * k);
        }
        if ((pr & (2 * k - 1)) == 0) {
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (oe[i] < e[7]) top8_insert(e, q, oe[i], oq[i]);
        }
    }
    if (lane != 0) return;
    const long long bi = (long long)by * a.nbx + kx;
    const int self = pack_pos(x, y);
    if (a.self_incl) {
        bool found = false;
#pragma unroll
        for (int i = 0; i < 8; ++i) found |= (q[i] == self);
        if (!found) {
#pragma unroll
            for (int i = 7; i > 0; --i) {
                e[i] = e[i - 1];
                q[i] = q[i - 1];
            }
            e[0] = 0.0f;
            q[0] = self;
        }
    }
    const int zr = a.radius << 24;
#pragma unroll
    for (int i = 0; i < 8; ++i) a.list[bi * 8 + i] = make_int2(pos_x(q[i]), pos_y(q[i]) | zr);
    if (a.errs) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a.errs[bi * 8 + i] = e[i];
    }
}

// ---------------------------------------------------------------------------
// Temporal predictive search (vszipcu src/bm3d.cu:663-756) and self inclusion
// (:758-788).  Starts from the spatial list; for direction -1 then +1 and
// t = 1..r a per-frame list is built from ps_range windows around the first
// ps_num entries of the previous list (t = 1: the spatial list), and its first
// ps_num entries are merged into the block's list.  Only those first ps_num entries of a
// per-frame list are ever read, so the per-frame list holds K >= ps_num entries: the
// first K of the reference's 8-entry list (K = 2 covers the default ps_num).  For SSD the
// kernel is held at 128 registers, 4 CTAs per SM, so that a 1080p plane at block_step 8
// (507 CTAs) runs in one wave; the other metrics keep their 3 CTAs per SM.
// ---------------------------------------------------------------------------
template <int M, int K>
__global__ void __launch_bounds__(128, M == M_SSD ? 4 : 3) zb_match_temporal(MatchArgs a) {
    const int lane = threadIdx.x & 31;
    const long long pair = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 1;
    const int hh = lane & 1;
    const long long nb = (long long)a.nby * a.nbx;
    if (pair >= nb) return;
    const int by = (int)(pair / a.nbx), kx = (int)(pair - (long long)by * a.nbx);
    const int W = a.w, H = a.h, r = a.radius, P = a.ps_range;
    const int x = min(a.bs * kx, W - 8), y = min(a.bs * by, H - 8);
    const unsigned pm = 3u << (lane & 30);
    const float *centre = a.frames + (long long)r * a.fstride + 4 * hh;

    float c[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) c[i][j] = __ldg(centre + (long long)(y + i) * a.pitch + x + j);
    const float st = ref_stat<M>(c, pm);
    float2 nc[4][4];
    if constexpr (M == M_SSD) neg_pairs(c, nc);

    float ge[8];
    int gq[8], gz[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int2 v = a.list[pair * 8 + i];
        ge[i] = a.errs[pair * 8 + i];
        gq[i] = pack_pos(v.x, v.y & 0xffffff);
        gz[i] = r;
    }
#pragma unroll 1
    for (int dir = -1; dir <= 1; dir += 2) {
        // each direction starts from the spatial list (still unchanged in memory)
        int lq[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int2 v = a.list[pair * 8 + i];
            lq[i] = pack_pos(v.x, v.y & 0xffffff);
        }
#pragma unroll 1
        for (int t = 1; t <= r; ++t) {
            const int zt = r + dir * t;
            const float *fp = a.frames + (long long)zt * a.fstride + 4 * hh;
            float fe[K];
            int fq[K];
#pragma unroll
            for (int i = 0; i < K; ++i) {
                fe[i] = ZB_FLT_MAX;
                fq[i] = 0;
            }
#pragma unroll
            for (int i = 0; i < K; ++i) {
                if (i < a.ps_num) {
                    const int xx = pos_x(lq[i]), yy = pos_y(lq[i]);
                    if constexpr (M == M_SSD)
                        scan_window_ssd2<K>(fp, a.pitch, max(xx - P, 0), min(xx + P, W - 8), max(yy - P, 0),
                                            min(yy + P, H - 8), nc, pm, fe, fq);
                    else
                        scan_window<M, K>(fp, a.pitch, max(xx - P, 0), min(xx + P, W - 8), max(yy - P, 0),
                                          min(yy + P, H - 8), c, st, pm, fe, fq);
                }
            }
#pragma unroll
            for (int i = 0; i < K; ++i)
                if (i < a.ps_num && fe[i] < ge[7]) top8_insert_z(ge, gq, gz, fe[i], fq[i], zt);
#pragma unroll
            for (int i = 0; i < K; ++i) lq[i] = fq[i];
        }
    }
    if (hh) return;
    const int self = pack_pos(x, y);
    bool found = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) found |= (gq[i] == self && gz[i] == r);
    if (!found) {
#pragma unroll
        for (int i = 7; i > 0; --i) {
            gq[i] = gq[i - 1];
            gz[i] = gz[i - 1];
        }
        gq[0] = self;
        gz[0] = r;
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) a.list[pair * 8 + i] = make_int2(pos_x(gq[i]), pos_y(gq[i]) | (gz[i] << 24));
}

// ---------------------------------------------------------------------------
// Collaborative filtering (vszipcu src/bm3d.cu:392-546) and aggregation into
// signed 64-bit fixed point.
// ---------------------------------------------------------------------------
static constexpr int kFilterWarps = 4;

__device__ __forceinline__ unsigned long long to_fix(float v) {
    return (unsigned long long)__float2ll_rn(v * kFixScale);
}

// ---------------------------------------------------------------------------
// Collaborative filtering with 16 lanes per group.  Lane (j, h), j = 0..7,
// h = 0..1, holds 32 of the group's 512 values, half of what a lane of an
// 8-lane group holds, so twice as many groups are resident per SM.  Every 1-D
// transform still runs on 8 values inside one lane, in the reference's order;
// between transforms the values move through shared memory.  The layouts
// (q, t = 0..3; the half h takes the interleaved indices 2q + h, 2t + h):
//   A  column x = j of patches 2q + h, all rows          gather, vertical forward
//   B  row fy = j of patches 2q + h, all columns         horizontal forward
//   C  column fx = j, rows fy = 2t + h, all patches      across patches (Wiener coefficients)
//   D  column fx = j of spectra 2q + h, all rows         shrinkage, vertical inverse
//   E  row y = j of spectra 2q + h, all columns          horizontal inverse
//   F  column x = j, rows y = 2t + h, all patches        inverse across patches, aggregation
// Registers: A, B, D, E as d[q * 8 + i]; C, F as d[p * 4 + t].  The strides of the
// three kinds of move (A->B and D->E, B->C and E->F, C->D) were chosen so that the
// 32 lanes of a warp (two groups) touch 32 distinct banks on every store and load.
// The shrinkage runs in layout D with the vertical inverse directly after it in
// registers, the same code shape as the reference (src/bm3d.cu:445, 457-478): its
// transforms write a * b + c and leave the fusing into FMAs to the compiler, and
// the compiler fuses this stage the reference's way only in that shape.
// ---------------------------------------------------------------------------
static constexpr int kGroupBuf = 592;    // floats per group in the move buffer
static constexpr int kCoeffBuf = 592;    // floats per group in the Wiener coefficient buffer

// A -> B and D -> E: 8x8 transpose of each of the lane's four patches
__device__ __forceinline__ void move_tr(float (&d)[32], float *gb, int h, int j, unsigned gm) {
    __syncwarp(gm);
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int i = 0; i < 8; ++i) gb[(2 * q + h) * 72 + i + 9 * j] = d[q * 8 + i];
    __syncwarp(gm);
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int i = 0; i < 8; ++i) d[q * 8 + i] = gb[(2 * q + h) * 72 + j + 9 * i];
}

// B -> C and E -> F: (patch 2q + h, row j, column i) -> (patch p, row 2t + h, column j)
__device__ __forceinline__ void move_bc(float (&d)[32], float *gb, int h, int j, unsigned gm) {
    __syncwarp(gm);
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int i = 0; i < 8; ++i) gb[(2 * q + h) * 72 + 9 * j + 2 * i] = d[q * 8 + i];
    __syncwarp(gm);
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int t = 0; t < 4; ++t) d[p * 4 + t] = gb[p * 72 + 9 * (2 * t + h) + 2 * j];
}

// C -> D: (spectrum p, row 2t + h, column j) -> (spectrum 2q + h, row i, column j)
__device__ __forceinline__ void move_cd(float (&d)[32], float *gb, int h, int j, unsigned gm) {
    __syncwarp(gm);
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int t = 0; t < 4; ++t) gb[p * 72 + 8 * (2 * t + h) + j] = d[p * 4 + t];
    __syncwarp(gm);
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int i = 0; i < 8; ++i) d[q * 8 + i] = gb[(2 * q + h) * 72 + 8 * i + j];
}

// layout A -> layout C through the forward 3D transform
template <class T2, class T1>
__device__ __forceinline__ void forward3_16(float (&d)[32], float *gb, int h, int j, unsigned gm) {
#pragma unroll
    for (int q = 0; q < 4; ++q) T2::fwd(&d[q * 8]);
    move_tr(d, gb, h, j, gm);
#pragma unroll
    for (int q = 0; q < 4; ++q) T2::fwd(&d[q * 8]);
    move_bc(d, gb, h, j, gm);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        float v[8];
#pragma unroll
        for (int p = 0; p < 8; ++p) v[p] = d[p * 4 + t];
        T1::fwd(v);
#pragma unroll
        for (int p = 0; p < 8; ++p) d[p * 4 + t] = v[p];
    }
}

// layout D (after the shrinkage) -> layout F through the rest of the inverse 3D
// transform: vertical, horizontal, then across patches
template <class T2, class T1>
__device__ __forceinline__ void inverse3_16(float (&d)[32], float *gb, int h, int j, unsigned gm) {
#pragma unroll
    for (int q = 0; q < 4; ++q) T2::inv(&d[q * 8]);
    move_tr(d, gb, h, j, gm);
#pragma unroll
    for (int q = 0; q < 4; ++q) T2::inv(&d[q * 8]);
    move_bc(d, gb, h, j, gm);
#pragma unroll
    for (int t = 0; t < 4; ++t) {
        float v[8];
#pragma unroll
        for (int p = 0; p < 8; ++p) v[p] = d[p * 4 + t];
        T1::inv(v);
#pragma unroll
        for (int p = 0; p < 8; ++p) d[p * 4 + t] = v[p];
    }
}

// the lane's four patches 2q + h, column j, into layout A
__device__ __forceinline__ void gather16(float (&d)[32], const float *plane, const FilterArgs &a, long long grp,
                                         int h, int j) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int2 v = a.list[grp * 8 + 2 * q + h];
        const float *s = plane + ((unsigned)v.y >> 24) * a.frame_stride + (long long)(v.y & 0xffffff) * a.pitch + v.x + j;
#pragma unroll
        for (int i = 0; i < 8; ++i) d[q * 8 + i] = __ldg(s + i * a.pitch);
    }
}

// Groups g0 + threadIdx.x / 16 (16 lanes each) of one entry; tbuf: kFilterWarps * 2 *
// kGroupBuf floats, cbuf (Wiener): (blockDim.x / 16) * kCoeffBuf floats.
template <bool FINAL, int T2D, int T1D>
__device__ __forceinline__ void filter16_groups(const FilterArgs &a, long long g0, float *tbuf, float *cbuf) {
    using T2 = typename TransformOf<T2D>::type;
    using T1 = typename TransformOf<T1D>::type;
    const int lane = threadIdx.x & 31;
    const int j = lane & 7, h = (lane >> 3) & 1, gw = lane >> 4;
    const unsigned gm = 0xffffu << (lane & 16);
    const long long grp = g0 + (threadIdx.x >> 4);
    if (grp >= a.nblocks) return;
    float *gb = tbuf + ((threadIdx.x >> 5) * 2 + gw) * kGroupBuf;
    float *cb = cbuf + (threadIdx.x >> 4) * kCoeffBuf;
    const float E = a.extractor;

    for (int pl = 0; pl < a.nplanes; ++pl) {
        const float sigma = pl == 0 ? a.sigma[0] : (pl == 1 ? a.sigma[1] : a.sigma[2]);
        if (a.chroma && sigma < ZB_FLT_EPS) continue;
        float d[32];
        float k = 0.0f;
        if constexpr (FINAL) {
            // Wiener coefficients r^2 / (r^2 + sigma^2) of the basic estimate's spectrum (the
            // reference rounds r^2 once and adds sigma^2 without FMA); the weight's sum of
            // squared coefficients (after the shrinkage below) is accumulated by FMA over
            // spectrum and row for column j in the reference's order: every lane runs the full
            // chain of its column.  The basic estimate and the noisy patches share one copy of
            // the forward transform's code.
            const float s2 = sigma * sigma;
#pragma unroll 1
            for (int pass = 0; pass < 2; ++pass) {
                gather16(d, a.src + (pass ? a.clip_stride : 0) + pl * a.plane_stride, a, grp, h, j);
                forward3_16<T2, T1>(d, gb, h, j, gm);
                if (pass) break;
#pragma unroll
                for (int p = 0; p < 8; ++p)
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        const float rv = d[p * 4 + t];
                        const float r2 = __fmul_rn(rv, rv);
                        float coeff = r2 / __fadd_rn(r2, s2);
                        if (p == 0 && t == 0 && h == 0 && j == 0) coeff = 1.0f;
                        cb[p * 72 + (2 * t + h) * 8 + j] = coeff;
                    }
                __syncwarp(gm);
            }
        } else {
            gather16(d, a.src + pl * a.plane_stride, a, grp, h, j);
            forward3_16<T2, T1>(d, gb, h, j, gm);
        }
        // shrinkage in layout D, right before the vertical inverse: d[q * 8 + i] is
        // spectrum 2q + h, row i, column j
        move_cd(d, gb, h, j, gm);
        if constexpr (!FINAL) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float val = d[q * 8 + i];
                    const float thr = (q == 0 && i == 0 && h == 0 && j == 0) ? 0.0f : sigma;
                    const float flag = fabsf(val) >= thr;
                    k += flag;
                    d[q * 8 + i] = flag ? (val * (1.0f / 4096.0f)) : 0.0f;
                }
            // kept-coefficient count: integer-valued, exact in any order
            k += __shfl_xor_sync(gm, k, 1, 16);
            k += __shfl_xor_sync(gm, k, 2, 16);
            k += __shfl_xor_sync(gm, k, 4, 16);
            k += __shfl_xor_sync(gm, k, 8, 16);
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    float val = d[q * 8 + i];
                    val *= cb[(2 * q + h) * 72 + i * 8 + j];
                    d[q * 8 + i] = val * (1.0f / 4096.0f);
                }
            // the weight's chain, here so that it can overlap the vertical inverse transforms
            // (it only reads the coefficient buffer)
#pragma unroll 8
            for (int p = 0; p < 8; ++p)
#pragma unroll
                for (int r = 0; r < 8; ++r) {
                    const float c = cb[p * 72 + r * 8 + j];
                    k = __fmaf_rn(c, c, k);
                }
            k += __shfl_xor_sync(gm, k, 1, 8);
            k += __shfl_xor_sync(gm, k, 2, 8);
            k += __shfl_xor_sync(gm, k, 4, 8);
        }
        const float w = 1.0f / k;
        inverse3_16<T2, T1>(d, gb, h, j, gm);

        unsigned long long *num = a.num + pl * a.acc_plane_stride;
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            const int2 v = a.list[grp * 8 + p];
            unsigned long long *q = num + ((unsigned)v.y >> 24) * a.acc_frame_stride +
                                    (long long)(v.y & 0xffffff) * a.pitch + v.x + j;
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const float val = __fmaf_rn(w, d[p * 4 + t], E) - E;
                atomicAdd(q + (2 * t + h) * a.pitch, to_fix(val));
            }
        }
        if (h == 0) {
            // lane j books the weight of patch j once, at its origin
            const float wq = (w + E) - E;
            const int2 v = a.list[grp * 8 + j];
            atomicAdd(a.den + pl * a.acc_plane_stride + ((unsigned)v.y >> 24) * a.acc_frame_stride +
                          (long long)(v.y & 0xffffff) * a.pitch + v.x,
                      to_fix(wq));
        }
        __syncwarp(gm);  // the coefficient buffer is rewritten by the next plane
    }
}

template <bool FINAL, int T2D, int T1D>
__global__ void __launch_bounds__(kFilterWarps * 32) zb_filter16(FilterArgs a) {
    __shared__ float tbuf[kFilterWarps * 2 * kGroupBuf];
    // Wiener: the group's 512 coefficients at [spectrum * 72 + row * 8 + column]
    extern __shared__ float cbuf[];
    filter16_groups<FINAL, T2D, T1D>(a, (long long)blockIdx.x * (blockDim.x >> 4), tbuf, cbuf);
}

// ---------------------------------------------------------------------------
// Finish: fixed point -> float.  The weight at a pixel is the 8x8 box sum of the
// origin weights whose patch covers it.  mode 0 writes num/den (radius 0,
// src/bm3d.cu:898-922, IEEE division); mode 1 writes the stacked accumulator
// planes [plane][t][2][h][pitch] of the temporal path (src/bm3d.zig:1224-1231).
// ---------------------------------------------------------------------------
struct FinishArgs {
    const unsigned long long *num, *den;
    long long acc_plane_stride, acc_frame_stride;
    int w, h, pitch;
    int tw;
    unsigned proc_mask;       // planes written (bit p)
    float *dst;               // mode 0: [planes][h][dst_pitch]; mode 1: stacked
    int dst_pitch;
    long long dst_plane_stride;
    int mode;
};

// One CTA per 32 x 32 output pixels of one plane (and frame slot): the 39 x 39 tile of
// origin weights that their 8x8 boxes cover is read once into shared memory, summed along
// rows (8 wide), then each thread slides an 8-row sum down its column for 4 pixels.  The
// sums are int64, exact in any order.
constexpr int kFinishRows = 32;

__global__ void __launch_bounds__(256) zb_finish(FinishArgs a) {
    constexpr int TR = kFinishRows + 7, TC = 32 + 7;
    __shared__ long long t[TR][TC + 1];
    __shared__ long long hs[TR][32];
    const int plane = blockIdx.z / a.tw, slot = blockIdx.z - plane * a.tw;
    if (!((a.proc_mask >> plane) & 1)) return;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * kFinishRows;
    const long long base = plane * a.acc_plane_stride + slot * a.acc_frame_stride;
    const unsigned long long *den = a.den + base;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    constexpr int PER = kFinishRows / 8;  // output rows per thread
    const int x = x0 + threadIdx.x;
    const int ry = threadIdx.y * PER;     // first tile row of this thread's pixels
    long long ns[PER];                    // this thread's numerators, loaded before the tile
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int y = y0 + ry + i;
        ns[i] = (x < a.w && y < a.h) ? (long long)a.num[base + (long long)y * a.pitch + x] : 0;
    }
    for (int i = tid; i < TR * TC; i += 256) {
        const int r = i / TC, c = i - r * TC;
        const int gy = y0 - 7 + r, gx = x0 - 7 + c;
        t[r][c] = (gy >= 0 && gy < a.h && gx >= 0 && gx < a.w) ? (long long)den[(long long)gy * a.pitch + gx] : 0;
    }
    __syncthreads();
    for (int i = tid; i < TR * 32; i += 256) {
        const int r = i >> 5, c = i & 31;
        long long s = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) s += t[r][c + k];
        hs[r][c] = s;
    }
    __syncthreads();
    if (x >= a.w) return;
    long long ds = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) ds += hs[ry + k][threadIdx.x];
#pragma unroll
    for (int i = 0; i < PER; ++i) {
        const int y = y0 + ry + i;
        if (y >= a.h) return;
        if (i > 0) ds += hs[ry + i + 7][threadIdx.x] - hs[ry + i - 1][threadIdx.x];
        const float nf = __ll2float_rn(ns[i]) * kFixInv;
        const float df = __ll2float_rn(ds) * kFixInv;
        if (a.mode == 0) {
            a.dst[plane * a.dst_plane_stride + (long long)y * a.dst_pitch + x] = __fdiv_rn(nf, df);
        } else {
            float *o = a.dst + plane * a.dst_plane_stride + (long long)slot * 2 * a.h * a.dst_pitch;
            o[(long long)y * a.dst_pitch + x] = nf;
            o[(long long)(a.h + y) * a.dst_pitch + x] = df;
        }
    }
}

// ---------------------------------------------------------------------------
// Batch: one persistent launch over a work list of several plane entries (of any sizes)
// that share the filter kind.  CTAs of 128 threads take items in order from a global
// counter: every match tile of every entry, then every filter chunk.  A filter chunk of an
// entry waits until all of that entry's match tiles are done (a bounded spin on its
// counter; on timeout the chunk is skipped and the status word set).  Match items never
// wait, and every item a CTA waits on was taken earlier by a running CTA, so the list
// always drains.  Lists are written and read within the launch with ordinary loads and a
// fence on both sides of the counter.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int batch_entry_of(const BatchArgs &b, long long item, bool filter) {
    int lo = 0, hi = b.nentries - 1;  // last entry whose first item <= item
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        const long long f = filter ? b.entries[mid].first_filter : b.entries[mid].first_match;
        if (f <= item) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// PHASE 0: the whole list in one launch; 1: match items only; 2: filter items only (the
// items of the other kind are skipped, so two stream-ordered launches cover the list, each
// kernel with the register budget of its own kind of work).
// PHASE 1: the match tiles (kBatchMatchRows warps per CTA); PHASE 2: the filter chunks
// (4 warps per CTA).  Each phase is one persistent launch with its own register budget.
template <bool FINAL, int T2D, int T1D, int PHASE>
__global__ void __launch_bounds__(PHASE == 1 ? kBatchMatchRows * 32 : 128) zb_batch(BatchArgs b) {
    extern __shared__ __align__(16) float dyn[];  // matching tile, or the Wiener coefficient buffer
    __shared__ float tbuf[PHASE == 1 ? 1 : kFilterWarps * 2 * kGroupBuf];
    __shared__ long long s_item;
    __shared__ int s_ok;
    static_assert(PHASE == 1 || PHASE == 2, "match phase or filter phase");
    const long long first = PHASE == 2 ? b.match_total : 0;
    const long long last = PHASE == 1 ? b.match_total : b.items_total;
    for (;;) {
        __syncthreads();  // the previous item is done with shared memory
        if (threadIdx.x == 0) s_item = first + (long long)atomicAdd(b.next, 1ull);
        __syncthreads();
        const long long item = s_item;
        if (item >= last) break;
        if constexpr (PHASE == 1) {
            const int e = batch_entry_of(b, item, false);
            const BatchEntry &E = b.entries[e];
            const int local = (int)(item - E.first_match);
            const int bx = local % E.tiles_x, by = local / E.tiles_x;
            if (E.m.bs == 4)
                match_tiled2_tile<true, 4>(E.m, bx, by, dyn);
            else
                match_tiled2_tile<false, 8>(E.m, bx, by, dyn);
            __threadfence();  // each thread's list stores before the tile's count
            __syncthreads();
            if (threadIdx.x == 0) atomicAdd(&b.match_done[e], 1u);
        } else {
            const int e = batch_entry_of(b, item, true);
            const BatchEntry &E = b.entries[e];
            if (threadIdx.x == 0) {
                const unsigned need = (unsigned)E.match_items + ((b.unsatisfiable && e == 0) ? 1u : 0u);
                volatile unsigned *done = b.match_done + e;
                int ok = 0;
                for (unsigned i = 0; i < b.wait_polls; ++i) {
                    if (*done >= need) {
                        ok = 1;
                        break;
                    }
                    __nanosleep(100);
                }
                if (!ok) atomicCAS(b.status, 0, 1);
                s_ok = ok;
            }
            __syncthreads();
            if (!s_ok) continue;  // this chunk is left out; the status tells the host
            __threadfence();      // the count before the lists, for every reading thread
            const long long g0 = (item - E.first_filter) * kBatchGroups;
#pragma unroll 1
            for (int g = 0; g < kBatchGroups; g += 128 / 16)
                filter16_groups<FINAL, T2D, T1D>(E.f, g0 + g, tbuf, dyn);
        }
    }
}

// ---------------------------------------------------------------------------
// Host-side launchers.
// ---------------------------------------------------------------------------
size_t match_tile_bytes(const MatchArgs &a, int rows_per_cta);

template <int M, bool SHARED, int BS>
static cudaError_t launch_tiled_t(const MatchArgs &a, int rows_per_cta, cudaStream_t st) {
    constexpr int NBW = SHARED ? 31 : 16;
    const int gx = (a.nbx_al + NBW - 1) / NBW;
    const int gy = (a.nby + rows_per_cta - 1) / rows_per_cta;
    const size_t smem = match_tile_bytes(a, rows_per_cta);
    auto k = zb_match_tiled<M, SHARED, BS>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<dim3(gx, gy), rows_per_cta * 32, smem, st>>>(a);
    return cudaGetLastError();
}

// packed FP32x2 SSD kernel: two pair-interleaved copies of the tile (swizzled pair rows)
static size_t match_tile2_bytes(const MatchArgs &a, int rows_per_cta) {
    return (size_t)((rows_per_cta - 1) * a.bs + 2 * a.range + 8) * 8 * tile2_g(a.tile_pitch, tile2_fixed(a.chunks)) *
           sizeof(float);
}

template <bool SHARED, int BS>
static cudaError_t launch_tiled2_t(const MatchArgs &a, int rows_per_cta, cudaStream_t st) {
    constexpr int NBW = SHARED ? 31 : 16;
    const int gx = (a.nbx_al + NBW - 1) / NBW;
    const int gy = (a.nby + rows_per_cta - 1) / rows_per_cta;
    const size_t smem = match_tile2_bytes(a, rows_per_cta);
    auto k = zb_match_tiled2<SHARED, BS>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<dim3(gx, gy), rows_per_cta * 32, smem, st>>>(a);
    return cudaGetLastError();
}

template <int M>
static cudaError_t launch_tiled_m(const MatchArgs &a, int rows_per_cta, cudaStream_t st) {
    if constexpr (M == M_SSD) {
        // SSD at block_step 4 / 8: the packed FP32x2 kernel whenever its two tiles fit
        if (match_tile2_bytes(a, rows_per_cta) <= 200 * 1024)
            return a.bs == 8 ? launch_tiled2_t<false, 8>(a, rows_per_cta, st)
                             : launch_tiled2_t<true, 4>(a, rows_per_cta, st);
    }
    if (a.bs == 8) return launch_tiled_t<M, false, 8>(a, rows_per_cta, st);
    if constexpr (Shareable<M>::value) return launch_tiled_t<M, true, 4>(a, rows_per_cta, st);
    return launch_tiled_t<M, false, 4>(a, rows_per_cta, st);
}

template <int M>
static cudaError_t launch_global_m(const MatchArgs &a, cudaStream_t st) {
    // listed blocks (gen_mode 2): the count is on the device, so size for every block
    const long long threads = (long long)a.nby * a.nbx * 2;
    zb_match_global<M><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a);
    return cudaGetLastError();
}

template <int M>
static cudaError_t launch_column_m(const MatchArgs &a, cudaStream_t st) {
    zb_match_column<M><<<(unsigned)((a.nby + 3) / 4), 128, 0, st>>>(a);
    return cudaGetLastError();
}

template <int M>
static cudaError_t launch_temporal_m(const MatchArgs &a, cudaStream_t st) {
    const long long threads = (long long)a.nby * a.nbx * 2;
    if (a.ps_num <= 2)
        zb_match_temporal<M, 2><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a);
    else
        zb_match_temporal<M, 8><<<(unsigned)((threads + 127) / 128), 128, 0, st>>>(a);
    return cudaGetLastError();
}

// Shared-memory bytes the tiled kernel needs for `rows_per_cta` block rows.
size_t match_tile_bytes(const MatchArgs &a, int rows_per_cta) {
    return (size_t)((rows_per_cta - 1) * a.bs + 2 * a.range + 8) * a.tile_pitch * sizeof(float);
}

bool tc_eligible(const MatchArgs &a);                          // zb3d_match_tc.cu
cudaError_t launch_match_tc(const MatchArgs &a, cudaStream_t st);

// The FP32 scan of the blocks the tensor-core kernel listed (SSD, radius 0).
cudaError_t launch_tc_fallback(MatchArgs a, cudaStream_t st) {
    a.self_incl = a.radius == 0;
    a.gen_mode = 2;
    return launch_global_m<M_SSD>(a, st);
}

cudaError_t launch_match(MatchArgs a, int metric, int rows_per_cta, bool use_tiled, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    const bool tiled = use_tiled && (a.bs == 4 || a.bs == 8);
    a.self_incl = a.radius == 0;
    if (metric == M_SSD && a.tc_ws != nullptr && tc_eligible(a)) {
        // tensor-core bound + exact re-rank; the blocks it lists get the FP32 scan
        if ((e = launch_match_tc(a, st)) != cudaSuccess) return e;
        a.gen_mode = 2;
        if ((e = launch_global_m<M_SSD>(a, st)) != cudaSuccess) return e;
        goto temporal;
    }
    if (tiled) {
        a.chunks = (2 * a.range + 1 + 3) / 4;
        a.tile_pitch = 128 + 4 * a.chunks;
        switch (metric) {
        case M_SSD: e = launch_tiled_m<M_SSD>(a, rows_per_cta, st); break;
        case M_SAD: e = launch_tiled_m<M_SAD>(a, rows_per_cta, st); break;
        case M_ZSSD: e = launch_tiled_m<M_ZSSD>(a, rows_per_cta, st); break;
        case M_ZSAD: e = launch_tiled_m<M_ZSAD>(a, rows_per_cta, st); break;
        default: e = launch_tiled_m<M_SSD_NORM>(a, rows_per_cta, st); break;
        }
        if (e != cudaSuccess) return e;
        if (a.nbx_al == a.nbx) goto temporal;
        switch (metric) {  // the clamped last column
        case M_SSD: e = launch_column_m<M_SSD>(a, st); break;
        case M_SAD: e = launch_column_m<M_SAD>(a, st); break;
        case M_ZSSD: e = launch_column_m<M_ZSSD>(a, st); break;
        case M_ZSAD: e = launch_column_m<M_ZSAD>(a, st); break;
        default: e = launch_column_m<M_SSD_NORM>(a, st); break;
        }
        if (e != cudaSuccess) return e;
        goto temporal;
    }
    a.gen_mode = 0;
    switch (metric) {
    case M_SSD: e = launch_global_m<M_SSD>(a, st); break;
    case M_SAD: e = launch_global_m<M_SAD>(a, st); break;
    case M_ZSSD: e = launch_global_m<M_ZSSD>(a, st); break;
    case M_ZSAD: e = launch_global_m<M_ZSAD>(a, st); break;
    default: e = launch_global_m<M_SSD_NORM>(a, st); break;
    }
    if (e != cudaSuccess) return e;
temporal:
    if (a.radius > 0) {
        switch (metric) {
        case M_SSD: e = launch_temporal_m<M_SSD>(a, st); break;
        case M_SAD: e = launch_temporal_m<M_SAD>(a, st); break;
        case M_ZSSD: e = launch_temporal_m<M_ZSSD>(a, st); break;
        case M_ZSAD: e = launch_temporal_m<M_ZSAD>(a, st); break;
        default: e = launch_temporal_m<M_SSD_NORM>(a, st); break;
        }
    }
    return e;
}

template <bool FINAL, int T2D, int T1D>
static cudaError_t launch_filter_t(const FilterArgs &a, cudaStream_t st) {
    const long long threads = (long long)a.nblocks * 16;
    const int tpb = kFilterWarps * 32;
    const int dyn = FINAL ? (tpb / 16) * kCoeffBuf * (int)sizeof(float) : 0;  // Wiener coefficient buffer
    auto k = zb_filter16<FINAL, T2D, T1D>;
    if (FINAL) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, dyn);
        if (e != cudaSuccess) return e;
    }
    k<<<(unsigned)((threads + tpb - 1) / tpb), tpb, dyn, st>>>(a);
    return cudaGetLastError();
}

template <bool FINAL, int T2D>
static cudaError_t launch_filter_f2(const FilterArgs &a, int t1d, cudaStream_t st) {
    switch (t1d) {
    case T_DCT: return launch_filter_t<FINAL, T2D, T_DCT>(a, st);
    case T_HAAR: return launch_filter_t<FINAL, T2D, T_HAAR>(a, st);
    case T_WHT: return launch_filter_t<FINAL, T2D, T_WHT>(a, st);
    default: return launch_filter_t<FINAL, T2D, T_BIOR15>(a, st);
    }
}

template <bool FINAL>
static cudaError_t launch_filter_f(const FilterArgs &a, int t2d, int t1d, cudaStream_t st) {
    switch (t2d) {
    case T_DCT: return launch_filter_f2<FINAL, T_DCT>(a, t1d, st);
    case T_HAAR: return launch_filter_f2<FINAL, T_HAAR>(a, t1d, st);
    case T_WHT: return launch_filter_f2<FINAL, T_WHT>(a, t1d, st);
    default: return launch_filter_f2<FINAL, T_BIOR15>(a, t1d, st);
    }
}

cudaError_t launch_filter(const FilterArgs &a, bool final_, int t2d, int t1d, cudaStream_t st) {
    return final_ ? launch_filter_f<true>(a, t2d, t1d, st) : launch_filter_f<false>(a, t2d, t1d, st);
}

cudaError_t launch_finish(const unsigned long long *num, const unsigned long long *den, long long acc_plane_stride,
                          long long acc_frame_stride, int w, int h, int pitch, int nplanes, int tw,
                          unsigned proc_mask, float *dst, int dst_pitch, long long dst_plane_stride, int mode,
                          cudaStream_t st) {
    FinishArgs a;
    a.num = num;
    a.den = den;
    a.acc_plane_stride = acc_plane_stride;
    a.acc_frame_stride = acc_frame_stride;
    a.w = w;
    a.h = h;
    a.pitch = pitch;
    a.tw = mode == 0 ? 1 : tw;
    a.proc_mask = proc_mask;
    a.dst = dst;
    a.dst_pitch = dst_pitch;
    a.dst_plane_stride = dst_plane_stride;
    a.mode = mode;
    dim3 grid((w + 31) / 32, (h + kFinishRows - 1) / kFinishRows, nplanes * a.tw);
    zb_finish<<<grid, dim3(32, 8), 0, st>>>(a);
    return cudaGetLastError();
}

// The clamped last block column of an entry (x = w - 8), which the tiled kernels leave out.
cudaError_t launch_clamped_column(MatchArgs a, cudaStream_t st) {
    a.self_incl = a.radius == 0;
    return launch_column_m<M_SSD>(a, st);
}

size_t match_tile2_bytes_rows(const MatchArgs &a, int rows_per_cta) { return match_tile2_bytes(a, rows_per_cta); }

// Bytes of dynamic shared memory a batch entry needs: its matching tile (kBatchMatchRows
// block rows), and the Wiener coefficient buffer of its filter chunks.
size_t batch_match_smem(const MatchArgs &m) { return match_tile2_bytes(m, kBatchMatchRows); }
size_t batch_filter_smem(bool final_) { return final_ ? (size_t)(128 / 16) * kCoeffBuf * sizeof(float) : 0; }

template <class K>
static cudaError_t launch_batch_k(K k, const BatchArgs &b, int threads, size_t smem, cudaStream_t st) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k, threads, smem) != cudaSuccess || per < 1) per = 1;
    k<<<sms * per, threads, smem, st>>>(b);
    return cudaGetLastError();
}

// The batch kernels for the filter kind (final, t2d, t1d); only the DCT in both dimensions
// is built in (other kinds run entry by entry).  The match items and the filter items run as
// two stream-ordered persistent launches (b.next must point at two counters); the filter
// chunks still check, bounded, that their entry's matching is complete.
// match_smem / filter_smem: dynamic shared memory of each kind of item.
cudaError_t launch_batch(BatchArgs b, bool final_, int t2d, int t1d, size_t match_smem, size_t filter_smem,
                         cudaStream_t st) {
    if (t2d != T_DCT || t1d != T_DCT) return cudaErrorNotSupported;
    cudaError_t e = launch_batch_k(final_ ? zb_batch<true, T_DCT, T_DCT, 1> : zb_batch<false, T_DCT, T_DCT, 1>, b,
                                   kBatchMatchRows * 32, match_smem, st);
    if (e != cudaSuccess) return e;
    b.next += 1;
    return launch_batch_k(final_ ? zb_batch<true, T_DCT, T_DCT, 2> : zb_batch<false, T_DCT, T_DCT, 2>, b, 128,
                          filter_smem > 0 ? filter_smem : 16, st);
}

}  // namespace zb
