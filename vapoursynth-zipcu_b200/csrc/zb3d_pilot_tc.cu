// Learned pilot: inference convolution on the 5th-generation tensor cores.
//
// y = conv3x3(x) + bias (ReLU), BF16 operands in shared memory, FP32 accumulators
// in tensor memory (tcgen05.mma kind::f16, M = 128 pixels of one image row).
//
// Activations use the channel-blocked layout [n][C / 8][h][w][8] (BF16): one
// channel block of an image row is a contiguous run of 16-byte pixels.
//
// Row-stationary implicit GEMM, no im2col.  A CTA walks down strips of 128
// columns; TMA stages each input row once (130 pixels with the halo, zero-filled
// outside the image) into a ring of row slots laid out [channel block][pixel][8].
// When the width is a multiple of 8 a box is 18 lines of 128 bytes (8-pixel
// groups from x0 - 8, so the halo pixel x0 - 1 sits at slot pixel 7); otherwise
// 130 lines of one 16-byte pixel from x0 - 1, which keeps the zero fill exact at a
// ragged right edge.  In that layout the pixels x + kx - 1 of channel block 2 s form the canonical
// no-swizzle K-major A operand (8-pixel core matrices 128 bytes apart = SBO, the
// two 8-channel halves one channel block apart = LBO).  Input row r feeds output
// rows r + 1, r and r - 1 through the kernel rows ky = 0, 1, 2, so B stacks the
// three ky weight blocks (N = 3 COUT) and one MMA per (kx, K-step) adds row r's
// share into the accumulators of all three output rows at once: each staged row
// is read 3 x CIN / 16 times as an operand instead of 9 x CIN / 16, and is free
// again as soon as its own MMAs complete.  For that the accumulators of
// consecutive output rows sit next to each other in tensor memory, in descending
// order (a ring of K slots; where the ring wraps, the MMA splits in two).  The
// first contribution to an accumulator (kx = 0, K-step 0 of the row that first
// touches it) is a separate MMA that overwrites instead of adding, so nothing
// has to clear tensor memory.
// A run of n output rows takes n + 2 input rows and n + 4 accumulators (the 4 at
// its ends only collect halo contributions and are discarded).
//
// Four CTAs per SM for layers of up to 32 channels, two with 48, each owning a
// contiguous range of tiles in (image, strip, row) order (balanced to one tile).  The
// row ring fills the shared memory the weights leave (up to 16 slots).
//
// Roles (192 or 384 threads): warp 0 lane 0 issues the TMA row loads, warp 1 lane 0
// issues the MMAs, warp 2 also owns the tensor-memory allocation, and one quad of
// epilogue warps (2-5) or two (4-7 and 8-11) drain the accumulators, warp w on the
// 32-lane quarter w % 4 of tensor memory; two quads take the accumulators in turn,
// so that one quad's tensor-memory loads and stores overlap the other's: bias, ReLU, BF16 store
// (16 bytes per channel block, 512 contiguous bytes per warp), or for the last
// layer channel 0 plus the residual in FP32.  mbarriers link the roles; every wait
// is bounded, and a timeout sets the status word and ends every role early.
//
// Same arithmetic as the mma.sync kernel in zb3d_pilot.cu (BF16 products, FP32
// sums, bias then ReLU then one BF16 rounding); only the summation order differs.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "zb3d_tcgen05.cuh"

namespace zb {
namespace pilot_tc {

using namespace tc05;

constexpr int TILE = 128;                // output pixels per tile (MMA M)
constexpr int BOX_PIX = 130;             // TMA box of 130 single pixels (any width)
constexpr int BOX_GROUPS = 18;           // TMA box of 18 groups of 8 pixels (width a multiple of 8)
constexpr int CB_BYTES = BOX_GROUPS * 128;  // one channel block of a staged row (2304 bytes)
constexpr int MAX_RING = 16;             // staged input row slots, at most
constexpr int MAX_CTAS_PER_SM = 4;       // independent pipelines per SM, at most
constexpr unsigned WAIT_LIMIT = 1u << 20;  // try_wait rounds on an mbarrier before giving up (about a second)

struct Args {
    const __nv_bfloat16 *wgt;  // [cout][9][cin]
    const float *bias;         // [cout]
    __nv_bfloat16 *y;          // [n][cout / 8][h][w][8] or null
    float *y0;                 // [n][h][y0_pitch] (images y0_stride apart) or null: channel 0 (+ resid) in FP32
    const float *resid;        // [n][h][resid_pitch] (images resid_stride apart) or null
    long long y0_stride, resid_stride;
    int y0_pitch, resid_pitch; // floats between rows (>= w)
    int n, h, w, relu;
    int strips;                // ceil(w / 128)
    int grouped;               // boxes of 8-pixel groups (w % 8 == 0), else of single pixels
    int *status;               // set non-zero when a wait timed out (may be null)
};

template <int CIN, int COUT>
struct Shape {
    static_assert(CIN % 16 == 0 && COUT % 16 == 0 && 3 * COUT <= 256, "unsupported layer shape");
    static constexpr int CB = CIN / 8;
    // Pipelines per SM: 4 for layers up to 32 channels, 2 with 48 (their weights and rows
    // need the shared memory).  With 4, a CTA is 6 warps (producer, MMA, one epilogue quad
    // in warps 2-5) with 128 tensor-memory columns; with 2, 12 warps (two epilogue quads in
    // warps 4-11) with 256 columns.
    static constexpr int CTAS = (CIN <= 32 && COUT <= 32) ? 4 : 2;
    static constexpr int EPI_GROUPS = CTAS == 4 ? 1 : 2;  // epilogue warp quads, taking accumulators in turn
    static constexpr int EPI_W0 = CTAS == 4 ? 2 : 4;       // first epilogue warp
    static constexpr int THREADS = 32 * (EPI_W0 + 4 * EPI_GROUPS);
    static constexpr int TMEM_COLS = 512 / CTAS;
    static constexpr int SMEM_BUDGET = CTAS == 4 ? 54 * 1024 : 112 * 1024;  // ring + weights, per CTA
    static constexpr int NACC = TMEM_COLS / COUT;  // accumulator slots
    static_assert(NACC >= 4, "accumulator ring too small");
    static constexpr int KSTEPS = CIN / 16;
    static constexpr int ROW_BYTES = CB * CB_BYTES;
    static constexpr int W_BYTES = 9 * CB * COUT * 16;
    static constexpr int RING_FIT = (SMEM_BUDGET - W_BYTES) / ROW_BYTES;
    static constexpr int RING = RING_FIT < MAX_RING ? RING_FIT : MAX_RING;
    static_assert(RING >= 4, "row ring too small");
    static constexpr int OFF_W = RING * ROW_BYTES;
    static constexpr int OFF_BAR = OFF_W + W_BYTES;
    static constexpr int NBAR = 2 * RING + 2 * NACC + 1;  // row_full, row_free, acc_full, acc_empty, drain
    static constexpr int OFF_MISC = OFF_BAR + NBAR * 8;
    static constexpr int OFF_BIAS = OFF_MISC + 16;    // after the tensor-memory address and abort flag
    static constexpr int SMEM = OFF_BIAS + COUT * 4 + 128;  // + alignment slack
    static_assert(CTAS * (SMEM + 1024) <= 228 * 1024, "CTAs per SM exceed the shared memory");
    static constexpr int B_ROWS = 3 * COUT;          // stacked ky blocks of one (kx, channel block)
};

// kind::f16 instruction descriptor: FP32 accumulator (bit 4), BF16 A (bits 7-9 = 1) and
// B (bits 10-12 = 1), both K-major, N >> 3 at bits 17-22, M >> 4 at bits 24-28
__host__ __device__ constexpr uint32_t idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(TILE >> 4) << 24);
}

// Shared-memory matrix descriptor, K-major without swizzle (layout type 0):
// start address, LBO (the two 8-element K halves) and SBO (8-row groups) in
// 16-byte units, version 1 at bits 46-47.
__device__ __forceinline__ uint64_t desc_k(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

// Waits for phase `parity` of an mbarrier.  Gives up when another role has
// aborted, or after WAIT_LIMIT tries: then it raises the abort flag and records
// `code` in the status word.
__device__ __forceinline__ bool wait_bar(uint32_t mbar, uint32_t parity, volatile int *abort_flag, int *status,
                                         int code) {
    for (unsigned i = 0; i < WAIT_LIMIT; ++i) {
        if (mbar_try(mbar, parity)) return true;
        if (*abort_flag) return false;
    }
    *abort_flag = 1;
    if (status) atomicExch(status, code);
    return false;
}

// one TMA box (130 pixels, or 18 groups of 8 pixels, from x) of row y of channel-block
// plane `plane` (= image * CIN / 8 + block)
__device__ __forceinline__ void tma_row(uint32_t dst, const CUtensorMap *map, int c, int x, int y, int plane,
                                        uint32_t mbar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
        "%5}], [%6];\n" ::"r"(dst),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c), "r"(x), "r"(y), "r"(plane), "r"(mbar)
        : "memory");
}

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    return (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(lo)) |
           ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(hi)) << 16);
}

// A maximal run of this CTA's tiles in one strip: output rows [ya, yb).
struct Seg {
    int img, x0, ya, yb;
};

// Tiles are numbered (image, strip, row); the CTA owns [t, t1).  Takes the next run.
__device__ __forceinline__ bool next_seg(const Args &p, long long &t, long long t1, Seg &k) {
    if (t >= t1) return false;
    const long long u = t / p.h;
    k.ya = (int)(t - u * p.h);
    k.img = (int)(u / p.strips);
    k.x0 = (int)(u - (long long)k.img * p.strips) * TILE;
    k.yb = (int)min((long long)p.h, k.ya + (t1 - t));
    t += k.yb - k.ya;
    return true;
}

template <int CIN, int COUT>
__global__ void __launch_bounds__(Shape<CIN, COUT>::THREADS, Shape<CIN, COUT>::CTAS)
    conv3x3_tc(const __grid_constant__ CUtensorMap xmap, Args p) {
    using S = Shape<CIN, COUT>;
    constexpr int RING = S::RING, NACC = S::NACC;
    extern __shared__ uint8_t smraw[];
    const uint32_t raw = smem_u32(smraw);
    const uint32_t pad = ((raw + 127u) & ~127u) - raw;
    uint8_t *sm = smraw + pad;
    const uint32_t sb = raw + pad;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t bar = sb + S::OFF_BAR;
    // barriers: row_full[RING], row_free[RING], acc_full[NACC], acc_empty[NACC], drain
    const uint32_t row_full = bar, row_free = bar + 8u * RING;
    const uint32_t acc_full = bar + 8u * (2 * RING), acc_empty = acc_full + 8u * NACC;
    const uint32_t drain = acc_empty + 8u * NACC;
    const long long tiles = (long long)p.n * p.strips * p.h;
    const long long t_begin = tiles * blockIdx.x / gridDim.x, t_end = tiles * (blockIdx.x + 1) / gridDim.x;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(sm + S::OFF_MISC);
    volatile int *abort_flag = reinterpret_cast<volatile int *>(sm + S::OFF_MISC + 4);
    // accumulator g (the CTA's running count) lives in slot NACC - 1 - g % NACC: the
    // slots of consecutive output rows descend, so rows r + 1, r, r - 1 are adjacent
    auto acc_slot = [](uint32_t g) { return (int)(NACC - 1 - g % NACC); };

    // weights as B operands [kx][channel block][ky][cout][8]: N = 3 COUT rows per (kx, block)
    for (int i = threadIdx.x; i < 9 * S::CB * COUT; i += S::THREADS) {
        const int co = i % COUT, r1 = i / COUT, ky = r1 % 3, r2 = r1 / 3, cb = r2 % S::CB, kx = r2 / S::CB;
        *reinterpret_cast<uint4 *>(sm + S::OFF_W + 16 * i) =
            __ldg(reinterpret_cast<const uint4 *>(p.wgt + ((size_t)co * 9 + ky * 3 + kx) * CIN + cb * 8));
    }
    float *sbias = reinterpret_cast<float *>(sm + S::OFF_BIAS);
    if (threadIdx.x < COUT) sbias[threadIdx.x] = p.bias ? __ldg(p.bias + threadIdx.x) : 0.0f;
    if (threadIdx.x == 0) {
        for (int s = 0; s < RING; ++s) {
            mbar_init(row_full + 8u * s, 1);
            mbar_init(row_free + 8u * s, 1);
        }
        for (int b = 0; b < NACC; ++b) {
            mbar_init(acc_full + 8u * b, 1);
            mbar_init(acc_empty + 8u * b, 4);
        }
        mbar_init(drain, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 2) tmem_alloc(smem_u32(tslot), S::TMEM_COLS);
    fence_async_smem();  // weights: generic stores -> MMA reads
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tmem = *tslot;

    if (warp == 0 && lane == 0) {
        // producer: input rows ya - 1 .. yb of every run, in order, into the ring
        uint32_t e = 0;
        bool ok = true;
        long long t = t_begin;
        Seg k;
        const uint32_t box_bytes = p.grouped ? CB_BYTES : BOX_PIX * 16;
        while (ok && next_seg(p, t, t_end, k)) {
            const int bx = p.grouped ? (k.x0 >> 3) - 1 : k.x0 - 1;  // first 8-pixel group / pixel of the box
            for (int r = k.ya - 1; r <= k.yb; ++r, ++e) {
                const int s = (int)(e % RING);
                if (e >= RING && !wait_bar(row_free + 8u * s, ((e / RING) - 1) & 1, abort_flag, p.status, 1)) {
                    ok = false;
                    break;
                }
                mbar_arrive_tx(row_full + 8u * s, S::CB * box_bytes);
                const uint32_t dst = sb + s * S::ROW_BYTES;
#pragma unroll
                for (int cb = 0; cb < S::CB; ++cb)
                    tma_row(dst + cb * CB_BYTES, &xmap, 0, bx, r, k.img * S::CB + cb, row_full + 8u * s);
            }
        }
        if (!ok) {
            // let the row loads already issued land before the CTA can end
            for (uint32_t q = e > RING ? e - RING : 0; q < e; ++q) {
                for (unsigned i = 0; i < WAIT_LIMIT && !mbar_try(row_full + 8u * (q % RING), (q / RING) & 1); ++i) {
                }
            }
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer: input row i of a run (global count e) adds into accumulators
        // g, g + 1, g + 2 (output rows r - 1, r, r + 1), g = run base + i
        // pixel x0 - 1 sits at slot pixel 7 (group boxes) or 0 (pixel boxes)
        const uint64_t a_desc0 = desc_k(sb + (p.grouped ? 7 * 16 : 0), CB_BYTES, 128);
        const uint64_t b_desc0 = desc_k(sb + S::OFF_W, S::B_ROWS * 16, 128);
        uint32_t e = 0, gbase = 0;
        bool ok = true;
        long long tt = t_begin;
        Seg k;
        while (ok && next_seg(p, tt, t_end, k)) {
            const int n = k.yb - k.ya;
            for (int i = 0; i <= n + 1 && ok; ++i, ++e) {
                const uint32_t g = gbase + (uint32_t)i;
                if (!wait_bar(row_full + 8u * (e % RING), (e / RING) & 1, abort_flag, p.status, 2)) {
                    ok = false;
                    break;
                }
                // accumulators touched for the first time: g, g + 1, g + 2 at the run's first row, else g + 2
                for (uint32_t q = (i == 0 ? g : g + 2); q <= g + 2; ++q)
                    if (q >= (uint32_t)NACC &&
                        !wait_bar(acc_empty + 8u * acc_slot(q), ((q / NACC) - 1) & 1, abort_flag, p.status, 3)) {
                        ok = false;
                        break;
                    }
                if (!ok) break;
                fence_after_sync();
                const uint64_t arow = a_desc0 + (uint64_t)((e % RING) * (S::ROW_BYTES >> 4));
                const int s0 = acc_slot(g);  // slot of output row r - 1 (ky = 2)
                // B rows ky * COUT .. of (kx, K-step): descriptor offsets in 16-byte units
                constexpr uint64_t KY1 = (COUT * 16) >> 4, KY2 = (2 * COUT * 16) >> 4;
                const uint32_t d0 = tmem + (uint32_t)(s0 * COUT);
#pragma unroll
                for (int kx = 0; kx < 3; ++kx)
#pragma unroll
                    for (int ks = 0; ks < S::KSTEPS; ++ks) {
                        const uint64_t ad = arow + (uint64_t)((2 * ks * CB_BYTES + kx * 16) >> 4);
                        const uint64_t bd = b_desc0 + (uint64_t)(((kx * S::CB + 2 * ks) * S::B_ROWS * 16) >> 4);
                        if (kx == 0 && ks == 0 && i > 0) {
                            // row r + 1's accumulator is fresh: its first product overwrites
                            const int s2 = s0 >= 2 ? s0 - 2 : s0 + NACC - 2;
                            mma_kind_f16(tmem + (uint32_t)(s2 * COUT), ad, bd, idesc_bf16(COUT), 0);
                            if (s0 >= 1) {  // slots s0 - 1, s0 = rows r, r - 1
                                mma_kind_f16(d0 - COUT, ad, bd + KY1, idesc_bf16(2 * COUT), 1);
                            } else {
                                mma_kind_f16(tmem + (uint32_t)((NACC - 1) * COUT), ad, bd + KY1, idesc_bf16(COUT), 1);
                                mma_kind_f16(tmem, ad, bd + KY2, idesc_bf16(COUT), 1);
                            }
                            continue;
                        }
                        // a run's first row: all three accumulators are fresh
                        const uint32_t acc = (kx == 0 && ks == 0) ? 0u : 1u;
                        if (s0 >= 2) {  // slots s0 - 2, s0 - 1, s0 = rows r + 1, r, r - 1: one MMA
                            mma_kind_f16(d0 - 2 * COUT, ad, bd, idesc_bf16(3 * COUT), acc);
                        } else if (s0 == 1) {  // slots 0, 1 = rows r, r - 1; slot NACC - 1 = row r + 1
                            mma_kind_f16(tmem, ad, bd + KY1, idesc_bf16(2 * COUT), acc);
                            mma_kind_f16(tmem + (uint32_t)((NACC - 1) * COUT), ad, bd, idesc_bf16(COUT), acc);
                        } else {  // slot 0 = row r - 1; slots NACC - 2, NACC - 1 = rows r + 1, r
                            mma_kind_f16(tmem, ad, bd + KY2, idesc_bf16(COUT), acc);
                            mma_kind_f16(tmem + (uint32_t)((NACC - 2) * COUT), ad, bd, idesc_bf16(2 * COUT), acc);
                        }
                    }
                mma_commit(row_free + 8u * (e % RING));  // the staged row is done
                mma_commit(acc_full + 8u * acc_slot(g));  // output row r - 1 is complete
                if (i == n + 1) {                         // the run's last two (halo) accumulators
                    mma_commit(acc_full + 8u * acc_slot(g + 1));
                    mma_commit(acc_full + 8u * acc_slot(g + 2));
                }
            }
            gbase += (uint32_t)(n + 4);
        }
        // every MMA issued has completed before the CTA ends
        mma_commit(drain);
        for (unsigned i = 0; i < WAIT_LIMIT && !mbar_try(drain, 0); ++i) {
        }
    } else if (warp >= S::EPI_W0) {
        // epilogue: warp w drains tensor-memory lanes 32 (w % 4) .. + 31 (pixels of the tile) of
        // the accumulators g with g % S::EPI_GROUPS == its quad
        const int q = warp & 3, grp = (warp - S::EPI_W0) >> 2;
        uint32_t g = 0;
        bool ok = true;
        long long tt = t_begin;
        Seg k;
        while (ok && next_seg(p, tt, t_end, k)) {
            const int n = k.yb - k.ya;
            // accumulator j of the run = output row ya - 2 + j; rows ya .. yb - 1 are real
            for (int j = 0; j < n + 4; ++j, ++g) {
                if ((int)(g % S::EPI_GROUPS) != grp) continue;
                const int slot = acc_slot(g);
                if (!wait_bar(acc_full + 8u * slot, (g / NACC) & 1, abort_flag, p.status, 4)) {
                    ok = false;
                    break;
                }
                fence_after_sync();
                const uint32_t ta = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(slot * COUT);
                const bool real = j >= 2 && j <= n + 1;
                float v[COUT];
                if (real) {
#pragma unroll
                    for (int cc = 0; cc < COUT; cc += 16) tmem_ld16(ta + cc, v + cc);
                    tmem_wait_ld();
                }
                fence_before_sync();
                __syncwarp();
                if (lane == 0) mbar_arrive(acc_empty + 8u * slot);
                const int x = k.x0 + q * 32 + lane;
                if (!real || x >= p.w) continue;
                const int y = k.ya - 2 + j;
                const size_t plane = (size_t)p.h * p.w;
                const size_t pix = (size_t)y * p.w + x;
#pragma unroll
                for (int i = 0; i < COUT; ++i) {
                    v[i] += sbias[i];
                    if (p.relu) v[i] = fmaxf(v[i], 0.0f);
                }
                if (p.y) {
                    uint4 *dst = reinterpret_cast<uint4 *>(p.y) + (size_t)k.img * (COUT / 8) * plane + pix;
#pragma unroll
                    for (int i = 0; i < COUT / 8; ++i)
                        dst[i * plane] = make_uint4(pack_bf16(v[8 * i], v[8 * i + 1]), pack_bf16(v[8 * i + 2], v[8 * i + 3]),
                                                    pack_bf16(v[8 * i + 4], v[8 * i + 5]), pack_bf16(v[8 * i + 6], v[8 * i + 7]));
                }
                if (p.y0)
                    p.y0[(size_t)k.img * p.y0_stride + (size_t)y * p.y0_pitch + x] =
                        v[0] + (p.resid ? p.resid[(size_t)k.img * p.resid_stride + (size_t)y * p.resid_pitch + x]
                                        : 0.0f);
            }
        }
    }
    fence_before_sync();
    __syncthreads();
    if (warp == 2) {
        __syncwarp();  // tcgen05.dealloc is .sync.aligned: reconverge after the per-lane waits
        fence_after_sync();
        tmem_dealloc(tmem, S::TMEM_COLS);
    }
}

// x0 [n][2][h][w][8]: block 0 = (noisy, sigma / 255 * level_scale, 0 x 6), block 1 = 0;
// the noisy images are noisy_stride floats apart, their rows `pitch` floats apart; the
// noise level of image i is sigma[i], or sigma_all when sigma is null
__global__ void pack_input_blocked(const float *noisy, long long noisy_stride, int pitch, const float *sigma,
                                   float sigma_all, int n, int h, int w, float level_scale, __nv_bfloat16 *x0) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long plane = (long long)h * w;
    if (i >= n * plane) return;
    const long long img = i / plane, pix = i - img * plane;
    const long long y = pix / w, x = pix - y * w;
    const float s = sigma ? sigma[img] : sigma_all;
    uint4 *o = reinterpret_cast<uint4 *>(x0) + img * 2 * plane + pix;
    o[0] = make_uint4(pack_bf16(noisy[img * noisy_stride + y * pitch + x], s * (1.0f / 255.0f) * level_scale), 0u, 0u,
                      0u);
    o[plane] = make_uint4(0u, 0u, 0u, 0u);
}

}  // namespace pilot_tc

// ---- launcher ----------------------------------------------------------------------

// Cap on the CTAs per SM of the launch grid: the shape's own count (3 or 2) fills each
// SM (fastest alone), 1 leaves room for kernels of other streams (step 2 of other frames)
static std::atomic<int> g_conv_ctas_per_sm{pilot_tc::MAX_CTAS_PER_SM};

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(f);
    }
    return fn;
}

template <int CIN, int COUT>
static cudaError_t conv_tc_t(const void *x, pilot_tc::Args a, cudaStream_t st) {
    using S = pilot_tc::Shape<CIN, COUT>;
    EncodeTiledFn enc = encode_tiled();
    if (!enc) return cudaErrorNotSupported;
    // channel-blocked input as a 4-D tensor (element, x, y, image * CIN / 8 + block): with
    // w % 8 == 0 an element run is 8 pixels x 8 channels (128 bytes) and x counts 8-pixel
    // groups, box 18 groups; else a run is one pixel (16 bytes), box 130 pixels
    CUtensorMap map;
    a.grouped = (a.w % 8) == 0;
    const cuuint64_t xs = a.grouped ? (cuuint64_t)(a.w / 8) : (cuuint64_t)a.w;
    const cuuint64_t dims[4] = {a.grouped ? 64ull : 8ull, xs, (cuuint64_t)a.h, (cuuint64_t)a.n * (CIN / 8)};
    const cuuint64_t strides[3] = {a.grouped ? 128ull : 16ull, (cuuint64_t)a.w * 16, (cuuint64_t)a.h * a.w * 16};
    const cuuint32_t box[4] = {a.grouped ? 64u : 8u, a.grouped ? (cuuint32_t)pilot_tc::BOX_GROUPS : (cuuint32_t)pilot_tc::BOX_PIX,
                               1, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    if (enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(x), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return cudaErrorInvalidValue;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    a.strips = (a.w + pilot_tc::TILE - 1) / pilot_tc::TILE;
    // S::CTAS CTAs per SM (capped by g_conv_ctas_per_sm), at least 4 tiles each
    const long long tiles = (long long)a.n * a.strips * a.h;
    const int per_sm = S::CTAS < g_conv_ctas_per_sm.load() ? S::CTAS : g_conv_ctas_per_sm.load();
    const long long want = (tiles + 3) / 4, slots = (long long)per_sm * sms;
    const int grid = (int)(want < slots ? want : slots);
    auto k = pilot_tc::conv3x3_tc<CIN, COUT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM);
    if (e != cudaSuccess) return e;
    k<<<grid, S::THREADS, S::SMEM, st>>>(map, a);
    return cudaGetLastError();
}

}  // namespace zb

// ---- entry points -------------------------------------------------------------------

namespace zb {

// One 3x3 convolution layer on the tensor cores (zb3d_pilot_conv3x3_tc), with row pitches
// for the FP32 output and residual planes.
cudaError_t pilot_conv_tc(const void *x, int n, int h, int w, int cin, const void *wgt, const float *bias, int cout,
                          int relu, void *y, float *y0, long long y0_stride, int y0_pitch, const float *resid,
                          long long resid_stride, int resid_pitch, int *status, cudaStream_t st) {
    if (n <= 0 || h <= 0 || w <= 0) return n == 0 ? cudaSuccess : cudaErrorInvalidValue;
    if ((reinterpret_cast<uintptr_t>(x) & 15) || (reinterpret_cast<uintptr_t>(wgt) & 15) ||
        (reinterpret_cast<uintptr_t>(y) & 15))
        return cudaErrorInvalidValue;
    pilot_tc::Args a{};
    a.wgt = static_cast<const __nv_bfloat16 *>(wgt);
    a.bias = bias;
    a.y = static_cast<__nv_bfloat16 *>(y);
    a.y0 = y0;
    a.resid = resid;
    a.y0_pitch = y0_pitch > 0 ? y0_pitch : w;
    a.resid_pitch = resid_pitch > 0 ? resid_pitch : w;
    if (a.y0_pitch < w || a.resid_pitch < w) return cudaErrorInvalidValue;
    a.y0_stride = y0_stride > 0 ? y0_stride : (long long)h * a.y0_pitch;
    a.resid_stride = resid_stride > 0 ? resid_stride : (long long)h * a.resid_pitch;
    if (a.y0_stride < (long long)h * a.y0_pitch || a.resid_stride < (long long)h * a.resid_pitch)
        return cudaErrorInvalidValue;
    a.n = n;
    a.h = h;
    a.w = w;
    a.relu = relu;
    a.status = status;
    if (cin == 16 && cout == 48) return conv_tc_t<16, 48>(x, a, st);
    if (cin == 48 && cout == 48) return conv_tc_t<48, 48>(x, a, st);
    if (cin == 48 && cout == 16) return conv_tc_t<48, 16>(x, a, st);
    if (cin == 16 && cout == 32) return conv_tc_t<16, 32>(x, a, st);
    if (cin == 32 && cout == 32) return conv_tc_t<32, 32>(x, a, st);
    if (cin == 32 && cout == 16) return conv_tc_t<32, 16>(x, a, st);
    if (cin == 16 && cout == 16) return conv_tc_t<16, 16>(x, a, st);
    return cudaErrorInvalidValue;
}

// The network input of n images (zb3d_pilot_pack_input_blocked), rows `pitch` floats apart;
// sigma: n device values, or null for sigma_all on every image.
cudaError_t pilot_pack_input(const float *noisy, long long noisy_stride, int pitch, const float *sigma,
                             float sigma_all, int n, int h, int w, float level_scale, void *x0, cudaStream_t st) {
    const long long np = (long long)n * h * w;
    if (np <= 0) return np == 0 ? cudaSuccess : cudaErrorInvalidValue;
    if (pitch <= 0) pitch = w;
    if (noisy_stride <= 0) noisy_stride = (long long)h * pitch;
    if (pitch < w || noisy_stride < (long long)h * pitch) return cudaErrorInvalidValue;
    pilot_tc::pack_input_blocked<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(
        noisy, noisy_stride, pitch, sigma, sigma_all, n, h, w, level_scale, static_cast<__nv_bfloat16 *>(x0));
    return cudaGetLastError();
}

}  // namespace zb

// ---- C ABI (include/zb3d.h) ---------------------------------------------------------

extern "C" int zb3d_pilot_conv3x3_tc(const void *x, int n, int h, int w, int cin, const void *wgt, const float *bias,
                                     int cout, int relu, void *y, float *y0, const float *resid, long long y0_stride,
                                     long long resid_stride, int *status, void *stream) {
    if (n == 0) return 0;
    if (y0_stride > 0 && y0_stride < (long long)h * w) return -1;
    if (resid_stride > 0 && resid_stride < (long long)h * w) return -1;
    return zb::pilot_conv_tc(x, n, h, w, cin, wgt, bias, cout, relu, y, y0, y0_stride, w, resid, resid_stride, w,
                             status, (cudaStream_t)stream) == cudaSuccess
               ? 0
               : -1;
}

extern "C" int zb3d_pilot_tc_ctas_per_sm(int ctas) {
    if (ctas < 1 || ctas > zb::pilot_tc::MAX_CTAS_PER_SM) return -1;
    zb::g_conv_ctas_per_sm.store(ctas);
    return 0;
}

extern "C" int zb3d_pilot_pack_input_blocked(const float *noisy, long long noisy_stride, const float *sigma, int n,
                                             int h, int w, float level_scale, void *x0, void *stream) {
    if ((long long)n * h * w < 0 || !sigma) return -1;
    return zb::pilot_pack_input(noisy, noisy_stride, w, sigma, 0.0f, n, h, w, level_scale, x0,
                                (cudaStream_t)stream) == cudaSuccess
               ? 0
               : -1;
}
