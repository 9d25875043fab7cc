// Learned pilot: kernels of a small residual convolutional network that stands in
// for the BM3D step-1 (hard-threshold) estimate as the reference of step 2.
//
// Network: 3x3 convolutions, 16, 32 or 48 channels, ReLU after all but the last; the
// input is the noisy plane plus a noise-level plane, the output (channel 0 of the
// last layer) is added to the noisy plane.  Weights and activations are BF16,
// every product is accumulated in FP32 (mma.sync m16n8k16 BF16 -> FP32).
//
// Layout: activations NHWC with the channel count padded to a multiple of 16
// (the input has 2 real channels of 16, the last layer 1 real output of 16);
// weights [cout][ky][kx][cin], i.e. each output channel's 9 * cin inputs are
// contiguous (the GEMM's K order); biases and gradients FP32.
//
// Forward: implicit GEMM per 8 x 16-pixel tile (M = 128 pixels, N = cout,
// K = 9 * cin) from a shared-memory halo tile and the layer's weights.  The
// same kernel does the backward pass to the input with the weights flipped in
// space and transposed in channels, and applies the ReLU derivative (the next
// layer's forward activation > 0) in its epilogue.  The weight gradient is a
// persistent kernel: GEMM with M = cout, N = cin per kernel tap, K = pixels,
// one warp per tap, FP32 partials flushed once per CTA.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstdint>

namespace zb {
namespace pilot {

constexpr int TW = 16, TH = 8;            // output tile: 16 columns x 8 rows = 128 pixels
constexpr int HW = TW + 2, HH = TH + 2;   // halo tile
constexpr int HPIX = HW * HH;

struct ConvArgs {
    const __nv_bfloat16 *x;   // [n][h][w][cin]
    const __nv_bfloat16 *wgt; // [cout][9][cin]
    const float *bias;        // [cout] or null
    const __nv_bfloat16 *mask;  // [n][h][w][cout] or null: zero the outputs where mask <= 0 (ReLU derivative)
    __nv_bfloat16 *y;         // [n][h][w][cout] or null
    float *y0;                // [n][h][w] or null: output channel 0 in FP32 (+ resid)
    const float *resid;       // [n][h][w] or null: added to y0
    int n, h, w;
    int relu;
};

struct WgradArgs {
    const __nv_bfloat16 *x;   // [n][h][w][cin]  forward input of the layer
    const __nv_bfloat16 *dy;  // [n][h][w][cout] gradient at the layer's pre-activation
    float *dw;                // [cout][9][cin]  accumulated (+=)
    float *db;                // [cout]          accumulated (+=)
    int n, h, w;
};

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

template <int CIN, int COUT>
struct FwdShape {
    static constexpr int PP = CIN + 8;         // halo pixel pitch (bf16): conflict-free fragment loads
    static constexpr int K = 9 * CIN;
    static constexpr int KP = K + 8;           // weight row pitch (bf16)
    static constexpr int SMEM = (HPIX * PP + COUT * KP) * 2;
};

// y = conv3x3(x) (+ bias, ReLU, mask); grid (ceil(w/16), ceil(h/8), n), 128 threads.
template <int CIN, int COUT>
__global__ void __launch_bounds__(128) conv3x3(ConvArgs p) {
    using S = FwdShape<CIN, COUT>;
    constexpr int NT = COUT / 8;
    extern __shared__ __align__(16) __nv_bfloat16 sm[];
    __nv_bfloat16 *sx = sm;
    __nv_bfloat16 *sw = sm + HPIX * S::PP;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, tig = lane & 3;
    const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH, img = blockIdx.z;
    const __nv_bfloat16 *xin = p.x + (size_t)img * p.h * p.w * CIN;
    for (int i = tid; i < HPIX * (CIN / 2); i += 128) {
        const int pix = i / (CIN / 2), cp = i - pix * (CIN / 2);
        const int yy = y0 - 1 + pix / HW, xx = x0 - 1 + pix % HW;
        uint32_t v = 0;
        if (yy >= 0 && yy < p.h && xx >= 0 && xx < p.w)
            v = reinterpret_cast<const uint32_t *>(xin + ((size_t)yy * p.w + xx) * CIN)[cp];
        reinterpret_cast<uint32_t *>(sx + pix * S::PP)[cp] = v;
    }
    for (int i = tid; i < COUT * (S::K / 2); i += 128) {
        const int co = i / (S::K / 2), kp = i - co * (S::K / 2);
        reinterpret_cast<uint32_t *>(sw + co * S::KP)[kp] = reinterpret_cast<const uint32_t *>(p.wgt + (size_t)co * S::K)[kp];
    }
    __syncthreads();

    float acc[2][NT][4];
#pragma unroll
    for (int mt = 0; mt < 2; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[mt][nt][k] = 0.0f;
    // warp w: output rows 2w and 2w + 1 (one m16 tile each: pixels = the row's 16 columns)
#pragma unroll 1
    for (int tap = 0; tap < 9; ++tap) {
        const int ky = tap / 3, kx = tap - 3 * ky;
#pragma unroll
        for (int cc = 0; cc < CIN; cc += 16) {
            uint32_t a[2][4];
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                const __nv_bfloat16 *base = sx + ((2 * warp + mt + ky) * HW + kx) * S::PP + cc + 2 * tig;
                a[mt][0] = ld32(base + g * S::PP);
                a[mt][1] = ld32(base + (g + 8) * S::PP);
                a[mt][2] = ld32(base + g * S::PP + 8);
                a[mt][3] = ld32(base + (g + 8) * S::PP + 8);
            }
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const __nv_bfloat16 *wb = sw + (nt * 8 + g) * S::KP + tap * CIN + cc + 2 * tig;
                const uint32_t b[2] = {ld32(wb), ld32(wb + 8)};
                mma_bf16(acc[0][nt], a[0], b);
                mma_bf16(acc[1][nt], a[1], b);
            }
        }
    }

    // epilogue: c0, c1 -> pixel column g, channels 8 nt + 2 tig (+1); c2, c3 -> column g + 8
    const size_t plane = (size_t)p.h * p.w;
#pragma unroll
    for (int mt = 0; mt < 2; ++mt) {
        const int yy = y0 + 2 * warp + mt;
        if (yy >= p.h) continue;
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int xx = x0 + g + 8 * half;
            if (xx >= p.w) continue;
            const size_t pix = (size_t)img * plane + (size_t)yy * p.w + xx;
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const int co = nt * 8 + 2 * tig;
                float v0 = acc[mt][nt][2 * half], v1 = acc[mt][nt][2 * half + 1];
                if (p.bias) {
                    v0 += p.bias[co];
                    v1 += p.bias[co + 1];
                }
                if (p.relu) {
                    v0 = fmaxf(v0, 0.0f);
                    v1 = fmaxf(v1, 0.0f);
                }
                if (p.mask) {
                    const uint32_t m = ld32(p.mask + pix * COUT + co);
                    if (!(__bfloat162float(__ushort_as_bfloat16((unsigned short)(m & 0xffff))) > 0.0f)) v0 = 0.0f;
                    if (!(__bfloat162float(__ushort_as_bfloat16((unsigned short)(m >> 16))) > 0.0f)) v1 = 0.0f;
                }
                if (p.y)
                    *reinterpret_cast<uint32_t *>(p.y + pix * COUT + co) = pack2(__float2bfloat16_rn(v0), __float2bfloat16_rn(v1));
                if (p.y0 && co == 0) p.y0[pix] = v0 + (p.resid ? p.resid[pix] : 0.0f);
            }
        }
    }
}

template <int CIN, int COUT>
struct WgShape {
    static constexpr int DP = TW * TH + 8;     // transposed gradient tile pitch (pixels)
    static constexpr int XP = HPIX + 6;        // transposed halo pitch (pixels)
    static constexpr int SMEM = (COUT * DP + CIN * XP) * 2;
};

// dw[co][tap][ci] += sum over pixels dy[p][co] * x[p + tap offset][ci]; db[co] += sum dy[p][co].
// Persistent: CTA b handles tiles b, b + gridDim.x, ...; 9 warps (one per tap) + the bias sums.
template <int CIN, int COUT>
__global__ void __launch_bounds__(288) conv3x3_wgrad(WgradArgs p) {
    using S = WgShape<CIN, COUT>;
    constexpr int MT = COUT / 16, NT = CIN / 8;
    extern __shared__ __align__(16) __nv_bfloat16 sm[];
    __nv_bfloat16 *dyT = sm;                    // [COUT][DP]: pixel index r * 16 + c
    __nv_bfloat16 *xT = sm + COUT * S::DP;      // [CIN][XP]:  halo index hr * 18 + hc
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31, g = lane >> 2, tig = lane & 3;
    const int ky = warp / 3, kx = warp - 3 * ky;
    const int tx = (p.w + TW - 1) / TW, ty = (p.h + TH - 1) / TH;
    const long long ntiles = (long long)tx * ty * p.n;
    float acc[MT][NT][4];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[mt][nt][k] = 0.0f;
    float bsum = 0.0f;  // thread tid < COUT: bias gradient of channel tid
    for (long long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int img = (int)(t / ((long long)tx * ty));
        const int rem = (int)(t - (long long)img * tx * ty);
        const int y0 = (rem / tx) * TH, x0 = (rem % tx) * TW;
        const size_t base = (size_t)img * p.h * p.w;
        __syncthreads();  // the previous tile's fragments are consumed
        for (int i = tid; i < TW * TH * COUT; i += 288) {
            const int pix = i / COUT, co = i - pix * COUT;
            const int yy = y0 + pix / TW, xx = x0 + pix % TW;
            __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
            if (yy < p.h && xx < p.w) v = p.dy[(base + (size_t)yy * p.w + xx) * COUT + co];
            dyT[co * S::DP + pix] = v;
        }
        for (int i = tid; i < HPIX * CIN; i += 288) {
            const int hp = i / CIN, ci = i - hp * CIN;
            const int yy = y0 - 1 + hp / HW, xx = x0 - 1 + hp % HW;
            __nv_bfloat16 v = __float2bfloat16_rn(0.0f);
            if (yy >= 0 && yy < p.h && xx >= 0 && xx < p.w) v = p.x[(base + (size_t)yy * p.w + xx) * CIN + ci];
            xT[ci * S::XP + hp] = v;
        }
        __syncthreads();
        if (tid < COUT) {
            float s = 0.0f;
            for (int q = 0; q < TW * TH; ++q) s += __bfloat162float(dyT[tid * S::DP + q]);
            bsum += s;
        }
#pragma unroll 1
        for (int r = 0; r < TH; ++r) {  // K step = the 16 pixels of tile row r
            uint32_t a[MT][4];
#pragma unroll
            for (int mt = 0; mt < MT; ++mt) {
                const __nv_bfloat16 *d = dyT + (16 * mt + g) * S::DP + 16 * r + 2 * tig;
                a[mt][0] = ld32(d);
                a[mt][1] = ld32(d + 8 * S::DP);
                a[mt][2] = ld32(d + 8);
                a[mt][3] = ld32(d + 8 * S::DP + 8);
            }
            const int h0 = (r + ky) * HW + kx + 2 * tig;  // halo index of pixel column 2 tig
#pragma unroll
            for (int nt = 0; nt < NT; ++nt) {
                const __nv_bfloat16 *xs = xT + (8 * nt + g) * S::XP + h0;
                const uint32_t b[2] = {pack2(xs[0], xs[1]), pack2(xs[8], xs[9])};
#pragma unroll
                for (int mt = 0; mt < MT; ++mt) mma_bf16(acc[mt][nt], a[mt], b);
            }
        }
    }
    // flush: c0, c1 -> co = 16 mt + g, ci = 8 nt + 2 tig (+1); c2, c3 -> co + 8
    const int tap = warp;
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int nt = 0; nt < NT; ++nt) {
            const int co = 16 * mt + g, ci = 8 * nt + 2 * tig;
            float *d0 = p.dw + ((size_t)co * 9 + tap) * CIN + ci;
            float *d1 = p.dw + ((size_t)(co + 8) * 9 + tap) * CIN + ci;
            atomicAdd(d0, acc[mt][nt][0]);
            atomicAdd(d0 + 1, acc[mt][nt][1]);
            atomicAdd(d1, acc[mt][nt][2]);
            atomicAdd(d1 + 1, acc[mt][nt][3]);
        }
    if (tid < COUT && p.db) atomicAdd(p.db + tid, bsum);
}

// ---- element-wise kernels ------------------------------------------------------

// x0[p][16]: channel 0 = noisy, channel 1 = sigma / 255 * level_scale, 2..15 = 0.
__global__ void pack_input(const float *noisy, const float *sigma, int n, int h, int w, float level_scale,
                           __nv_bfloat16 *x0) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long np = (long long)n * h * w;
    if (i >= np) return;
    const int img = (int)(i / ((long long)h * w));
    uint32_t *o = reinterpret_cast<uint32_t *>(x0 + i * 16);
    o[0] = pack2(__float2bfloat16_rn(noisy[i]), __float2bfloat16_rn(sigma[img] * (1.0f / 255.0f) * level_scale));
#pragma unroll
    for (int k = 1; k < 8; ++k) o[k] = 0;
}

// dy[p][16] = scale * 2 (y - t) / count in channel 0; partial[blockIdx.x] = the CTA's
// sum of (y - t)^2 in FP32 (the caller adds the partials up on the host).
__global__ void __launch_bounds__(256) mse_grad(const float *y, const float *t, long long count, float scale,
                                               __nv_bfloat16 *dy, float *partial) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    float e2 = 0.0f;
    if (i < count) {
        const float d = y[i] - t[i];
        e2 = d * d;
        uint32_t *o = reinterpret_cast<uint32_t *>(dy + i * 16);
        o[0] = pack2(__float2bfloat16_rn(scale * 2.0f * d / (float)count), __float2bfloat16_rn(0.0f));
#pragma unroll
        for (int k = 1; k < 8; ++k) o[k] = 0;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
    __shared__ float ws[8];
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = e2;
    __syncthreads();
    if (threadIdx.x == 0 && partial)
        partial[blockIdx.x] = ((ws[0] + ws[1]) + (ws[2] + ws[3])) + ((ws[4] + ws[5]) + (ws[6] + ws[7]));
}

// Adam on FP32 master weights; g is the loss-scaled gradient (divided by gscale here);
// the BF16 copy used by the kernels is refreshed.  keep (may be null): 0 = parameter frozen at 0.
__global__ void adam(float *w, float *m, float *v, const float *g, long long count, float lr, float b1, float b2,
                     float eps, float c1, float c2, float gscale, const float *keep, __nv_bfloat16 *w16) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i] / gscale;
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    if (keep && keep[i] == 0.0f) wi = 0.0f;
    w[i] = wi;
    if (w16) w16[i] = __float2bfloat16_rn(wi);
}

// wt[ci][tap'][co] = w[co][8 - tap'][ci]: the weights of the backward pass to the input.
__global__ void flip_weights(const __nv_bfloat16 *w, int cin, int cout, __nv_bfloat16 *wt) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= cin * 9 * cout) return;
    const int ci = i / (9 * cout), rem = i - ci * 9 * cout, tap = rem / cout, co = rem - tap * cout;
    wt[i] = w[((size_t)co * 9 + (8 - tap)) * cin + ci];
}

__global__ void f32_to_bf16(const float *a, long long count, __nv_bfloat16 *b) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) b[i] = __float2bfloat16_rn(a[i]);
}

}  // namespace pilot

// ---- launchers -----------------------------------------------------------------------

template <int CIN, int COUT>
static cudaError_t conv_t(const pilot::ConvArgs &a, cudaStream_t st) {
    using S = pilot::FwdShape<CIN, COUT>;
    auto k = pilot::conv3x3<CIN, COUT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM);
    if (e != cudaSuccess) return e;
    const dim3 grid((a.w + pilot::TW - 1) / pilot::TW, (a.h + pilot::TH - 1) / pilot::TH, a.n);
    k<<<grid, 128, S::SMEM, st>>>(a);
    return cudaGetLastError();
}

template <int CIN, int COUT>
static cudaError_t wgrad_t(const pilot::WgradArgs &a, cudaStream_t st) {
    using S = pilot::WgShape<CIN, COUT>;
    auto k = pilot::conv3x3_wgrad<CIN, COUT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, S::SMEM);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long tiles = (long long)((a.w + pilot::TW - 1) / pilot::TW) * ((a.h + pilot::TH - 1) / pilot::TH) * a.n;
    const int grid = (int)(tiles < 2LL * sms ? tiles : 2LL * sms);
    k<<<grid, 288, S::SMEM, st>>>(a);
    return cudaGetLastError();
}

cudaError_t pilot_conv(int cin, int cout, const pilot::ConvArgs &a, cudaStream_t st) {
    if (cin == 16 && cout == 48) return conv_t<16, 48>(a, st);
    if (cin == 48 && cout == 48) return conv_t<48, 48>(a, st);
    if (cin == 48 && cout == 16) return conv_t<48, 16>(a, st);
    if (cin == 16 && cout == 32) return conv_t<16, 32>(a, st);
    if (cin == 32 && cout == 32) return conv_t<32, 32>(a, st);
    if (cin == 32 && cout == 16) return conv_t<32, 16>(a, st);
    if (cin == 16 && cout == 16) return conv_t<16, 16>(a, st);
    return cudaErrorInvalidValue;
}

cudaError_t pilot_wgrad(int cin, int cout, const pilot::WgradArgs &a, cudaStream_t st) {
    if (cin == 16 && cout == 48) return wgrad_t<16, 48>(a, st);
    if (cin == 48 && cout == 48) return wgrad_t<48, 48>(a, st);
    if (cin == 48 && cout == 16) return wgrad_t<48, 16>(a, st);
    if (cin == 16 && cout == 32) return wgrad_t<16, 32>(a, st);
    if (cin == 32 && cout == 32) return wgrad_t<32, 32>(a, st);
    if (cin == 32 && cout == 16) return wgrad_t<32, 16>(a, st);
    if (cin == 16 && cout == 16) return wgrad_t<16, 16>(a, st);
    return cudaErrorInvalidValue;
}

}  // namespace zb

// ---- C ABI (include/zb3d.h) ---------------------------------------------------------

extern "C" {

int zb3d_pilot_conv3x3(const void *x, int n, int h, int w, int cin, const void *wgt, const float *bias, int cout,
                       int relu, const void *mask, void *y, float *y0, const float *resid, void *stream) {
    zb::pilot::ConvArgs a{};
    a.x = static_cast<const __nv_bfloat16 *>(x);
    a.wgt = static_cast<const __nv_bfloat16 *>(wgt);
    a.bias = bias;
    a.mask = static_cast<const __nv_bfloat16 *>(mask);
    a.y = static_cast<__nv_bfloat16 *>(y);
    a.y0 = y0;
    a.resid = resid;
    a.n = n;
    a.h = h;
    a.w = w;
    a.relu = relu;
    return zb::pilot_conv(cin, cout, a, (cudaStream_t)stream) == cudaSuccess ? 0 : -1;
}

int zb3d_pilot_conv3x3_wgrad(const void *x, const void *dy, int n, int h, int w, int cin, int cout, float *dw,
                             float *db, void *stream) {
    zb::pilot::WgradArgs a{};
    a.x = static_cast<const __nv_bfloat16 *>(x);
    a.dy = static_cast<const __nv_bfloat16 *>(dy);
    a.dw = dw;
    a.db = db;
    a.n = n;
    a.h = h;
    a.w = w;
    return zb::pilot_wgrad(cin, cout, a, (cudaStream_t)stream) == cudaSuccess ? 0 : -1;
}

int zb3d_pilot_pack_input(const float *noisy, const float *sigma, int n, int h, int w, float level_scale, void *x0,
                          void *stream) {
    const long long np = (long long)n * h * w;
    zb::pilot::pack_input<<<(unsigned)((np + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        noisy, sigma, n, h, w, level_scale, static_cast<__nv_bfloat16 *>(x0));
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int zb3d_pilot_mse_grad(const float *y, const float *t, long long count, float scale, void *dy,
                        float *loss_partials, void *stream) {
    zb::pilot::mse_grad<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        y, t, count, scale, static_cast<__nv_bfloat16 *>(dy), loss_partials);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int zb3d_pilot_adam(float *w, float *m, float *v, const float *g, long long count, float lr, float b1, float b2,
                    float eps, int step, float gscale, const float *keep, void *w16, void *stream) {
    const float c1 = 1.0f - powf(b1, (float)step), c2 = 1.0f - powf(b2, (float)step);
    zb::pilot::adam<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        w, m, v, g, count, lr, b1, b2, eps, c1, c2, gscale, keep, static_cast<__nv_bfloat16 *>(w16));
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int zb3d_pilot_flip_weights(const void *w, int cin, int cout, void *wt, void *stream) {
    const int count = cin * 9 * cout;
    zb::pilot::flip_weights<<<(count + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
        static_cast<const __nv_bfloat16 *>(w), cin, cout, static_cast<__nv_bfloat16 *>(wt));
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int zb3d_pilot_to_bf16(const float *a, long long count, void *b, void *stream) {
    zb::pilot::f32_to_bf16<<<(unsigned)((count + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
        a, count, static_cast<__nv_bfloat16 *>(b));
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // extern "C"
