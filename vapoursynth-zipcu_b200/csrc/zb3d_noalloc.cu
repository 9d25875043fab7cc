// One BM3D pass over one device-resident plane without any device allocation.
//
// Some callers cannot call cudaMalloc while they run: a frame server that fixes
// every plugin's device-memory budget when it loads them and must not see it grow
// at frame time, or a real-time host that cannot afford cudaMalloc's implicit
// device-wide synchronisation in the middle of a frame.  zb3d_bm3d_plane_noalloc
// serves them: its scratch (the fixed-point accumulators and the match lists) is
// a fixed array compiled into this library, so a call allocates nothing.
//
// Cost and limits: every GPU that loads the library holds the array (24 MiB)
// until the process exits; a plane needs at most kAccPixels pitched pixels of
// accumulators and kListBlocks reference blocks, larger ones are rejected; all
// calls share the one array, so calls that overlap on the GPU race.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/zb3d.h"
#include "zb3d_args.h"

// pitched pixels per accumulator plane, reference blocks, and the scratch size:
// [num accumulators | weight accumulators | match lists] = 24 MiB
#define ZB_NOALLOC_ACC_PIXELS (size_t(1) << 20)
#define ZB_NOALLOC_LIST_BLOCKS (size_t(1) << 17)
#define ZB_NOALLOC_BYTES (2 * ZB_NOALLOC_ACC_PIXELS * 8 + ZB_NOALLOC_LIST_BLOCKS * 64)
#define ZB_NOALLOC_FLT_EPSILON 1.19209290e-7f

static __device__ __align__(256) unsigned char zb_noalloc_scratch[ZB_NOALLOC_BYTES];

namespace zb {

cudaError_t launch_match(MatchArgs a, int metric, int rows_per_cta, bool use_tiled, cudaStream_t st);
size_t match_tile_bytes(const MatchArgs &a, int rows_per_cta);
cudaError_t launch_filter(const FilterArgs &a, bool final_, int t2d, int t1d, cudaStream_t st);
cudaError_t launch_finish(const unsigned long long *num, const unsigned long long *den, long long acc_plane_stride,
                          long long acc_frame_stride, int w, int h, int pitch, int nplanes, int tw,
                          unsigned proc_mask, float *dst, int dst_pitch, long long dst_plane_stride, int mode,
                          cudaStream_t st);

namespace {

constexpr size_t kAccPixels = ZB_NOALLOC_ACC_PIXELS;
constexpr size_t kListBlocks = ZB_NOALLOC_LIST_BLOCKS;
constexpr size_t kAccBytes = kAccPixels * sizeof(unsigned long long);
constexpr size_t kListBytes = kListBlocks * 8 * sizeof(int2);
static_assert(2 * kAccBytes + kListBytes == ZB_NOALLOC_BYTES, "scratch layout");

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch[kMaxDevices] = {};

void set_err(char *err, size_t n, const char *msg) {
    if (err && n) snprintf(err, n, "%s", msg);
}

// Device address of the scratch array on the current device.  The name of a
// __device__ array is only a host-side handle; the address comes from the
// runtime, looked up once per device with that device current, and kept for the
// life of the process: a caller that resets a device (cudaDeviceReset) must not
// call this entry point on that device again.
unsigned char *scratch_for_current_device(char *err, size_t errlen) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_err(err, errlen, "zb3d_bm3d_plane_noalloc: no usable current CUDA device.");
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, zb_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            if (err && errlen)
                snprintf(err, errlen, "zb3d_bm3d_plane_noalloc: cudaGetSymbolAddress failed (%s).",
                         cudaGetErrorString(e));
            return nullptr;
        }
        g_scratch[dev] = static_cast<unsigned char *>(p);
    }
    return g_scratch[dev];
}

}  // namespace
}  // namespace zb

extern "C" int zb3d_bm3d_plane_noalloc(const float *d_src, float *d_dst, int width, int height, int pitch,
                                       int final_, float sigma, int block_step, int bm_range, int extractor_exp,
                                       void *stream, char *err, size_t errlen) {
    using namespace zb;
    if (!d_src || !d_dst || width < 8 || height < 8 || pitch < width || block_step < 1 || block_step > 8 ||
        bm_range < 1 || !(sigma >= 0.0f)) {
        set_err(err, errlen, "zb3d_bm3d_plane_noalloc: invalid arguments (plane at least 8x8, pitch >= width, "
                             "block_step 1..8, bm_range > 0, sigma >= 0).");
        return -1;
    }
    const size_t pixels = (size_t)height * pitch;
    const int nbx = (width - 8 + block_step - 1) / block_step + 1;
    const int nby = (height - 8 + block_step - 1) / block_step + 1;
    const size_t nblocks = (size_t)nbx * nby;
    if (pixels > kAccPixels || nblocks > kListBlocks) {
        if (err && errlen)
            snprintf(err, errlen,
                     "zb3d_bm3d_plane_noalloc: plane too large for the built-in scratch (%zu pitched pixels and %zu "
                     "blocks requested, limits %zu and %zu).",
                     pixels, nblocks, kAccPixels, kListBlocks);
        return -1;
    }
    cudaStream_t st = (cudaStream_t)stream;
    // sigma below FLT_EPSILON: the plane is not processed and the output is the noisy
    // plane itself, as the reference's output frame keeps unprocessed planes of the
    // noisy clip (vszipcu src/bm3d.zig:1017, :702-703)
    if (sigma < ZB_NOALLOC_FLT_EPSILON) {
        const float *noisy = d_src + (final_ ? pixels : 0);
        const cudaError_t ce = cudaMemcpy2DAsync(d_dst, (size_t)pitch * 4, noisy, (size_t)pitch * 4,
                                                 (size_t)width * 4, (size_t)height, cudaMemcpyDeviceToDevice, st);
        if (ce != cudaSuccess) {
            if (err && errlen)
                snprintf(err, errlen, "zb3d_bm3d_plane_noalloc: copy failed (%s).", cudaGetErrorString(ce));
            return -1;
        }
        return 0;
    }
    unsigned char *base = scratch_for_current_device(err, errlen);
    if (!base) return -1;
    unsigned long long *num = reinterpret_cast<unsigned long long *>(base);
    unsigned long long *den = reinterpret_cast<unsigned long long *>(base + kAccBytes);
    int2 *list = reinterpret_cast<int2 *>(base + 2 * kAccBytes);

    // the array keeps the previous call's sums: both accumulators start from zero
    cudaError_t e = cudaMemsetAsync(num, 0, pixels * sizeof(unsigned long long), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(den, 0, pixels * sizeof(unsigned long long), st);

    // scaled sigma as the reference host stores it (vszipcu src/bm3d.zig:1019-1024)
    const unsigned bits = final_ ? 0x3e40c0c1u : 0x3f021bb6u;
    float factor;
    memcpy(&factor, &bits, 4);
    const float s = sigma * factor;

    MatchArgs ma{};
    ma.frames = d_src;  // clip 0: the plane matched on (noisy, or the basic estimate)
    ma.fstride = (long long)pixels;
    ma.w = width;
    ma.h = height;
    ma.pitch = pitch;
    ma.bs = block_step;
    ma.range = bm_range;
    ma.nbx = nbx;
    ma.nby = nby;
    ma.nbx_al = (width - 8) / block_step + 1;
    ma.list = list;
    bool tiled = block_step == 4 || block_step == 8;
    if (tiled) {
        MatchArgs t = ma;
        t.chunks = (2 * bm_range + 1 + 3) / 4;
        t.tile_pitch = 128 + 4 * t.chunks;
        tiled = match_tile_bytes(t, 4) <= 200 * 1024;
    }
    if (e == cudaSuccess) e = launch_match(ma, M_SSD, 4, tiled, st);

    FilterArgs fa{};
    fa.src = d_src;
    fa.plane_stride = (long long)pixels;
    fa.clip_stride = (long long)pixels;
    fa.frame_stride = (long long)pixels;
    fa.w = width;
    fa.h = height;
    fa.pitch = pitch;
    fa.nplanes = 1;
    fa.chroma = 0;
    fa.list = list;
    fa.nblocks = (int)nblocks;
    fa.sigma[0] = fa.sigma[1] = fa.sigma[2] = s;
    fa.extractor = extractor_exp != 0 ? ldexpf(1.0f, extractor_exp) : 0.0f;
    fa.num = num;
    fa.den = den;
    fa.acc_plane_stride = (long long)pixels;
    fa.acc_frame_stride = (long long)pixels;
    if (e == cudaSuccess) e = launch_filter(fa, final_ != 0, 0, 0, st);
    if (e == cudaSuccess)
        e = launch_finish(num, den, (long long)pixels, (long long)pixels, width, height, pitch, 1, 1, 1u, d_dst,
                          pitch, (long long)pixels, 0, st);
    if (e != cudaSuccess) {
        if (err && errlen)
            snprintf(err, errlen, "zb3d_bm3d_plane_noalloc: launch failed (%s).", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}
