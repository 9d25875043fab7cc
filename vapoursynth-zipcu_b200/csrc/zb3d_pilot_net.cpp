// The learned pilot as a self-contained network object behind the C ABI: weights file
// loading (format below), the gate, and the whole forward pass (input packing, the 3x3
// convolution stack on the tensor cores, the residual output) into a plane of any row
// pitch.  No torch: device buffers are plain pointers, the workspace is the caller's.
//
// Weights file "ZB3DPLT1" (little-endian), written by zb3d.pilot.save_weights:
//   char magic[8] = "ZB3DPLT1"; u32 version = 1; u32 width, layers; f32 level_scale;
//   u32 gate_frames (held-out frames per gate level); f32 tol; u32 n_gate;
//   n_gate x {f32 sigma, u32 plane_width, u32 plane_height, f32 delta_db};
//   per layer l of arch(width, layers): f32 w[cout][3][3][cin], f32 b[cout];
//   u32 crc32 (IEEE 802.3, zlib's) of every byte before it.
// arch: (16, width), (width, width) x (layers - 2), (width, 16); the 2 real input
// channels (noisy, noise level) and the 1 real output channel are zero-padded to 16.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "zb3d.h"

namespace zb {
cudaError_t pilot_conv_tc(const void *x, int n, int h, int w, int cin, const void *wgt, const float *bias, int cout,
                          int relu, void *y, float *y0, long long y0_stride, int y0_pitch, const float *resid,
                          long long resid_stride, int resid_pitch, int *status, cudaStream_t st);
cudaError_t pilot_pack_input(const float *noisy, long long noisy_stride, int pitch, const float *sigma,
                             float sigma_all, int n, int h, int w, float level_scale, void *x0, cudaStream_t st);
}  // namespace zb

struct zb3d_pilot {
    int device = 0;
    int width = 0, layers = 0;
    float level_scale = 0.0f;
    int gate_frames = 0;
    float tol = 0.05f;
    struct Level {
        float sigma;
        int w, h;
        float delta;  // mean two-pass PSNR difference, pilot minus plain step 1 (dB)
    };
    std::vector<Level> gate;
    std::vector<std::pair<int, int>> shapes;    // (cin, cout)
    std::vector<void *> w16;                    // BF16 [cout][3][3][cin] per layer
    std::vector<float *> b32;                   // FP32 [cout] per layer

    ~zb3d_pilot() {
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(device);
        for (void *p : w16) cudaFree(p);
        for (float *p : b32) cudaFree(p);
        cudaSetDevice(prev);
    }
};

namespace zb {
int pilot_device(const zb3d_pilot *p) { return p ? p->device : -1; }
}  // namespace zb

namespace {

void perr(char *err, size_t n, const char *fmt, ...) {
    if (!err || n == 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, n, fmt, ap);
    va_end(ap);
}

uint32_t crc32_ieee(const unsigned char *p, size_t n) {
    static uint32_t table[256];
    static bool init = [] {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1) ? 0xEDB88320u ^ (c >> 1) : c >> 1;
            table[i] = c;
        }
        return true;
    }();
    (void)init;
    uint32_t c = 0xFFFFFFFFu;
    for (size_t i = 0; i < n; ++i) c = table[(c ^ p[i]) & 0xFF] ^ (c >> 8);
    return c ^ 0xFFFFFFFFu;
}

// Sequential little-endian reader over the file bytes.
struct Reader {
    const unsigned char *p;
    size_t n, at = 0;
    bool ok = true;
    template <typename T>
    T get() {
        T v{};
        if (at + sizeof(T) > n) {
            ok = false;
            return v;
        }
        memcpy(&v, p + at, sizeof(T));
        at += sizeof(T);
        return v;
    }
    const float *floats(size_t count) {
        if (count > (n - at) / 4) {
            ok = false;
            return nullptr;
        }
        const float *f = reinterpret_cast<const float *>(p + at);
        at += count * 4;
        return f;
    }
};

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" {

zb3d_pilot *zb3d_pilot_from_memory(const void *data, size_t bytes, int device_id, char *err, size_t errlen) {
    const unsigned char *p = static_cast<const unsigned char *>(data);
    if (!p || bytes < 8 + 4 + 4) {
        perr(err, errlen, "zb3d pilot: weights data too short");
        return nullptr;
    }
    if (memcmp(p, "ZB3DPLT1", 8) != 0) {
        perr(err, errlen, "zb3d pilot: not a ZB3DPLT1 weights file");
        return nullptr;
    }
    uint32_t stored = 0;
    memcpy(&stored, p + bytes - 4, 4);
    if (crc32_ieee(p, bytes - 4) != stored) {
        perr(err, errlen, "zb3d pilot: weights checksum mismatch (file damaged)");
        return nullptr;
    }
    Reader r{p + 8, bytes - 8 - 4};
    const uint32_t version = r.get<uint32_t>();
    std::unique_ptr<zb3d_pilot> net(new zb3d_pilot());
    net->device = device_id;
    net->width = (int)r.get<uint32_t>();
    net->layers = (int)r.get<uint32_t>();
    net->level_scale = r.get<float>();
    net->gate_frames = (int)r.get<uint32_t>();
    net->tol = r.get<float>();
    const uint32_t ngate = r.get<uint32_t>();
    if (!r.ok || version != 1) {
        perr(err, errlen, "zb3d pilot: unsupported weights version %u", version);
        return nullptr;
    }
    if ((net->width != 16 && net->width != 32 && net->width != 48) || net->layers < 2 || net->layers > 64 ||
        !(net->level_scale > 0.0f) || ngate > 1024 || !(net->tol >= 0.0f)) {
        perr(err, errlen, "zb3d pilot: unsupported architecture (%d channels x %d layers)", net->width, net->layers);
        return nullptr;
    }
    for (uint32_t i = 0; i < ngate; ++i) {
        zb3d_pilot::Level lv;
        lv.sigma = r.get<float>();
        lv.w = (int)r.get<uint32_t>();
        lv.h = (int)r.get<uint32_t>();
        lv.delta = r.get<float>();
        if (lv.w <= 0 || lv.h <= 0 || !(lv.sigma >= 0.0f)) r.ok = false;
        net->gate.push_back(lv);
    }
    net->shapes.emplace_back(16, net->width);
    for (int l = 1; l < net->layers - 1; ++l) net->shapes.emplace_back(net->width, net->width);
    net->shapes.emplace_back(net->width, 16);
    size_t need = 0;  // weight and bias floats the architecture has
    for (const auto &sh : net->shapes) need += (size_t)sh.second * 9 * sh.first + (size_t)sh.second;
    if (!r.ok || r.n - r.at != need * 4) {
        perr(err, errlen, "zb3d pilot: weights size does not match the architecture");
        return nullptr;
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device_id < 0 || device_id >= ndev) {
        cudaGetLastError();
        perr(err, errlen, "zb3d pilot: invalid device ID");
        return nullptr;
    }
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(device_id);
    float *staging = nullptr;
    bool ok = r.ok;
    for (size_t l = 0; ok && l < net->shapes.size(); ++l) {
        const int cin = net->shapes[l].first, cout = net->shapes[l].second;
        const size_t nw = (size_t)cout * 9 * cin;
        const float *w = r.floats(nw);
        const float *b = r.floats((size_t)cout);
        if (!r.ok) {
            ok = false;
            break;
        }
        void *w16 = nullptr;
        float *b32 = nullptr;
        ok = cudaMalloc(&w16, nw * 2) == cudaSuccess;
        if (w16) net->w16.push_back(w16);
        ok = ok && cudaMalloc(&b32, (size_t)cout * 4) == cudaSuccess;
        if (b32) net->b32.push_back(b32);
        ok = ok && cudaMalloc(&staging, nw * 4) == cudaSuccess;
        ok = ok && cudaMemcpy(staging, w, nw * 4, cudaMemcpyHostToDevice) == cudaSuccess;
        // the same FP32 -> BF16 rounding kernel the training code uses for its weights
        ok = ok && zb3d_pilot_to_bf16(staging, (long long)nw, w16, nullptr) == 0;
        ok = ok && cudaMemcpy(b32, b, (size_t)cout * 4, cudaMemcpyHostToDevice) == cudaSuccess;
        ok = ok && cudaDeviceSynchronize() == cudaSuccess;
        cudaFree(staging);
        staging = nullptr;
    }
    cudaSetDevice(prev);
    if (!ok) {
        cudaGetLastError();
        perr(err, errlen, "zb3d pilot: out of device memory");
        return nullptr;
    }
    return net.release();
}

zb3d_pilot *zb3d_pilot_load(const char *path, int device_id, char *err, size_t errlen) {
    FILE *fp = path ? fopen(path, "rb") : nullptr;
    if (!fp) {
        perr(err, errlen, "zb3d pilot: cannot open weights file %s", path ? path : "(null)");
        return nullptr;
    }
    std::vector<unsigned char> buf;
    unsigned char chunk[65536];
    size_t got;
    while ((got = fread(chunk, 1, sizeof(chunk), fp)) > 0) buf.insert(buf.end(), chunk, chunk + got);
    const bool bad = ferror(fp) != 0;
    fclose(fp);
    if (bad) {
        perr(err, errlen, "zb3d pilot: cannot read weights file %s", path);
        return nullptr;
    }
    return zb3d_pilot_from_memory(buf.data(), buf.size(), device_id, err, errlen);
}

void zb3d_pilot_free(zb3d_pilot *p) { delete p; }

void zb3d_pilot_describe(const zb3d_pilot *p, int *width, int *layers, int *gate_levels) {
    if (width) *width = p ? p->width : 0;
    if (layers) *layers = p ? p->layers : 0;
    if (gate_levels) *gate_levels = p ? (int)p->gate.size() : 0;
}

int zb3d_pilot_gate_level(const zb3d_pilot *p, int i, float *sigma, int *width, int *height, float *delta_db) {
    if (!p || i < 0 || i >= (int)p->gate.size()) return -1;
    if (sigma) *sigma = p->gate[i].sigma;
    if (width) *width = p->gate[i].w;
    if (height) *height = p->gate[i].h;
    if (delta_db) *delta_db = p->gate[i].delta;
    return 0;
}

int zb3d_pilot_accepts(const zb3d_pilot *p, float sigma, int width, int height) {
    if (!p || p->gate.empty() || !(sigma >= 0.0f) || width <= 0 || height <= 0) return 0;
    // the calibrated plane size nearest in area (log scale) and, among its levels, the noise
    // level nearest to sigma decide (ties: the smaller size, the lower level)
    const double la = std::log2((double)width * height);
    size_t best = 0;
    for (size_t i = 1; i < p->gate.size(); ++i) {
        const auto &a = p->gate[i], &b = p->gate[best];
        const double da = std::fabs(std::log2((double)a.w * a.h) - la), db = std::fabs(std::log2((double)b.w * b.h) - la);
        const double sa = std::fabs(a.sigma - sigma), sb = std::fabs(b.sigma - sigma);
        const double aa = (double)a.w * a.h, ab = (double)b.w * b.h;
        if (da < db || (da == db && (aa < ab || (aa == ab && (sa < sb || (sa == sb && a.sigma < b.sigma))))))
            best = i;
    }
    return p->gate[best].delta >= -p->tol ? 1 : 0;
}

size_t zb3d_pilot_workspace_bytes(const zb3d_pilot *p, int width, int height) {
    if (!p || width <= 0 || height <= 0) return 0;
    const size_t px = (size_t)width * height;
    // the packed input (16 channels) and two ping-pong activations (width channels), BF16
    return align256(px * 16 * 2) + 2 * align256(px * (size_t)p->width * 2);
}

int zb3d_pilot_run(const zb3d_pilot *p, const float *d_noisy, int width, int height, int pitch, float sigma,
                   float *d_out, int out_pitch, void *d_workspace, int *d_status, void *stream) {
    if (!p || !d_noisy || !d_out || !d_workspace || width <= 0 || height <= 0) return -1;
    if (pitch <= 0) pitch = width;
    if (out_pitch <= 0) out_pitch = width;
    if (pitch < width || out_pitch < width || (reinterpret_cast<uintptr_t>(d_workspace) & 255)) return -1;
    const cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t px = (size_t)width * height;
    char *ws = static_cast<char *>(d_workspace);
    void *x0 = ws;
    void *act[2] = {ws + align256(px * 16 * 2), ws + align256(px * 16 * 2) + align256(px * (size_t)p->width * 2)};
    if (zb::pilot_pack_input(d_noisy, 0, pitch, nullptr, sigma, 1, height, width, p->level_scale, x0, st) !=
        cudaSuccess)
        return -1;
    const void *x = x0;
    const int last = (int)p->shapes.size() - 1;
    for (int l = 0; l <= last; ++l) {
        const int cin = p->shapes[l].first, cout = p->shapes[l].second;
        cudaError_t e;
        if (l < last) {
            e = zb::pilot_conv_tc(x, 1, height, width, cin, p->w16[l], p->b32[l], cout, 1, act[l & 1], nullptr, 0, 0,
                                  nullptr, 0, 0, d_status, st);
            x = act[l & 1];
        } else {
            // channel 0 of the last layer plus the noisy plane: the pilot estimate
            e = zb::pilot_conv_tc(x, 1, height, width, cin, p->w16[l], p->b32[l], cout, 0, nullptr, d_out, 0,
                                  out_pitch, d_noisy, 0, pitch, d_status, st);
        }
        if (e != cudaSuccess) return -1;
    }
    return 0;
}

}  // extern "C"
