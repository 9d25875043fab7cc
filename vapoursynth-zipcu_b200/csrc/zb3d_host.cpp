// zb3d host: argument validation, plane entries, stream-slot pool, device frame
// caches, host<->device staging, and the C ABI of include/zb3d.h.
//
// Mirrors the filter host of vszipcu (src/bm3d.zig, src/pool.zig,
// src/framecache.zig) in C++ over the CUDA runtime: the kernels are compiled
// ahead of time for sm_100a, so there is no NVRTC step and one kernel serves
// every frame size and option set.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cfloat>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <sys/stat.h>
#include <map>
#include <thread>
#include <tuple>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/zb3d.h"
#include "zb3d_args.h"

namespace zb {

cudaError_t launch_match(MatchArgs a, int metric, int rows_per_cta, bool use_tiled, cudaStream_t st);
bool tc_eligible(const MatchArgs &a);
cudaError_t launch_match_tc(const MatchArgs &a, cudaStream_t st);
cudaError_t launch_tc_fallback(MatchArgs a, cudaStream_t st);
int tc_debug_cols(const MatchArgs &a);
int pilot_device(const zb3d_pilot *p);
size_t match_tile_bytes(const MatchArgs &a, int rows_per_cta);
size_t match_tile2_bytes_rows(const MatchArgs &a, int rows_per_cta);
size_t batch_match_smem(const MatchArgs &m);
size_t batch_filter_smem(bool final_);
cudaError_t launch_batch(BatchArgs b, bool final_, int t2d, int t1d, size_t match_smem, size_t filter_smem,
                         cudaStream_t st);
cudaError_t launch_clamped_column(MatchArgs a, cudaStream_t st);
cudaError_t filter_precision_init(int dev);
size_t filter_precision_stack_floats(long long nblocks);
cudaError_t launch_filter_precision(const FilterArgs &a, bool final_, float *stack, float *basic, float *weight,
                                    int *status, cudaStream_t st);
cudaError_t launch_filter(const FilterArgs &a, bool final_, int t2d, int t1d, cudaStream_t st);
cudaError_t launch_finish(const unsigned long long *num, const unsigned long long *den, long long acc_plane_stride,
                          long long acc_frame_stride, int w, int h, int pitch, int nplanes, int tw,
                          unsigned proc_mask, float *dst, int dst_pitch, long long dst_plane_stride, int mode,
                          cudaStream_t st);
cudaError_t launch_vagg(const float *const *stacks, const int *z, int tw, int w, int h, int pitch, int nplanes,
                        unsigned proc_mask, float *dst, int dst_pitch, long long dst_plane_stride, cudaStream_t st);

namespace {

constexpr float kFltEpsilon = 1.19209290e-7f;
constexpr int kMaxRadius = 16;
constexpr int kMaxTw = 2 * kMaxRadius + 1;

void set_err(char *err, size_t n, const char *fmt, ...) {
    if (!err || n == 0) return;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, n, fmt, ap);
    va_end(ap);
}

bool eq_lower(const char *s, const char *lit) {
    size_t n = strlen(lit);
    if (strlen(s) != n) return false;
    for (size_t i = 0; i < n; ++i)
        if (std::tolower((unsigned char)s[i]) != lit[i]) return false;
    return true;
}

int parse_metric(const char *s) {
    if (eq_lower(s, "ssd")) return M_SSD;
    if (eq_lower(s, "sad")) return M_SAD;
    if (eq_lower(s, "zssd")) return M_ZSSD;
    if (eq_lower(s, "zsad")) return M_ZSAD;
    if (eq_lower(s, "ssd/norm")) return M_SSD_NORM;
    return -1;
}

int parse_transform(const char *s) {
    if (eq_lower(s, "dct")) return 0;
    if (eq_lower(s, "haar")) return 1;
    if (eq_lower(s, "wht")) return 2;
    if (eq_lower(s, "bior1.5")) return 3;
    return -1;
}

float f32_from_bits(uint32_t b) {
    float f;
    memcpy(&f, &b, 4);
    return f;
}

// per-plane array with the reference's fallback rule (src/bm3d.zig:953-963)
template <class T>
void per_plane(const T *given, int n, T base, T out[3]) {
    for (int i = 0; i < 3; ++i) out[i] = i < n ? given[i] : (i == 0 ? base : out[i - 1]);
}

int pick(int v, int dflt) { return v == ZB3D_UNSET ? dflt : v; }

int round_up(int v, int m) { return (v + m - 1) / m * m; }

// ---------------------------------------------------------------------------
// Device LRU cache with all-or-nothing claims.  A request claims every key it
// needs at once or waits without holding anything, so requests never deadlock
// while the capacity covers one request per concurrent caller.
// ---------------------------------------------------------------------------
class DevCache {
  public:
    struct Slot {
        long long key = -1;
        void *buf = nullptr;
        cudaEvent_t ev = nullptr;
        int refs = 0;
        unsigned long long stamp = 0;
        bool ready = false;
    };

    ~DevCache() { clear(); }

    bool init(size_t bytes, int n) {
        slots_.resize(n);
        for (auto &s : slots_) {
            if (cudaMalloc(&s.buf, bytes) != cudaSuccess) return false;
            if (cudaEventCreateWithFlags(&s.ev, cudaEventDisableTiming) != cudaSuccess) return false;
        }
        return true;
    }

    void clear() {
        for (auto &s : slots_) {
            if (s.buf) cudaFree(s.buf);
            if (s.ev) cudaEventDestroy(s.ev);
        }
        slots_.clear();
    }

    void *buf(int i) { return slots_[i].buf; }
    cudaEvent_t ev(int i) { return slots_[i].ev; }

    // keys must be distinct; load[i] tells the caller to fill and publish slot idx[i]
    void acquire(const long long *keys, int n, int *idx, bool *load) {
        std::unique_lock<std::mutex> lk(mu_);
        for (;;) {
            bool busy = false;
            for (int k = 0; k < n && !busy; ++k)
                for (auto &s : slots_)
                    if (s.key == keys[k] && !s.ready) {
                        busy = true;
                        break;
                    }
            if (busy) {
                cv_.wait(lk);
                continue;
            }
            int claimed = 0;
            for (; claimed < n; ++claimed) {
                int found = -1;
                load[claimed] = false;
                for (int i = 0; i < (int)slots_.size(); ++i)
                    if (slots_[i].key == keys[claimed]) {
                        found = i;
                        break;
                    }
                if (found < 0) {
                    for (int i = 0; i < (int)slots_.size(); ++i) {
                        if (slots_[i].refs) continue;
                        bool mine = false;
                        for (int j = 0; j < claimed; ++j) mine |= idx[j] == i;
                        if (mine) continue;
                        if (found < 0 || slots_[i].stamp < slots_[found].stamp) found = i;
                    }
                    if (found < 0) break;
                    slots_[found].key = keys[claimed];
                    slots_[found].ready = false;
                    load[claimed] = true;
                }
                idx[claimed] = found;
                slots_[found].refs += 1;
                slots_[found].stamp = ++clock_;
            }
            if (claimed == n) return;
            for (int j = 0; j < claimed; ++j) {
                slots_[idx[j]].refs -= 1;
                if (load[j]) slots_[idx[j]].key = -1;
            }
            cv_.notify_all();
            cv_.wait(lk);
        }
    }

    void publish(int i) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            slots_[i].ready = true;
        }
        cv_.notify_all();
    }

    void abandon(int i) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (!slots_[i].ready) slots_[i].key = -1;
        }
        cv_.notify_all();
    }

    void release(const int *idx, int n) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (int k = 0; k < n; ++k) slots_[idx[k]].refs -= 1;
        }
        cv_.notify_all();
    }

  private:
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<Slot> slots_;
    unsigned long long clock_ = 0;
};

}  // namespace

struct Entry {
    int w, h, pitch;
    int nplanes;
    int planes[3];
    float sigma[3];        // scaled (the filter's step)
    float sigma_basic[3];  // scaled with the step-1 factor (the plain step 1 of the pilot form)
    float sigma_raw[3];    // as given (8-bit scale)
    bool pilot_step1 = false;  // pilot form: the pilot makes this entry's step 1 (else the plain step 1)
    int bs, range, ps_num, ps_range;
    unsigned proc_mask;
    int metric, t2d, t1d;
    int nbx, nby, nbx_al;
    long long nblocks;
    size_t plane_elems;            // h * pitch
    size_t src_off, src_elems;     // window layout [clips][planes][tw][h][pitch]
    size_t dst_off, dst_elems;     // window output: [planes][h][pitch], stacked [planes][tw][2][h][pitch] if r > 0
    size_t out_off;                // BM3Dv2 temporal frame output [planes][h][pitch]
    size_t frame_off;              // offset inside one cached source frame [clips][entry planes][h][pitch]
    int form = 0;                  // block matching: 0 FP32 scan, 1 tensor-core bound + exact re-rank
    int rows = 4;                  // block rows per CTA of the tiled FP32 matchers
};

// Device scratch of one in-flight frame (the reference's per-stream slot).
struct Slot {
    cudaStream_t st = nullptr, cst = nullptr;
    cudaEvent_t ev_up = nullptr;
    float *d_src = nullptr, *d_dst = nullptr;
    unsigned long long *num = nullptr, *den = nullptr;
    int2 *list = nullptr;
    float *errs = nullptr;
    int *tc_ws = nullptr;                    // tensor-core form: fallback list
    unsigned long long *tc_stats = nullptr;  // tensor-core form: counters
    float *h_stage = nullptr;
    size_t stage_up = 0, stage_down = 0;
    void *pilot_ws = nullptr;         // pilot form: the network's activations
    int *dev_status = nullptr;        // tensor-core pipelines (pilot, precision filter): wait status (device)
    int *h_dev_status = nullptr;      // its page-locked read-back
    float *pf_stack = nullptr, *pf_basic = nullptr, *pf_weight = nullptr;  // precision filter stacks

    void destroy() {
        if (st) cudaStreamDestroy(st);
        if (cst) cudaStreamDestroy(cst);
        if (ev_up) cudaEventDestroy(ev_up);
        cudaFree(d_src);
        cudaFree(d_dst);
        cudaFree(num);
        cudaFree(den);
        cudaFree(list);
        cudaFree(errs);
        cudaFree(tc_ws);
        cudaFree(tc_stats);
        cudaFree(pilot_ws);
        cudaFree(dev_status);
        cudaFree(pf_stack);
        cudaFree(pf_basic);
        cudaFree(pf_weight);
        if (h_stage) cudaFreeHost(h_stage);
        if (h_dev_status) cudaFreeHost(h_dev_status);
        *this = Slot();
    }
};

struct Filter {
    // configuration
    zb3d_video_info vi{};
    zb3d_video_info vi_out{};
    bool v2 = false, passthrough = false;
    bool final_ = false, chroma = false, fused = false, zero_init = true;
    int match_form = -1;           // -1: chosen per entry by the autotuner; 0 / 1: forced
    int filter_form = 0;           // 0: FP32 SIMT transforms (bitwise); 1: tensor-core TF32-split 2D transforms
    const zb3d_pilot *pilot = nullptr;  // pilot form (BM3Dv2 two-pass in one call), not owned
    size_t pilot_ws_bytes = 0;
    int radius = 0, tw = 1;
    int nclips = 1;
    float extractor = 0.0f;
    bool process[3] = {false, false, false};
    int device = 0;
    int num_streams = 4;
    std::vector<Entry> entries;
    size_t sum_src = 0, sum_dst = 0, sum_out = 0, frame_elems = 0;
    size_t acc_elems = 0;          // largest entry accumulator (planes * tw * h * pitch)
    long long max_blocks = 0;

    // slot pool (src/pool.zig)
    std::vector<Slot> slots;
    std::vector<int> free_slots;
    std::mutex pool_mu;
    std::condition_variable pool_cv;

    // temporal caches (src/framecache.zig): source frames and accumulator stacks
    DevCache src_cache, acc_cache;

    // CUDA graphs of whole windows / entries, captured once per buffer pair and replayed
    std::mutex graph_mu;
    std::map<std::tuple<const void *, const void *, int>, cudaGraphExec_t> graphs;
    bool graphs_ok = true;

    // optional launch timing (zb3d_profile_enable)
    bool profile = false;
    std::mutex prof_mu;
    std::vector<cudaEvent_t> prof_match, prof_filter;  // start/stop pairs

    bool stacked_out() const { return radius > 0 && !v2; }
    // output of one window (one centre): stacked accumulators when radius > 0
    size_t dst_entry_elems(const Entry &e) const {
        return radius > 0 ? (size_t)e.nplanes * tw * 2 * e.plane_elems : (size_t)e.nplanes * e.plane_elems;
    }
};

namespace {

int acquire_slot(Filter *f) {
    std::unique_lock<std::mutex> lk(f->pool_mu);
    f->pool_cv.wait(lk, [&] { return !f->free_slots.empty(); });
    int s = f->free_slots.back();
    f->free_slots.pop_back();
    return s;
}

void release_slot(Filter *f, int s) {
    {
        std::lock_guard<std::mutex> lk(f->pool_mu);
        f->free_slots.push_back(s);
    }
    f->pool_cv.notify_one();
}

bool alloc_slot(Filter *f, Slot &s) {
    auto ok = [](cudaError_t e) { return e == cudaSuccess; };
    const size_t src = f->sum_src;
    const size_t dst = std::max(f->sum_dst, f->sum_out);
    if (!ok(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking))) return false;
    if (!ok(cudaStreamCreateWithFlags(&s.cst, cudaStreamNonBlocking))) return false;
    if (!ok(cudaEventCreateWithFlags(&s.ev_up, cudaEventDisableTiming))) return false;
    if (!ok(cudaMalloc(&s.d_src, src * sizeof(float)))) return false;
    if (!ok(cudaMalloc(&s.d_dst, dst * sizeof(float)))) return false;
    if (!ok(cudaMalloc(&s.num, f->acc_elems * 8))) return false;
    if (!ok(cudaMalloc(&s.den, f->acc_elems * 8))) return false;
    if (!ok(cudaMalloc(&s.list, f->max_blocks * 8 * sizeof(int2)))) return false;
    if (f->radius > 0 && !ok(cudaMalloc(&s.errs, f->max_blocks * 8 * sizeof(float)))) return false;
    if (f->match_form != 0) {
        if (!ok(cudaMalloc(&s.tc_ws, (kTcWsList + f->max_blocks) * sizeof(int)))) return false;
        if (!ok(cudaMalloc(&s.tc_stats, 4 * sizeof(unsigned long long)))) return false;
        if (!ok(cudaMemset(s.tc_stats, 0, 4 * sizeof(unsigned long long)))) return false;
    }
    if (f->pilot && f->pilot_ws_bytes && !ok(cudaMalloc(&s.pilot_ws, f->pilot_ws_bytes))) return false;
    if (f->filter_form == 1) {
        const size_t fl = filter_precision_stack_floats(f->max_blocks);
        if (!ok(cudaMalloc(&s.pf_stack, fl * sizeof(float)))) return false;
        if (f->final_ && !ok(cudaMalloc(&s.pf_basic, fl * sizeof(float)))) return false;
        if (!ok(cudaMalloc(&s.pf_weight, (size_t)f->max_blocks * sizeof(float)))) return false;
    }
    if (f->pilot || f->filter_form == 1) {
        if (!ok(cudaMalloc(&s.dev_status, sizeof(int)))) return false;
        if (!ok(cudaMemset(s.dev_status, 0, sizeof(int)))) return false;
        if (!ok(cudaHostAlloc((void **)&s.h_dev_status, sizeof(int), cudaHostAllocDefault))) return false;
        *s.h_dev_status = 0;
    }
    s.stage_up = f->v2 && f->radius > 0 ? f->frame_elems : src;
    s.stage_down = dst;
    if (!ok(cudaHostAlloc((void **)&s.h_stage, (s.stage_up + s.stage_down) * sizeof(float), cudaHostAllocDefault)))
        return false;
    return true;
}

// Block matching of one entry into the slot's match list.
cudaError_t run_match(Filter *f, Slot &s, const Entry &en, const float *src) {
        MatchArgs ma{};
        ma.frames = src;  // clip 0, plane 0: the matching plane of every window frame
        ma.fstride = (long long)en.plane_elems;
        ma.w = en.w;
        ma.h = en.h;
        ma.pitch = en.pitch;
        ma.bs = en.bs;
        ma.range = en.range;
        ma.radius = f->radius;
        ma.ps_num = en.ps_num;
        ma.ps_range = en.ps_range;
        ma.nbx = en.nbx;
        ma.nby = en.nby;
        ma.nbx_al = en.nbx_al;
        ma.list = s.list;
        ma.errs = f->radius > 0 ? s.errs : nullptr;
        ma.tc_ws = en.form == 1 ? s.tc_ws : nullptr;  // null: the FP32 scan
        ma.tc_stats = s.tc_stats;
        const int rows = en.rows;
        bool tiled = (en.bs == 4 || en.bs == 8);
        if (tiled) {
            MatchArgs t = ma;
            t.chunks = (2 * en.range + 1 + 3) / 4;
            t.tile_pitch = 128 + 4 * t.chunks;
            tiled = match_tile_bytes(t, rows) <= 200 * 1024;
        }
        return launch_match(ma, en.metric, rows, tiled, s.st);
}

// ---- autotuner: per-entry matching configuration -----------------------------
// Replaces the reference's per-configuration module cache (src/bm3d.zig:57-70,
// 780-835): kernels here are compiled ahead of time, so what is cached is the
// fastest launch configuration of the matching stage for a plane geometry,
// timed on this GPU.  Every candidate gives bit-identical lists, so the choice
// never changes results.  Cache file: $ZB3D_TUNE_CACHE, else
// $XDG_CACHE_HOME/zb3d/tune-v2.txt or ~/.cache/zb3d/tune-v2.txt; one line per key
// "key form rows".  ZB3D_AUTOTUNE=0 turns the timing off (defaults are used).
struct TuneCache {
    std::mutex mu;
    bool loaded = false;
    std::string path;
    std::map<std::string, std::pair<int, int>> best;
};

TuneCache &tune_cache() {
    static TuneCache *c = new TuneCache();
    return *c;
}

std::string tune_path() {
    const char *p = getenv("ZB3D_TUNE_CACHE");
    if (p && *p) return p;
    const char *x = getenv("XDG_CACHE_HOME");
    if (x && *x) return std::string(x) + "/zb3d/tune-v2.txt";
    const char *h = getenv("HOME");
    if (h && *h) return std::string(h) + "/.cache/zb3d/tune-v2.txt";
    return "";
}

void tune_load(TuneCache &c) {
    c.loaded = true;
    c.path = tune_path();
    if (c.path.empty()) return;
    FILE *fp = fopen(c.path.c_str(), "r");
    if (!fp) return;
    char key[256];
    int form, rows;
    while (fscanf(fp, "%255s %d %d", key, &form, &rows) == 3) c.best[key] = {form, rows};
    fclose(fp);
}

void tune_store(TuneCache &c, const std::string &key, int form, int rows) {
    c.best[key] = {form, rows};
    if (c.path.empty()) return;
    const size_t cut = c.path.find_last_of('/');
    if (cut != std::string::npos) {
        const std::string dir = c.path.substr(0, cut), parent = dir.substr(0, dir.find_last_of('/'));
        mkdir(parent.c_str(), 0755);
        mkdir(dir.c_str(), 0755);
    }
    FILE *fp = fopen(c.path.c_str(), "a");
    if (!fp) return;
    fprintf(fp, "%s %d %d\n", key.c_str(), form, rows);
    fclose(fp);
}

// Whether the packed SSD kernel's tile for `rows` block rows per CTA fits (that kernel
// takes up to 8 warps; the other tiled kernels take at most 4).
bool tiled2_rows_fit(const Entry &e, int rows) {
    if (e.metric != M_SSD || (e.bs != 4 && e.bs != 8)) return false;
    MatchArgs t{};
    t.bs = e.bs;
    t.range = e.range;
    t.chunks = (2 * e.range + 1 + 3) / 4;
    t.tile_pitch = 128 + 4 * t.chunks;
    return match_tile2_bytes_rows(t, rows) <= 200 * 1024;
}

// Chooses e.form / e.rows: FP32 scan with 2 or 4 block rows per CTA (tiled block
// steps 4 and 8), also 8 for the packed SSD kernel, or the tensor-core form (ssd,
// where eligible), by timing
// each on a synthetic plane of the entry's geometry with slot s's buffers.
void tune_entry(Filter *f, Slot &s, Entry &e) {
    e.rows = 4;
    MatchArgs ga{};
    ga.w = e.w;
    ga.h = e.h;
    ga.bs = e.bs;
    ga.range = e.range;
    const bool tc_ok = e.metric == M_SSD && f->match_form != 0 && s.tc_ws != nullptr && tc_eligible(ga);
    const bool tiled = e.bs == 4 || e.bs == 8;
    e.form = (f->match_form == 1 && tc_ok) ? 1 : 0;
    std::vector<std::pair<int, int>> cands;
    if (f->match_form != 1 || !tc_ok) {
        if (tiled)
            for (int r : {2, 4}) cands.push_back({0, r});
        if (tiled2_rows_fit(e, 8)) cands.push_back({0, 8});
    }
    if (tc_ok && f->match_form != 0) cands.push_back({1, 4});
    if (cands.size() < 2) return;
    const char *off = getenv("ZB3D_AUTOTUNE");
    if (off && strcmp(off, "0") == 0) return;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, f->device) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    char key[256];
    snprintf(key, sizeof key, "sm%d%d-%dsm_w%d_h%d_p%d_bs%d_R%d_m%d_r%d_c%d_f%d", prop.major, prop.minor,
             prop.multiProcessorCount, e.w, e.h, e.pitch, e.bs, e.range, e.metric, f->radius, f->nclips,
             f->match_form);
    TuneCache &c = tune_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    if (!c.loaded || tune_path() != c.path) {  // first use, or the cache file was redirected
        c.best.clear();
        tune_load(c);
    }
    auto it = c.best.find(key);
    if (it != c.best.end()) {
        const int form = it->second.first, rows = it->second.second;
        if ((form == 0 && (rows == 2 || rows == 4 || (rows == 8 && tiled2_rows_fit(e, 8)))) || (form == 1 && tc_ok)) {
            e.form = form;
            e.rows = rows;
        }
        return;
    }
    // synthetic plane in [0, 1]: gradient, a texture and uniform noise, in every window frame
    std::vector<float> host((size_t)e.h * e.pitch, 0.0f);
    unsigned st = 0x9e3779b9u;
    for (int y = 0; y < e.h; ++y)
        for (int x = 0; x < e.w; ++x) {
            st = st * 1664525u + 1013904223u;
            const float noise = ((st >> 8) * (1.0f / 16777216.0f) - 0.5f) * 0.08f;
            host[(size_t)y * e.pitch + x] = 0.25f + 0.25f * (x + y) / (float)(e.w + e.h) +
                                            0.1f * sinf(0.37f * x + 0.21f * y) + noise;
        }
    cudaEvent_t a = nullptr, b = nullptr;
    bool ok = cudaEventCreate(&a) == cudaSuccess && cudaEventCreate(&b) == cudaSuccess;
    for (int t = 0; ok && t < f->tw; ++t)
        ok = cudaMemcpy(s.d_src + e.src_off + (size_t)t * e.plane_elems, host.data(), host.size() * sizeof(float),
                        cudaMemcpyHostToDevice) == cudaSuccess;
    float best_ms = 3.0e38f;
    int bform = -1, brows = e.rows;
    for (const auto &cand : cands) {
        if (!ok) break;
        Entry t = e;
        t.form = cand.first;
        t.rows = cand.second;
        float lo = 3.0e38f;
        bool good = true;
        for (int it2 = 0; it2 < 4 && good; ++it2) {
            good = cudaEventRecord(a, s.st) == cudaSuccess &&
                   run_match(f, s, t, s.d_src + e.src_off) == cudaSuccess && cudaEventRecord(b, s.st) == cudaSuccess &&
                   cudaEventSynchronize(b) == cudaSuccess;
            float ms = 0.0f;
            if (good && cudaEventElapsedTime(&ms, a, b) == cudaSuccess && it2 > 0) lo = std::min(lo, ms);
        }
        if (!good) {  // a configuration that cannot launch here is skipped
            cudaGetLastError();
            continue;
        }
        if (lo < best_ms) {
            best_ms = lo;
            bform = cand.first;
            brows = cand.second;
        }
    }
    ok = ok && bform >= 0;
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    if (s.tc_stats) cudaMemset(s.tc_stats, 0, 4 * sizeof(unsigned long long));
    if (!ok) {
        cudaGetLastError();
        return;
    }
    e.form = bform;
    e.rows = brows;
    tune_store(c, key, bform, brows);
}

cudaEvent_t prof_event(Filter *f, std::vector<cudaEvent_t> &v, cudaStream_t st) {
    cudaEvent_t ev = nullptr;
    if (cudaEventCreate(&ev) != cudaSuccess) return nullptr;
    cudaEventRecord(ev, st);
    std::lock_guard<std::mutex> lk(f->prof_mu);
    v.push_back(ev);
    return ev;
}

// Runs every entry of one window (d_src, entry layout) into d_dst on the slot's stream.
cudaError_t run_entry(Filter *f, Slot &s, const Entry &en, const float *src, float *dst, bool basic = false);
cudaError_t run_entry_steps(Filter *f, Slot &s, const Entry &en, const float *src, float *dst);

// Runs `fn(s)` (launches on s.st) as a CUDA graph: captured once per key on the slot's
// own stream, then replayed on `launch`.  A window's whole launch sequence (memsets,
// matching, filtering, finishing of every plane) becomes one graph launch.  Graphs bake
// in the slot's scratch buffers, so replays of one key must not overlap (the device
// entry points' rule).  ZB3D_GRAPHS=0, profiling, or a failed capture -> direct launches.
template <class Fn>
cudaError_t run_graphed(Filter *f, Slot &s, std::tuple<const void *, const void *, int> key, cudaStream_t launch,
                        Fn fn) {
    static const bool env_off = [] {
        const char *v = getenv("ZB3D_GRAPHS");
        return v && strcmp(v, "0") == 0;
    }();
    if (env_off || f->profile || !f->graphs_ok) {
        Slot d = s;
        d.st = launch;
        return fn(d);
    }
    cudaGraphExec_t exec = nullptr;
    {
        std::lock_guard<std::mutex> lk(f->graph_mu);
        auto it = f->graphs.find(key);
        if (it != f->graphs.end()) exec = it->second;
    }
    if (!exec) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(s.st, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const cudaError_t e1 = fn(s);
            e = cudaStreamEndCapture(s.st, &g);
            if (e1 != cudaSuccess) e = e1;
            if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
            if (g) cudaGraphDestroy(g);
        }
        if (e != cudaSuccess) {  // not capturable here: launch directly from now on
            cudaGetLastError();
            if (exec) cudaGraphExecDestroy(exec);
            f->graphs_ok = false;
            Slot d = s;
            d.st = launch;
            return fn(d);
        }
        std::lock_guard<std::mutex> lk(f->graph_mu);
        if (f->graphs.size() >= 256) {  // bounded: drop everything, re-capture on demand
            for (auto &kv : f->graphs) cudaGraphExecDestroy(kv.second);
            f->graphs.clear();
        }
        f->graphs[key] = exec;
    }
    return cudaGraphLaunch(exec, launch);
}

cudaError_t run_window(Filter *f, Slot &s, const float *d_src, float *d_dst) {
    for (const Entry &en : f->entries) {
        cudaError_t e = run_entry_steps(f, s, en, d_src + en.src_off, d_dst + en.dst_off);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// One entry with, in the pilot form, its step 1 first: the pilot (or the plain step 1
// where the gate refused the entry's sigma) writes the reference planes (clip 0 of the
// entry's block) from the noisy planes (clip 1); then step 2 runs as with a ref clip.
cudaError_t run_entry_steps(Filter *f, Slot &s, const Entry &en, const float *src, float *dst) {
    if (f->pilot) {
        float *ref = const_cast<float *>(src);  // clip 0: [planes][h][pitch] (radius 0)
        const float *noisy = src + (size_t)en.nplanes * en.plane_elems;
        cudaError_t e = cudaSuccess;
        if (en.pilot_step1) {
            for (int i = 0; i < en.nplanes && e == cudaSuccess; ++i) {
                if (!((en.proc_mask >> i) & 1)) continue;
                if (zb3d_pilot_run(f->pilot, noisy + (size_t)i * en.plane_elems, en.w, en.h, en.pitch,
                                   en.sigma_raw[i], ref + (size_t)i * en.plane_elems, en.pitch, s.pilot_ws,
                                   s.dev_status, s.st) != 0)
                    e = cudaErrorLaunchFailure;
            }
        } else {
            e = run_entry(f, s, en, noisy, ref, true);
        }
        if (e != cudaSuccess) return e;
    }
    return run_entry(f, s, en, src, dst);
}

// One entry: src = its [clips][planes][tw][h][pitch] block, dst = its output block.
// basic: the plain step 1 of the pilot form (hard threshold, step-1 sigma) on the noisy
// planes at src (one clip), written to dst as [planes][h][pitch].
cudaError_t run_entry(Filter *f, Slot &s, const Entry &en, const float *src, float *dst, bool basic) {
    cudaError_t e = cudaSuccess;
    {
        const size_t acc = (size_t)en.nplanes * f->tw * en.plane_elems;
        if ((e = cudaMemsetAsync(s.num, 0, acc * 8, s.st)) != cudaSuccess) return e;
        if ((e = cudaMemsetAsync(s.den, 0, acc * 8, s.st)) != cudaSuccess) return e;
        if (f->profile) prof_event(f, f->prof_match, s.st);
        if ((e = run_match(f, s, en, src)) != cudaSuccess) return e;
        if (f->profile) prof_event(f, f->prof_match, s.st);
        FilterArgs fa{};
        fa.src = src;
        fa.plane_stride = (long long)f->tw * en.plane_elems;
        fa.clip_stride = (long long)en.nplanes * fa.plane_stride;
        fa.frame_stride = (long long)en.plane_elems;
        fa.w = en.w;
        fa.h = en.h;
        fa.pitch = en.pitch;
        fa.nplanes = en.nplanes;
        fa.chroma = f->chroma;
        fa.list = s.list;
        fa.nblocks = (int)en.nblocks;
        for (int i = 0; i < 3; ++i) fa.sigma[i] = basic ? en.sigma_basic[i] : en.sigma[i];
        fa.extractor = f->extractor;
        fa.num = s.num;
        fa.den = s.den;
        fa.acc_frame_stride = (long long)en.plane_elems;
        fa.acc_plane_stride = (long long)f->tw * en.plane_elems;
        if (f->profile) prof_event(f, f->prof_filter, s.st);
        if (f->filter_form == 1)
            e = launch_filter_precision(fa, f->final_ && !basic, s.pf_stack, s.pf_basic, s.pf_weight, s.dev_status,
                                        s.st);
        else
            e = launch_filter(fa, f->final_ && !basic, en.t2d, en.t1d, s.st);
        if (e != cudaSuccess) return e;
        if (f->profile) prof_event(f, f->prof_filter, s.st);
        if (f->radius == 0) {
            e = launch_finish(s.num, s.den, fa.acc_plane_stride, fa.acc_frame_stride, en.w, en.h, en.pitch,
                              en.nplanes, 1, en.proc_mask, dst, en.pitch, (long long)en.plane_elems, 0, s.st);
        } else {
            e = launch_finish(s.num, s.den, fa.acc_plane_stride, fa.acc_frame_stride, en.w, en.h, en.pitch,
                              en.nplanes, f->tw, en.proc_mask, dst, en.pitch,
                              (long long)f->tw * 2 * en.plane_elems, 1, s.st);
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Host threads for the staging copies of pageable frames.  A plane's rows are split over
// them (the caller takes a share too), so one frame's copy draws on several cores' memory
// bandwidth.  ZB3D_COPY_THREADS sets the count (default: half the hardware threads, at
// most 8; 0 = copies on the calling thread only).  The pool lives for the process.
class CopyPool {
public:
    static CopyPool &get() {
        static CopyPool *p = new CopyPool();  // never destroyed: workers may be waiting at exit
        return *p;
    }
    int workers() const { return (int)n_; }
    // fn(k) for k in [0, n): tasks 1.. go to the workers, the caller runs task 0 and then
    // helps with any queued task until all n are done
    void run(int n, const std::function<void(int)> &fn) {
        if (n <= 1 || n_ == 0) {
            for (int k = 0; k < n; ++k) fn(k);
            return;
        }
        struct Batch {
            std::mutex mu;
            std::condition_variable cv;
            int left;
        };
        auto b = std::make_shared<Batch>();
        b->left = n;
        auto done = [b] {
            std::lock_guard<std::mutex> lk(b->mu);
            if (--b->left == 0) b->cv.notify_all();
        };
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (int k = 1; k < n; ++k)
                q_.emplace_back([fn, k, done] {
                    fn(k);
                    done();
                });
        }
        cv_.notify_all();
        fn(0);
        done();
        for (;;) {  // help: the queue may hold this batch's tasks while every worker is busy
            std::function<void()> t;
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (q_.empty()) break;
                t = std::move(q_.front());
                q_.pop_front();
            }
            t();
        }
        std::unique_lock<std::mutex> lk(b->mu);
        b->cv.wait(lk, [&] { return b->left == 0; });
    }

private:
    CopyPool() {
        const char *v = getenv("ZB3D_COPY_THREADS");
        unsigned hw = std::thread::hardware_concurrency();
        n_ = v ? (unsigned)std::max(0, atoi(v)) : std::min(8u, std::max(1u, hw / 2));
        for (unsigned i = 0; i < n_; ++i)
            std::thread([this] {
                for (;;) {
                    std::function<void()> t;
                    {
                        std::unique_lock<std::mutex> lk(mu_);
                        cv_.wait(lk, [&] { return !q_.empty(); });
                        t = std::move(q_.front());
                        q_.pop_front();
                    }
                    t();
                }
            }).detach();
    }
    unsigned n_ = 0;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> q_;
};

// Row copies of a plane, split into chunks of at least 1 MiB over the copy pool.
void copy_rows(char *dst, ptrdiff_t dst_stride, const char *src, ptrdiff_t src_stride, size_t row_bytes, int h) {
    CopyPool &pool = CopyPool::get();
    const size_t bytes = row_bytes * (size_t)h;
    const int chunks = (int)std::min<size_t>((size_t)pool.workers() + 1, std::max<size_t>(1, bytes >> 20));
    const int per = (h + chunks - 1) / chunks;
    pool.run(chunks, [&](int k) {
        const int y0 = k * per, y1 = std::min(h, y0 + per);
        for (int y = y0; y < y1; ++y) memcpy(dst + (ptrdiff_t)y * dst_stride, src + (ptrdiff_t)y * src_stride, row_bytes);
    });
}

void copy_plane_in(float *dst, int pitch, const float *src, ptrdiff_t stride_bytes, int w, int h) {
    copy_rows((char *)dst, (ptrdiff_t)pitch * sizeof(float), (const char *)src, stride_bytes, (size_t)w * sizeof(float),
              h);
}

void copy_plane_out(float *dst, ptrdiff_t stride_bytes, const float *src, int pitch, int w, int h) {
    copy_rows((char *)dst, stride_bytes, (const char *)src, (ptrdiff_t)pitch * sizeof(float), (size_t)w * sizeof(float),
              h);
}

int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// Page-locked (cudaHostAlloc'd or registered) host memory: copies to and from
// it are DMA transfers the stream runs asynchronously, with no staging copy.
bool is_pinned(const void *p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

// Pool of page-locked host blocks for zb3d_host_alloc: freed blocks are kept by
// size and reused, so steady-state frame allocation costs no cudaHostAlloc.
struct HostPool {
    std::mutex mu;
    std::multimap<size_t, void *> free_blocks;
    std::map<void *, size_t> sizes;
};
HostPool &host_pool() {
    static HostPool *p = new HostPool();  // never destroyed: frames may outlive static destructors
    return *p;
}

}  // namespace

}  // namespace zb

using zb::Entry;
using zb::Filter;

// ---- batches: one persistent launch over the plane entries of many windows ----

namespace zb {
namespace {

// Scratch of a batch: per-entry match lists and accumulators, the entry table, item
// counters and the status word.  The synchronous call shares one per device (grown on
// demand); a graph handle owns its own.
struct BatchBuffers {
    char *arena = nullptr;
    size_t arena_bytes = 0;
    BatchEntry *h_entries = nullptr;  // page-locked
    size_t h_cap = 0;
    int *h_status = nullptr;          // page-locked
    cudaEvent_t ev_start = nullptr;   // the launching stream at the start of a batch

    void release() {
        cudaFree(arena);
        if (h_entries) cudaFreeHost(h_entries);
        if (h_status) cudaFreeHost(h_status);
        if (ev_start) cudaEventDestroy(ev_start);
        *this = BatchBuffers();
    }
};

struct BatchCtx {
    std::mutex mu;
    BatchBuffers buf;
};

BatchCtx &batch_ctx(int dev) {
    static BatchCtx *ctx = new BatchCtx[64];  // never destroyed: device memory may outlive static destructors
    return ctx[dev];
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

// Entries the batch kernel takes: spatial SSD matching at block_step 4 or 8 on the FP32
// scan with the tiled kernel, radius 0, DCT in both dimensions, no pilot.
bool batch_eligible(const Filter *f, const Entry &en) {
    if (f->pilot || f->filter_form != 0 || f->radius != 0 || en.metric != M_SSD || (en.bs != 4 && en.bs != 8) ||
        en.form != 0)
        return false;
    if (en.t2d != 0 || en.t1d != 0) return false;
    MatchArgs m{};
    m.bs = en.bs;
    m.range = en.range;
    m.chunks = (2 * en.range + 1 + 3) / 4;
    m.tile_pitch = 128 + 4 * m.chunks;
    return match_tile2_bytes_rows(m, kBatchMatchRows) <= 200 * 1024;
}


struct BatchItem {
    int job;
    const Entry *en;
};

// A batch's work list and scratch layout: eligible entries grouped by filter step (hard
// threshold, Wiener), the others run on their own.
struct BatchPlan {
    std::vector<zb3d_batch_job> jobs;
    int device = 0;
    std::vector<BatchItem> groups[2], fallback;
    int nent = 0;
    size_t counters = 0, need = 0;
    std::vector<size_t> list_off, acc_off;
};

bool plan_batch(const zb3d_batch_job *jobs, int njobs, BatchPlan &p, char *err, size_t errlen) {
    if (njobs <= 0 || !jobs) {
        set_err(err, errlen, "zb3d_process_batch: no jobs.");
        return false;
    }
    const Filter *f0 = reinterpret_cast<const Filter *>(jobs[0].filter);
    for (int j = 0; j < njobs; ++j) {
        const Filter *f = reinterpret_cast<const Filter *>(jobs[j].filter);
        if (!f || f->passthrough || f->slots.empty() || !jobs[j].d_src || !jobs[j].d_dst) {
            set_err(err, errlen, "zb3d_process_batch: job %d has no filter to run or no buffers.", j);
            return false;
        }
        if (f->device != f0->device) {
            set_err(err, errlen, "zb3d_process_batch: the jobs' filters are on different devices.");
            return false;
        }
    }
    p.device = f0->device;
    if (p.device < 0 || p.device >= 64) {
        set_err(err, errlen, "zb3d_process_batch: device %d is beyond the 64 devices the batch path serves.",
                p.device);
        return false;
    }
    p.jobs.assign(jobs, jobs + njobs);
    for (int j = 0; j < njobs; ++j) {
        const Filter *f = reinterpret_cast<const Filter *>(jobs[j].filter);
        for (const Entry &en : f->entries) {
            if (batch_eligible(f, en)) p.groups[f->final_ ? 1 : 0].push_back({j, &en});
            else p.fallback.push_back({j, &en});
        }
    }
    // scratch layout: [counters | status | entries | lists | accumulators]
    p.nent = (int)(p.groups[0].size() + p.groups[1].size());
    p.counters = align256(32 + 4 * (size_t)p.nent);
    p.need = p.counters + 256 + align256(sizeof(BatchEntry) * (size_t)std::max(p.nent, 1));
    for (int g = 0; g < 2; ++g)
        for (const BatchItem &it : p.groups[g]) {
            p.list_off.push_back(p.need);
            p.need += align256((size_t)it.en->nblocks * 8 * sizeof(int2));
        }
    for (int g = 0; g < 2; ++g)
        for (const BatchItem &it : p.groups[g]) {
            p.acc_off.push_back(p.need);
            p.need += 2 * align256((size_t)it.en->nplanes * it.en->plane_elems * 8);
        }
    return true;
}

// Scratch of at least the plan's size (grown when smaller; `st` is synchronised first).
bool ensure_buffers(BatchBuffers &b, const BatchPlan &p, cudaStream_t st, char *err, size_t errlen) {
    if (p.need > b.arena_bytes) {
        cudaStreamSynchronize(st);
        cudaFree(b.arena);
        b.arena = nullptr;
        b.arena_bytes = 0;
        if (cudaMalloc(&b.arena, p.need) != cudaSuccess) {
            cudaGetLastError();
            set_err(err, errlen, "zb3d_process_batch: out of device memory (%zu MiB of scratch).", p.need >> 20);
            return false;
        }
        b.arena_bytes = p.need;
    }
    if ((size_t)p.nent > b.h_cap || !b.h_status) {
        cudaStreamSynchronize(st);
        if (b.h_entries) cudaFreeHost(b.h_entries);
        b.h_entries = nullptr;
        b.h_cap = 0;
        const size_t cap = std::max<size_t>(p.nent, 16);
        if (cudaHostAlloc((void **)&b.h_entries, cap * sizeof(BatchEntry), cudaHostAllocDefault) != cudaSuccess ||
            (!b.h_status && cudaHostAlloc((void **)&b.h_status, sizeof(int), cudaHostAllocDefault) != cudaSuccess)) {
            cudaGetLastError();
            set_err(err, errlen, "zb3d_process_batch: out of page-locked host memory.");
            return false;
        }
        b.h_cap = cap;
    }
    if (!b.ev_start && cudaEventCreateWithFlags(&b.ev_start, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        set_err(err, errlen, "zb3d_process_batch: cannot create an event.");
        return false;
    }
    return true;
}

// One slot of each filter whose entries run outside the work list (waits for a free one).
std::map<Filter *, int> hold_slots(const BatchPlan &p) {
    std::map<Filter *, int> held;
    for (const BatchItem &it : p.fallback) {
        Filter *f = reinterpret_cast<Filter *>(p.jobs[it.job].filter);
        if (!held.count(f)) held.emplace(f, acquire_slot(f));
    }
    return held;
}

void release_slots(std::map<Filter *, int> &held) {
    for (auto &h : held) {
        cudaStreamSynchronize(h.first->slots[h.second].st);
        release_slot(h.first, h.second);
    }
    held.clear();
}

// The whole batch on `st`: entries outside the work list on the held slots' streams (after
// what `st` holds so far, joined back at the end), the work-list launches and the finishes,
// then the status word into b.h_status.  Builds the entry table in b.h_entries; with stream
// capture the copy of that table is part of the graph and the table must stay as it is.
cudaError_t enqueue_batch(const BatchPlan &p, BatchBuffers &b, std::map<Filter *, int> &held, unsigned wait_polls,
                          int unsatisfiable, cudaStream_t st) {
    cudaError_t ce = cudaEventRecord(b.ev_start, st);
    for (auto &h : held)
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(h.first->slots[h.second].st, b.ev_start, 0);
    for (const BatchItem &it : p.fallback) {
        if (ce != cudaSuccess) break;
        Filter *f = reinterpret_cast<Filter *>(p.jobs[it.job].filter);
        Slot &s = f->slots[held.at(f)];
        ce = run_entry_steps(f, s, *it.en, p.jobs[it.job].d_src + it.en->src_off, p.jobs[it.job].d_dst + it.en->dst_off);
    }
    char *arena = b.arena;
    unsigned long long *d_next = reinterpret_cast<unsigned long long *>(arena);  // [2][2]: group, kind
    unsigned *d_done = reinterpret_cast<unsigned *>(arena + 32);                 // [nent]
    int *d_status = reinterpret_cast<int *>(arena + p.counters);
    BatchEntry *d_entries = reinterpret_cast<BatchEntry *>(arena + p.counters + 256);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(arena, 0, p.counters + 256, st);
    // accumulators start at zero
    if (ce == cudaSuccess && p.nent > 0) ce = cudaMemsetAsync(arena + p.acc_off[0], 0, p.need - p.acc_off[0], st);
    size_t smem[2] = {0, 0};  // per group: matching tiles
    long long totals[2][2] = {{0, 0}, {0, 0}};  // [group] (match items, all items)
    int idx = 0;
    for (int g = 0; g < 2 && ce == cudaSuccess; ++g) {
        long long nm = 0;
        const int first = idx;
        for (const BatchItem &it : p.groups[g]) {
            const Filter *f = reinterpret_cast<const Filter *>(p.jobs[it.job].filter);
            const Entry &en = *it.en;
            const float *src = p.jobs[it.job].d_src + en.src_off;
            BatchEntry &B = b.h_entries[idx];
            B = BatchEntry{};
            int2 *list = reinterpret_cast<int2 *>(arena + p.list_off[idx]);
            unsigned long long *num = reinterpret_cast<unsigned long long *>(arena + p.acc_off[idx]);
            unsigned long long *den = reinterpret_cast<unsigned long long *>(
                arena + p.acc_off[idx] + align256((size_t)en.nplanes * en.plane_elems * 8));
            MatchArgs &m = B.m;
            m.frames = src;  // clip 0, plane 0: the matching plane
            m.fstride = (long long)en.plane_elems;
            m.w = en.w;
            m.h = en.h;
            m.pitch = en.pitch;
            m.bs = en.bs;
            m.range = en.range;
            m.nbx = en.nbx;
            m.nby = en.nby;
            m.nbx_al = en.nbx_al;
            m.chunks = (2 * en.range + 1 + 3) / 4;
            m.tile_pitch = 128 + 4 * m.chunks;
            m.list = list;
            m.self_incl = 1;
            FilterArgs &fa = B.f;
            fa.src = src;
            fa.plane_stride = (long long)en.plane_elems;
            fa.clip_stride = (long long)en.nplanes * fa.plane_stride;
            fa.frame_stride = (long long)en.plane_elems;
            fa.w = en.w;
            fa.h = en.h;
            fa.pitch = en.pitch;
            fa.nplanes = en.nplanes;
            fa.chroma = f->chroma;
            fa.list = list;
            fa.nblocks = (int)en.nblocks;
            for (int i = 0; i < 3; ++i) fa.sigma[i] = en.sigma[i];
            fa.extractor = f->extractor;
            fa.num = num;
            fa.den = den;
            fa.acc_frame_stride = (long long)en.plane_elems;
            fa.acc_plane_stride = (long long)en.plane_elems;
            const int nbw = en.bs == 4 ? 31 : 16;
            B.tiles_x = (en.nbx_al + nbw - 1) / nbw;
            B.match_items = B.tiles_x * ((en.nby + kBatchMatchRows - 1) / kBatchMatchRows);
            B.filter_items = (int)((en.nblocks + kBatchGroups - 1) / kBatchGroups);
            B.first_match = nm;
            nm += B.match_items;
            smem[g] = std::max(smem[g], batch_match_smem(m));
            // the clamped last column, before the batch launch (the batch's lists are complete
            // when its filter chunks read them)
            if (en.nbx_al != en.nbx && (ce = launch_clamped_column(m, st)) != cudaSuccess) break;
            ++idx;
        }
        long long nf = nm;
        for (int i = first; i < idx; ++i) {
            b.h_entries[i].first_filter = nf;
            nf += b.h_entries[i].filter_items;
        }
        totals[g][0] = nm;
        totals[g][1] = nf;
    }
    if (ce == cudaSuccess && p.nent > 0)
        ce = cudaMemcpyAsync(d_entries, b.h_entries, sizeof(BatchEntry) * (size_t)p.nent, cudaMemcpyHostToDevice, st);
    for (int g = 0, base = 0; g < 2 && ce == cudaSuccess; base += (int)p.groups[g].size(), ++g) {
        if (p.groups[g].empty()) continue;
        BatchArgs a{};
        a.entries = d_entries + base;
        a.nentries = (int)p.groups[g].size();
        a.match_total = totals[g][0];
        a.items_total = totals[g][1];
        a.next = d_next + 2 * g;
        a.match_done = d_done + base;
        a.status = d_status;
        a.wait_polls = wait_polls ? wait_polls : (1u << 22);
        a.unsatisfiable = unsatisfiable && g == (p.groups[0].empty() ? 1 : 0);
        ce = launch_batch(a, g == 1, 0, 0, smem[g], batch_filter_smem(g == 1), st);
        for (int i = 0; i < (int)p.groups[g].size() && ce == cudaSuccess; ++i) {
            const BatchItem &it = p.groups[g][i];
            const Entry &en = *it.en;
            const BatchEntry &B = b.h_entries[base + i];
            ce = launch_finish(B.f.num, B.f.den, B.f.acc_plane_stride, B.f.acc_frame_stride, en.w, en.h, en.pitch,
                               en.nplanes, 1, en.proc_mask, p.jobs[it.job].d_dst + en.dst_off, en.pitch,
                               (long long)en.plane_elems, 0, st);
        }
    }
    for (auto &h : held) {
        if (ce != cudaSuccess) break;
        Slot &s = h.first->slots[h.second];
        ce = cudaEventRecord(s.ev_up, s.st);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(st, s.ev_up, 0);
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(b.h_status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st);
    return ce;
}
}  // namespace
}  // namespace zb

extern "C" {

void zb3d_args_init(zb3d_args *a) {
    memset(a, 0, sizeof *a);
    a->radius = a->chroma = a->device_id = a->num_streams = a->extractor_exp = ZB3D_UNSET;
    a->zero_init = a->fast_fused = a->match_form = a->filter_form = ZB3D_UNSET;
}

const char *zb3d_version(void) { return "zb3d 0.1.0 (sm_100a)"; }

void *zb3d_host_alloc(size_t bytes) {
    zb::HostPool &hp = zb::host_pool();
    const size_t sz = (bytes + 4095) & ~(size_t)4095;
    {
        std::lock_guard<std::mutex> lk(hp.mu);
        auto it = hp.free_blocks.find(sz);
        if (it != hp.free_blocks.end()) {
            void *p = it->second;
            hp.free_blocks.erase(it);
            return p;
        }
    }
    void *p = nullptr;
    if (cudaHostAlloc(&p, sz, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    std::lock_guard<std::mutex> lk(hp.mu);
    hp.sizes[p] = sz;
    return p;
}

void zb3d_host_free(void *p) {
    if (!p) return;
    zb::HostPool &hp = zb::host_pool();
    std::lock_guard<std::mutex> lk(hp.mu);
    auto it = hp.sizes.find(p);
    if (it != hp.sizes.end()) hp.free_blocks.emplace(it->second, p);
}

int zb3d_agg_z(int i, int n, int nframes, int radius) {
    return std::min(std::max(2 * radius - i, n - nframes + 1 + radius), n + radius);
}

static Filter *create_impl(const zb3d_video_info *clip, const zb3d_args *a, int v2, char *err, size_t errlen) {
    using namespace zb;
    zb3d_args dflt;
    if (!a) {
        zb3d_args_init(&dflt);
        a = &dflt;
    }
    std::unique_ptr<Filter> f(new Filter());
    f->vi = *clip;
    f->v2 = v2 != 0;
    const zb3d_video_info &vi = *clip;

    if (f->v2) {
        // BM3Dv2: planes whose sigma is below FLT_EPSILON pass through; all of them -> the clip itself
        bool proc[3] = {true, true, true};
        for (int i = 0; i < 3; ++i) {
            if (i < a->n_sigma)
                proc[i] = !(a->sigma[i] < kFltEpsilon);
            else if (i > 0)
                proc[i] = proc[i - 1];
        }
        bool skip = true;
        for (int i = 0; i < std::min(vi.num_planes, 3); ++i)
            if (proc[i]) skip = false;
        if (skip) {
            f->passthrough = true;
            f->vi_out = vi;
            return f.release();
        }
    }
    if (vi.width <= 0 || vi.height <= 0 || vi.sample_type != ZB3D_FLOAT || vi.bits_per_sample != 32) {
        set_err(err, errlen, "BM3D: only constant format 32 bit float input supported.");
        return nullptr;
    }
    if (a->ref) {
        const zb3d_video_info &r = *a->ref;
        if (r.color_family != vi.color_family || r.sample_type != vi.sample_type ||
            r.bits_per_sample != vi.bits_per_sample || r.subsampling_w != vi.subsampling_w ||
            r.subsampling_h != vi.subsampling_h) {
            set_err(err, errlen, "BM3D: \"ref\" must be of the same format as \"clip\".");
            return nullptr;
        }
        if (r.width != vi.width || r.height != vi.height) {
            set_err(err, errlen, "BM3D: \"ref\" must be of the same dimensions as \"clip\".");
            return nullptr;
        }
        if (r.num_frames != vi.num_frames) {
            set_err(err, errlen, "BM3D: \"ref\" must be of the same number of frames as \"clip\".");
            return nullptr;
        }
        f->final_ = true;
    }
    if (a->pilot) {
        if (!f->v2) {
            set_err(err, errlen, "BM3D: \"pilot\" needs BM3Dv2.");
            return nullptr;
        }
        if (a->ref) {
            set_err(err, errlen, "BM3D: \"pilot\" makes the reference itself; \"ref\" must not be given.");
            return nullptr;
        }
        if (pick(a->radius, 0) != 0) {
            set_err(err, errlen, "BM3D: \"pilot\" needs radius 0.");
            return nullptr;
        }
        if (zb::pilot_device(a->pilot) != pick(a->device_id, 0)) {
            set_err(err, errlen, "BM3D: \"pilot\" was loaded on another device.");
            return nullptr;
        }
        f->pilot = a->pilot;
        f->final_ = true;  // the filter's own step is step 2
    }
    float sigma[3];
    per_plane<float>(a->sigma, a->n_sigma, 3.0f, sigma);
    for (float s : sigma)
        if (!(s >= 0)) {
            set_err(err, errlen, "BM3D: \"sigma\" must be non-negative.");
            return nullptr;
        }
    for (int i = 0; i < 3; ++i) f->process[i] = !(sigma[i] < kFltEpsilon);
    // f32(2.7*0.75*64/255) / f32(0.75*64/255) as the reference stores them (src/bm3d.zig:1019-1024)
    const float factor = f->final_ ? f32_from_bits(0x3e40c0c1u) : f32_from_bits(0x3f021bb6u);
    float sigma_raw[3], sigma_basic[3];
    for (int i = 0; i < 3; ++i) {
        sigma_raw[i] = sigma[i];
        sigma_basic[i] = sigma[i] * f32_from_bits(0x3f021bb6u);
    }
    for (float &s : sigma) s *= factor;

    int block_step[3], bm_range[3], ps_num[3], ps_range[3];
    per_plane<int>(a->block_step, a->n_block_step, 8, block_step);
    for (int v : block_step)
        if (v <= 0 || v > 8) {
            set_err(err, errlen, "BM3D: \"block_step\" must be in range [1, 8].");
            return nullptr;
        }
    per_plane<int>(a->bm_range, a->n_bm_range, 9, bm_range);
    for (int v : bm_range)
        if (v <= 0) {
            set_err(err, errlen, "BM3D: \"bm_range\" must be positive.");
            return nullptr;
        }
    per_plane<int>(a->ps_num, a->n_ps_num, 2, ps_num);
    for (int v : ps_num)
        if (v <= 0 || v > 8) {
            set_err(err, errlen, "BM3D: \"ps_num\" must be in range [1, 8].");
            return nullptr;
        }
    per_plane<int>(a->ps_range, a->n_ps_range, 4, ps_range);
    for (int v : ps_range)
        if (v <= 0) {
            set_err(err, errlen, "BM3D: \"ps_range\" must be positive.");
            return nullptr;
        }
    f->radius = pick(a->radius, 0);
    if (f->radius < 0) {
        set_err(err, errlen, "BM3D: \"radius\" must be non-negative.");
        return nullptr;
    }
    if (f->radius > kMaxRadius) {
        set_err(err, errlen, "BM3D: \"radius\" must be <= 16.");
        return nullptr;
    }
    f->tw = 2 * f->radius + 1;
    f->fused = f->v2 && pick(a->fast_fused, 0) != 0 && f->radius > 0;
    f->chroma = pick(a->chroma, 0) != 0;
    if (f->chroma && (vi.color_family != ZB3D_YUV || vi.subsampling_w != 0 || vi.subsampling_h != 0)) {
        set_err(err, errlen, "BM3D: clip format must be YUV444 when \"chroma\" is true.");
        return nullptr;
    }
    f->zero_init = pick(a->zero_init, 1) != 0;
    f->match_form = pick(a->match_form, -1);
    if (f->match_form != -1 && f->match_form != 0 && f->match_form != 1) {
        set_err(err, errlen, "BM3D: \"match_form\" must be 0 or 1.");
        return nullptr;
    }
    f->filter_form = pick(a->filter_form, 0);
    if (f->filter_form != 0 && f->filter_form != 1) {
        set_err(err, errlen, "BM3D: \"filter_form\" must be 0 or 1.");
        return nullptr;
    }
    const int extractor_exp = pick(a->extractor_exp, 0);
    f->extractor = extractor_exp != 0 ? std::ldexp(1.0f, extractor_exp) : 0.0f;

    int metric[3] = {M_SSD, M_SSD, M_SSD}, t2d[3] = {0, 0, 0}, t1d[3] = {0, 0, 0};
    for (int i = 0; i < 3; ++i) {
        if (i < a->n_bm_error_s) {
            metric[i] = parse_metric(a->bm_error_s[i]);
            if (metric[i] < 0) {
                set_err(err, errlen, "BM3D: invalid \"bm_error_s\".");
                return nullptr;
            }
        } else if (i > 0) {
            metric[i] = metric[i - 1];
        }
        if (i < a->n_transform_2d_s) {
            t2d[i] = parse_transform(a->transform_2d_s[i]);
            if (t2d[i] < 0) {
                set_err(err, errlen, "BM3D: invalid \"transform_2d_s\".");
                return nullptr;
            }
        } else if (i > 0) {
            t2d[i] = t2d[i - 1];
        }
        if (i < a->n_transform_1d_s) {
            t1d[i] = parse_transform(a->transform_1d_s[i]);
            if (t1d[i] < 0) {
                set_err(err, errlen, "BM3D: invalid \"transform_1d_s\".");
                return nullptr;
            }
        } else if (i > 0) {
            t1d[i] = t1d[i - 1];
        }
    }
    f->device = pick(a->device_id, 0);
    if (f->device < 0) {
        set_err(err, errlen, "BM3D: invalid device ID.");
        return nullptr;
    }
    if (a->num_streams != ZB3D_UNSET && (a->num_streams < 1 || a->num_streams > 32)) {
        set_err(err, errlen, "BM3D: num_streams must be 1..32.");
        return nullptr;
    }
    f->num_streams = pick(a->num_streams, 4);

    bool any = false;
    for (int i = 0; i < vi.num_planes && i < 3; ++i) any |= f->process[i];
    if (!any) {
        set_err(err, errlen, "BM3D: all planes have sigma < FLT_EPSILON (nothing to process).");
        return nullptr;
    }
    f->nclips = f->final_ ? 2 : 1;
    if (f->filter_form == 1)
        for (int i = 0; i < 3; ++i)
            if (f->process[i] && (t2d[i] != 0 || t1d[i] != 0)) {
                set_err(err, errlen, "BM3D: \"filter_form\" 1 needs the DCT in both dimensions.");
                return nullptr;
            }

    auto fill_geom = [&](Entry &e) {
        e.pitch = round_up(e.w, 32);
        e.plane_elems = (size_t)e.h * e.pitch;
        e.nbx = (e.w - 8 + e.bs - 1) / e.bs + 1;
        e.nby = (e.h - 8 + e.bs - 1) / e.bs + 1;
        e.nbx_al = (e.w - 8) / e.bs + 1;
        e.nblocks = (long long)e.nbx * e.nby;
    };
    if (f->chroma) {
        Entry e{};
        e.w = vi.width;
        e.h = vi.height;
        e.nplanes = 3;
        for (int i = 0; i < 3; ++i) {
            e.planes[i] = i;
            e.sigma[i] = sigma[i];
            e.sigma_basic[i] = sigma_basic[i];
            e.sigma_raw[i] = sigma_raw[i];
        }
        e.bs = block_step[0];
        e.range = bm_range[0];
        e.ps_num = ps_num[0];
        e.ps_range = ps_range[0];
        e.proc_mask = 0;
        for (int i = 0; i < 3; ++i) e.proc_mask |= (unsigned)f->process[i] << i;
        e.metric = metric[0];
        e.t2d = t2d[0];
        e.t1d = t1d[0];
        if (vi.width < 8 || vi.height < 8) {
            set_err(err, errlen, "BM3D: every processed plane must be at least 8x8.");
            return nullptr;
        }
        fill_geom(e);
        f->entries.push_back(e);
    } else {
        for (int p = 0; p < vi.num_planes && p < 3; ++p) {
            if (!f->process[p]) continue;
            Entry e{};
            e.w = p == 0 ? vi.width : vi.width >> vi.subsampling_w;
            e.h = p == 0 ? vi.height : vi.height >> vi.subsampling_h;
            if (e.w < 8 || e.h < 8) {
                set_err(err, errlen, "BM3D: every processed plane must be at least 8x8.");
                return nullptr;
            }
            e.nplanes = 1;
            e.planes[0] = p;
            e.sigma[0] = e.sigma[1] = e.sigma[2] = sigma[p];
            e.sigma_basic[0] = e.sigma_basic[1] = e.sigma_basic[2] = sigma_basic[p];
            e.sigma_raw[0] = e.sigma_raw[1] = e.sigma_raw[2] = sigma_raw[p];
            e.bs = block_step[p];
            e.range = bm_range[p];
            e.ps_num = ps_num[p];
            e.ps_range = ps_range[p];
            e.proc_mask = 1;
            e.metric = metric[p];
            e.t2d = t2d[p];
            e.t1d = t1d[p];
            fill_geom(e);
            f->entries.push_back(e);
        }
    }
    size_t src_off = 0, dst_off = 0, out_off = 0, frame_off = 0;
    for (Entry &e : f->entries) {
        if (e.w > 65535 || e.h > 65535) {
            set_err(err, errlen, "BM3D: frame too large (planes are limited to 65535x65535).");
            return nullptr;
        }
        e.src_off = src_off;
        e.src_elems = (size_t)f->nclips * e.nplanes * f->tw * e.plane_elems;
        e.dst_off = dst_off;
        e.dst_elems = f->dst_entry_elems(e);
        e.out_off = out_off;
        e.frame_off = frame_off;
        src_off += e.src_elems;
        dst_off += e.dst_elems;
        out_off += (size_t)e.nplanes * e.plane_elems;
        frame_off += (size_t)f->nclips * e.nplanes * e.plane_elems;
        f->acc_elems = std::max(f->acc_elems, (size_t)e.nplanes * f->tw * e.plane_elems);
        f->max_blocks = std::max(f->max_blocks, e.nblocks);
        // int32 index limits of the reference (src/bm3d.zig:1190-1201)
        if (e.src_elems >= (1ull << 31) || (size_t)e.nplanes * f->tw * 2 * e.plane_elems >= (1ull << 31)) {
            set_err(err, errlen, "BM3D: frame/radius too large (a device region exceeds 2^31 samples).");
            return nullptr;
        }
        if (e.plane_elems * f->tw * 2 * 4 >= (1ull << 32)) {
            set_err(err, errlen, "BM3D: stacked output plane too large (exceeds 4 GiB).");
            return nullptr;
        }
    }
    if (f->pilot) {
        // the pilot makes step 1 of an entry when its gate accepts every processed plane's sigma
        for (Entry &e : f->entries) {
            e.pilot_step1 = true;
            for (int i = 0; i < e.nplanes; ++i)
                if (((e.proc_mask >> i) & 1) && !zb3d_pilot_accepts(f->pilot, e.sigma_raw[i], e.w, e.h))
                    e.pilot_step1 = false;
            if (e.pilot_step1)
                f->pilot_ws_bytes = std::max(f->pilot_ws_bytes, zb3d_pilot_workspace_bytes(f->pilot, e.w, e.h));
        }
    }
    f->sum_src = src_off;
    f->sum_dst = dst_off;
    f->sum_out = out_off;
    f->frame_elems = frame_off;

    f->vi_out = vi;
    if (f->stacked_out()) {
        const long long mult = 2LL * (2LL * f->radius + 1);
        if ((long long)vi.height * mult > INT_MAX) {
            set_err(err, errlen, "BM3D: clip too tall for the stacked output.");
            return nullptr;
        }
        f->vi_out.height = (int)(vi.height * mult);
    }

    // ---- CUDA resources (src/bm3d.zig:772-951) ----
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || f->device >= ndev) {
        set_err(err, errlen, "BM3D: invalid device ID.");
        return nullptr;
    }
    cudaSetDevice(f->device);
    if (f->filter_form == 1 && filter_precision_init(f->device) != cudaSuccess) {
        cudaGetLastError();
        set_err(err, errlen, "BM3D: the precision filter could not be set up on the device.");
        return nullptr;
    }
    f->slots.resize(f->num_streams);
    int made = 0;
    for (auto &s : f->slots) {
        if (!alloc_slot(f.get(), s)) {
            s.destroy();
            cudaGetLastError();
            if (made > 0) break;  // keep the slots that fit (src/pool.zig:31-49)
            set_err(err, errlen, "BM3D: out of device memory.");
            return nullptr;
        }
        ++made;
    }
    f->slots.resize(made);
    for (int i = made - 1; i >= 0; --i) f->free_slots.push_back(i);
    for (Entry &e : f->entries) tune_entry(f.get(), f->slots[0], e);
    if (f->v2 && f->radius > 0) {
        // source frames: one request spans 4r+1 frames; accumulator stacks: 2r+1 centres
        const int span = 4 * f->radius + 1;
        const int n_src = span * (made + 1);
        const int n_acc = f->tw * (made + 1);
        const size_t stack_bytes = f->sum_dst * sizeof(float);
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const size_t need = (size_t)f->frame_elems * 4 * n_src + stack_bytes * (size_t)n_acc;
        if (need + (256u << 20) > free_b || !f->src_cache.init(f->frame_elems * sizeof(float), n_src) ||
            !f->acc_cache.init(stack_bytes, n_acc)) {
            cudaGetLastError();
            if (!f->fused) {
                set_err(err, errlen, "BM3D: out of device memory.");
                for (auto &s : f->slots) s.destroy();
                return nullptr;
            }
            set_err(err, errlen,
                    "BM3Dv2: fast_fused needs at least %zu MiB of accumulator cache (%d slots x %zu MiB) but only "
                    "%zu MiB of device memory is free. Use fast_fused=False (composed BM3D + VAggregate, much less "
                    "VRAM), or lower num_streams/radius.",
                    (stack_bytes * f->tw) >> 20, f->tw, stack_bytes >> 20, free_b >> 20);
            for (auto &s : f->slots) s.destroy();
            return nullptr;
        }
    }
    return f.release();
}

zb3d_filter *zb3d_create(const zb3d_video_info *clip, const zb3d_args *args, int v2, char *err, size_t errlen) {
    if (!clip) {
        zb::set_err(err, errlen, "BM3D: clip is required.");
        return nullptr;
    }
    return reinterpret_cast<zb3d_filter *>(create_impl(clip, args, v2, err, errlen));
}

void zb3d_output_info(const zb3d_filter *fp, zb3d_video_info *out) {
    *out = reinterpret_cast<const Filter *>(fp)->vi_out;
}

void zb3d_frame_range(const zb3d_filter *fp, int n, int *first, int *last) {
    const Filter *f = reinterpret_cast<const Filter *>(fp);
    const int req = f->passthrough ? 0 : (f->v2 ? 2 * f->radius : f->radius);
    *first = std::max(n - req, 0);
    *last = std::min(n + req, f->vi.num_frames - 1);
}

void zb3d_output_props(const zb3d_filter *fp, int *radius, int process[3]) {
    const Filter *f = reinterpret_cast<const Filter *>(fp);
    *radius = f->radius;
    for (int i = 0; i < 3; ++i) process[i] = f->process[i];
}

int zb3d_num_entries(const zb3d_filter *fp) { return (int)reinterpret_cast<const Filter *>(fp)->entries.size(); }

int zb3d_entry_layout_get(const zb3d_filter *fp, int e, zb3d_entry_layout *o) {
    const Filter *f = reinterpret_cast<const Filter *>(fp);
    if (e < 0 || e >= (int)f->entries.size()) return -1;
    const Entry &en = f->entries[e];
    o->nplanes = en.nplanes;
    for (int i = 0; i < 3; ++i) o->plane[i] = en.planes[i];
    o->width = en.w;
    o->height = en.h;
    o->pitch = en.pitch;
    o->tw = f->tw;
    o->nclips = f->nclips;
    o->src_offset = en.src_off;
    o->src_elems = en.src_elems;
    o->dst_offset = en.dst_off;
    o->dst_elems = en.dst_elems;
    return 0;
}

size_t zb3d_src_elems(const zb3d_filter *fp) { return reinterpret_cast<const Filter *>(fp)->sum_src; }
size_t zb3d_dst_elems(const zb3d_filter *fp) { return reinterpret_cast<const Filter *>(fp)->sum_dst; }

int zb3d_process_batch_ex(const zb3d_batch_job *jobs, int njobs, void *stream, unsigned wait_polls,
                          int unsatisfiable, char *err, size_t errlen) {
    using namespace zb;
    BatchPlan p;
    if (!plan_batch(jobs, njobs, p, err, errlen)) return -1;
    cudaSetDevice(p.device);
    const cudaStream_t st = (cudaStream_t)stream;
    BatchCtx &ctx = batch_ctx(p.device);
    std::lock_guard<std::mutex> lk(ctx.mu);
    if (!ensure_buffers(ctx.buf, p, st, err, errlen)) return -1;
    std::map<Filter *, int> held = hold_slots(p);
    cudaError_t ce = enqueue_batch(p, ctx.buf, held, wait_polls, unsatisfiable, st);
    const cudaError_t cs = cudaStreamSynchronize(st);
    if (ce == cudaSuccess) ce = cs;
    release_slots(held);
    if (ce != cudaSuccess) {
        set_err(err, errlen, "zb3d_process_batch: %s.", cudaGetErrorString(ce));
        return -1;
    }
    if (*ctx.buf.h_status != 0) {
        set_err(err, errlen,
                "zb3d_process_batch: a filter chunk gave up waiting for its entry's matching (status %d); the "
                "outputs of this batch are incomplete.",
                *ctx.buf.h_status);
        return -1;
    }
    return 0;
}

// A batch captured once into a CUDA graph with its own scratch; replays are launches.
struct zb3d_batch {
    zb::BatchPlan plan;
    zb::BatchBuffers buf;
    std::map<Filter *, int> held;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
};

zb3d_batch *zb3d_batch_create(const zb3d_batch_job *jobs, int njobs, char *err, size_t errlen) {
    using namespace zb;
    std::unique_ptr<zb3d_batch> b(new zb3d_batch());
    if (!plan_batch(jobs, njobs, b->plan, err, errlen)) return nullptr;
    cudaSetDevice(b->plan.device);
    auto fail = [&](const char *what, cudaError_t e) -> zb3d_batch * {
        cudaGetLastError();
        set_err(err, errlen, "zb3d_batch_create: %s (%s).", what, cudaGetErrorString(e));
        if (b->cap) cudaStreamSynchronize(b->cap);
        release_slots(b->held);
        if (b->exec) cudaGraphExecDestroy(b->exec);
        if (b->cap) cudaStreamDestroy(b->cap);
        b->buf.release();
        return nullptr;
    };
    cudaError_t e = cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fail("cannot create a stream", e);
    if (!ensure_buffers(b->buf, b->plan, b->cap, err, errlen)) {
        cudaStreamDestroy(b->cap);
        b->buf.release();
        return nullptr;
    }
    b->held = hold_slots(b->plan);
    cudaGraph_t g = nullptr;
    e = cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail("cannot capture", e);
    const cudaError_t e1 = enqueue_batch(b->plan, b->buf, b->held, 0, 0, b->cap);
    e = cudaStreamEndCapture(b->cap, &g);
    if (e1 != cudaSuccess) e = e1;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
    if (g) cudaGraphDestroy(g);
    if (e != cudaSuccess) return fail("the batch could not be captured as a graph", e);
    *b->buf.h_status = 0;
    return b.release();
}

int zb3d_batch_launch(zb3d_batch *b, void *stream, char *err, size_t errlen) {
    if (!b || !b->exec) {
        zb::set_err(err, errlen, "zb3d_batch_launch: no batch.");
        return -1;
    }
    cudaSetDevice(b->plan.device);
    const cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) {
        zb::set_err(err, errlen, "zb3d_batch_launch: %s.", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

int zb3d_batch_status(zb3d_batch *b, char *err, size_t errlen) {
    if (!b || !b->buf.h_status) {
        zb::set_err(err, errlen, "zb3d_batch_status: no batch.");
        return -1;
    }
    const int st = *b->buf.h_status;
    if (st != 0) {
        zb::set_err(err, errlen,
                    "zb3d_batch_status: a filter chunk gave up waiting for its entry's matching (status %d); the "
                    "outputs of the last launch are incomplete.",
                    st);
        return -1;
    }
    return 0;
}

void zb3d_batch_free(zb3d_batch *b) {
    if (!b) return;
    cudaSetDevice(b->plan.device);
    if (b->cap) cudaStreamSynchronize(b->cap);
    cudaDeviceSynchronize();  // replays may still run on the callers' streams
    if (b->exec) cudaGraphExecDestroy(b->exec);
    zb::release_slots(b->held);
    if (b->cap) cudaStreamDestroy(b->cap);
    b->buf.release();
    delete b;
}

int zb3d_process_batch(const zb3d_batch_job *jobs, int njobs, void *stream, char *err, size_t errlen) {
    return zb3d_process_batch_ex(jobs, njobs, stream, 0, 0, err, errlen);
}

int zb3d_process_device(zb3d_filter *fp, const float *d_src, float *d_dst, void *stream, char *err, size_t errlen) {
    Filter *f = reinterpret_cast<Filter *>(fp);
    if (f->passthrough || f->slots.empty()) {
        zb::set_err(err, errlen, "BM3D: nothing to process on the device.");
        return -1;
    }
    cudaSetDevice(f->device);
    zb::Slot &s = f->slots[0];
    const cudaStream_t st = stream ? (cudaStream_t)stream : s.st;
    cudaError_t e = zb::run_graphed(f, s, std::make_tuple((const void *)d_src, (const void *)d_dst, -1), st,
                                    [&](zb::Slot &x) { return zb::run_window(f, x, d_src, d_dst); });
    if (e != cudaSuccess) {
        zb::set_err(err, errlen, "BM3D: process frame failed (%s).", cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

int zb3d_process_entry_device(zb3d_filter *fp, int e, const float *d_src, float *d_dst, void *stream, char *err,
                              size_t errlen) {
    Filter *f = reinterpret_cast<Filter *>(fp);
    if (f->passthrough || e < 0 || e >= (int)f->entries.size()) {
        zb::set_err(err, errlen, "BM3D: no such entry.");
        return -1;
    }
    cudaSetDevice(f->device);
    zb::Slot &s = f->slots[0];
    const cudaStream_t st = stream ? (cudaStream_t)stream : s.st;
    const zb::Entry &en = f->entries[e];
    cudaError_t ce = zb::run_graphed(f, s, std::make_tuple((const void *)d_src, (const void *)d_dst, e), st,
                                     [&](zb::Slot &x) { return zb::run_entry_steps(f, x, en, d_src, d_dst); });
    if (ce != cudaSuccess) {
        zb::set_err(err, errlen, "BM3D: process frame failed (%s).", cudaGetErrorString(ce));
        return -1;
    }
    return 0;
}

void zb3d_profile_enable(zb3d_filter *fp, int on) { reinterpret_cast<Filter *>(fp)->profile = on != 0; }

int zb3d_profile_collect(zb3d_filter *fp, double *match_ms, int *match_launches, double *filter_ms,
                         int *filter_launches) {
    Filter *f = reinterpret_cast<Filter *>(fp);
    std::lock_guard<std::mutex> lk(f->prof_mu);
    auto sum = [](std::vector<cudaEvent_t> &v, double *ms, int *n) {
        double t = 0.0;
        int k = 0;
        for (size_t i = 0; i + 1 < v.size(); i += 2) {
            cudaEventSynchronize(v[i + 1]);
            float x = 0.0f;
            if (cudaEventElapsedTime(&x, v[i], v[i + 1]) == cudaSuccess) {
                t += x;
                ++k;
            }
        }
        for (cudaEvent_t ev : v) cudaEventDestroy(ev);
        v.clear();
        if (ms) *ms = t;
        if (n) *n = k;
    };
    sum(f->prof_match, match_ms, match_launches);
    sum(f->prof_filter, filter_ms, filter_launches);
    return 0;
}

int zb3d_match_device(zb3d_filter *fp, int e, const float *d_src, int32_t *d_list, void *stream, char *err,
                      size_t errlen) {
    Filter *f = reinterpret_cast<Filter *>(fp);
    if (f->passthrough || e < 0 || e >= (int)f->entries.size()) {
        zb::set_err(err, errlen, "BM3D: no such entry.");
        return -1;
    }
    cudaSetDevice(f->device);
    zb::Slot s = f->slots[0];
    s.st = stream ? (cudaStream_t)stream : f->slots[0].st;
    const Entry &en = f->entries[e];
    cudaError_t ce = zb::run_match(f, s, en, d_src + en.src_off);
    if (ce == cudaSuccess)
        ce = cudaMemcpyAsync(d_list, s.list, (size_t)en.nblocks * 8 * sizeof(int2), cudaMemcpyDeviceToDevice, s.st);
    if (ce != cudaSuccess) {
        zb::set_err(err, errlen, "BM3D: matching failed (%s).", cudaGetErrorString(ce));
        return -1;
    }
    return 0;
}

int zb3d_entry_tuning(const zb3d_filter *fp, int e, int *form, int *rows) {
    const Filter *f = reinterpret_cast<const Filter *>(fp);
    if (f->passthrough || e < 0 || e >= (int)f->entries.size()) return -1;
    *form = f->entries[e].form;
    *rows = f->entries[e].rows;
    return 0;
}

int zb3d_match_stats(zb3d_filter *fp, unsigned long long out[4], int reset) {
    Filter *f = reinterpret_cast<Filter *>(fp);
    for (int i = 0; i < 4; ++i) out[i] = 0;
    if (f->passthrough) return 0;
    cudaSetDevice(f->device);
    for (zb::Slot &s : f->slots) {
        if (!s.tc_stats) continue;
        unsigned long long v[4];
        if (cudaStreamSynchronize(s.st) != cudaSuccess ||
            cudaMemcpy(v, s.tc_stats, sizeof v, cudaMemcpyDeviceToHost) != cudaSuccess)
            return -1;
        for (int i = 0; i < 4; ++i) out[i] += v[i];
        if (reset && cudaMemset(s.tc_stats, 0, sizeof v) != cudaSuccess) return -1;
    }
    return 0;
}

static zb::MatchArgs probe_args(int width, int height, int pitch, int bs, int range) {
    zb::MatchArgs a{};
    a.w = width;
    a.h = height;
    a.pitch = pitch;
    a.bs = bs;
    a.range = range;
    a.nbx = (width - 8 + bs - 1) / bs + 1;
    a.nby = (height - 8 + bs - 1) / bs + 1;
    a.nbx_al = (width - 8) / bs + 1;
    a.radius = 0;
    a.ps_num = 2;
    a.ps_range = 4;
    return a;
}

int zb3d_tc_probe_cols(int width, int height, int block_step, int bm_range) {
    const zb::MatchArgs a = probe_args(width, height, width, block_step, bm_range);
    return zb::tc_eligible(a) ? zb::tc_debug_cols(a) : 0;
}

int zb3d_tc_probe(const float *d_plane, int width, int height, int pitch, int block_step, int bm_range,
                  int32_t *d_list, float *d_dist, unsigned long long *d_prof, unsigned long long stats[4], char *err,
                  size_t errlen) {
    using namespace zb;
    if (width < 8 || height < 8 || block_step < 1 || block_step > 8 || bm_range < 1 || pitch < width) {
        set_err(err, errlen, "zb3d_tc_probe: bad geometry.");
        return -1;
    }
    MatchArgs a = probe_args(width, height, pitch, block_step, bm_range);
    if (!tc_eligible(a)) return 1;
    a.frames = d_plane;
    a.list = reinterpret_cast<int2 *>(d_list);
    a.tc_dbg = d_dist;
    a.tc_prof = d_prof;
    const long long nb = (long long)a.nbx * a.nby;
    int *ws = nullptr;
    unsigned long long *st = nullptr;
    cudaError_t ce = cudaMalloc(&ws, (kTcWsList + nb) * sizeof(int));
    if (ce == cudaSuccess) ce = cudaMalloc(&st, 4 * sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = cudaMemset(st, 0, 4 * sizeof(unsigned long long));
    a.tc_ws = ws;
    a.tc_stats = st;
    // the tensor-core kernel alone first, then the FP32 scan of the blocks it listed, each
    // synchronised, so that an error is attributed to the kernel that raised it
    a.self_incl = 1;
    const char *stage = "tensor-core kernel";
    if (ce == cudaSuccess) ce = launch_match_tc(a, nullptr);
    if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
    int ws_head[7] = {0, 0, 0, 0, 0, 0, 0};
    if (ce == cudaSuccess) ce = cudaMemcpy(ws_head, ws, sizeof ws_head, cudaMemcpyDeviceToHost);
    if (ce == cudaSuccess) {
        stage = "FP32 scan of the listed blocks";
        ce = launch_tc_fallback(a, nullptr);
    }
    if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
    if (ce == cudaSuccess) ce = cudaMemcpy(stats, st, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(ws);
    cudaFree(st);
    if (ce != cudaSuccess) {
        set_err(err, errlen, "zb3d_tc_probe: %s (%s).", cudaGetErrorString(ce), stage);
        return -1;
    }
    if (ws_head[2]) {
        set_err(err, errlen, "zb3d_tc_probe: self-check %d failed (values %d %d %d, tile %d).", ws_head[2],
                ws_head[3], ws_head[4], ws_head[5], ws_head[6]);
        return -1;
    }
    if (ws_head[1]) {
        set_err(err, errlen, "zb3d_tc_probe: an MMA wait timed out (its tiles went to the FP32 scan).");
        return -1;
    }
    return 0;
}

int zb3d_vaggregate_device(const float *const *stacks, const int *z, int tw, int width, int height, int pitch,
                           int nplanes, unsigned proc_mask, float *d_dst, void *stream) {
    return zb::launch_vagg(stacks, z, tw, width, height, pitch, nplanes, proc_mask, d_dst, pitch,
                           (long long)height * pitch, (cudaStream_t)stream) == cudaSuccess
               ? 0
               : -1;
}

// ---- host-frame path ------------------------------------------------------

static int get_frame_window(Filter *f, int n, const zb3d_frame *clip_frames, const zb3d_frame *ref_frames,
                            zb3d_frame_out *dst, char *err, size_t errlen) {
    using namespace zb;
    int first, last;
    zb3d_frame_range(reinterpret_cast<zb3d_filter *>(f), n, &first, &last);
    const int nf = f->vi.num_frames;
    const int slot = acquire_slot(f);
    Slot &s = f->slots[slot];
    cudaSetDevice(f->device);
    // the window [clips][planes][t][h][pitch] per entry, plane by plane: page-locked
    // caller planes are copied to the device directly; any other plane goes through the
    // slot's pinned staging buffer (copy threads), and its upload is issued at once, so it
    // overlaps the staging copy of the next plane (src/bm3d.zig:295-373)
    auto each_src = [&](auto fn) {
        for (const Entry &e : f->entries)
            for (int c = f->pilot ? 1 : 0; c < f->nclips; ++c) {  // pilot form: step 1 makes clip 0
                const zb3d_frame *frames = (f->final_ && c == 0) ? ref_frames : clip_frames;
                for (int i = 0; i < e.nplanes; ++i)
                    for (int t = 0; t < f->tw; ++t) {
                        const int idx = clampi(n - f->radius + t, 0, nf - 1);
                        const zb3d_frame &fr = frames[idx - first];
                        const int p = e.planes[i];
                        fn(e, e.src_off + ((size_t)(c * e.nplanes + i) * f->tw + t) * e.plane_elems, fr.ptr[p],
                           fr.stride[p]);
                    }
            }
    };
    cudaError_t ce = cudaSuccess;
    each_src([&](const Entry &e, size_t off, const float *ptr, ptrdiff_t stride) {
        if (ce != cudaSuccess) return;
        if (is_pinned(ptr)) {
            ce = cudaMemcpy2DAsync(s.d_src + off, (size_t)e.pitch * sizeof(float), ptr, (size_t)stride,
                                   (size_t)e.w * sizeof(float), e.h, cudaMemcpyHostToDevice, s.cst);
        } else {
            copy_plane_in(s.h_stage + off, e.pitch, ptr, stride, e.w, e.h);
            ce = cudaMemcpyAsync(s.d_src + off, s.h_stage + off, e.plane_elems * sizeof(float),
                                 cudaMemcpyHostToDevice, s.cst);
        }
    });
    if (ce == cudaSuccess) ce = cudaEventRecord(s.ev_up, s.cst);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s.st, s.ev_up, 0);
    if (ce == cudaSuccess)
        ce = run_graphed(f, s, std::make_tuple((const void *)s.d_src, (const void *)s.d_dst, -1), s.st,
                         [&](Slot &x) { return run_window(f, x, x.d_src, x.d_dst); });
    if (ce == cudaSuccess && s.dev_status)
        ce = cudaMemcpyAsync(s.h_dev_status, s.dev_status, sizeof(int), cudaMemcpyDeviceToHost, s.st);
    // page-locked output planes receive the result directly, the others through staging
    // (denoised planes; the stacked accumulator layout always goes through staging)
    float *down = s.h_stage + s.stage_up;
    std::vector<std::pair<const Entry *, int>> staged_out;  // (entry, plane of the entry)
    if (!f->stacked_out()) {
        for (const Entry &e : f->entries)
            for (int i = 0; i < e.nplanes; ++i) {
                if (!((e.proc_mask >> i) & 1) || ce != cudaSuccess) continue;
                const int p = e.planes[i];
                const size_t off = e.dst_off + (size_t)i * e.plane_elems;
                if (is_pinned(dst->ptr[p])) {
                    ce = cudaMemcpy2DAsync(dst->ptr[p], (size_t)dst->stride[p], s.d_dst + off,
                                           (size_t)e.pitch * sizeof(float), (size_t)e.w * sizeof(float), e.h,
                                           cudaMemcpyDeviceToHost, s.st);
                } else {
                    ce = cudaMemcpyAsync(down + off, s.d_dst + off, e.plane_elems * sizeof(float),
                                         cudaMemcpyDeviceToHost, s.st);
                    staged_out.emplace_back(&e, i);
                }
            }
    } else if (ce == cudaSuccess) {
        ce = cudaMemcpyAsync(down, s.d_dst, f->sum_dst * sizeof(float), cudaMemcpyDeviceToHost, s.st);
    }
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s.st);
    if (ce != cudaSuccess) {
        cudaStreamSynchronize(s.cst);
        cudaStreamSynchronize(s.st);
        release_slot(f, slot);
        set_err(err, errlen, "BM3D: process frame failed. (%s)", cudaGetErrorString(ce));
        return -1;
    }
    if (s.h_dev_status && *s.h_dev_status != 0) {
        // a tensor-core pipeline wait ran out: the frame is incomplete
        *s.h_dev_status = 0;
        cudaMemsetAsync(s.dev_status, 0, sizeof(int), s.st);
        cudaStreamSynchronize(s.st);
        release_slot(f, slot);
        set_err(err, errlen, "BM3D: process frame failed. (a tensor-core pipeline timed out)");
        return -1;
    }
    for (const auto &pe : staged_out) {
        const Entry &e = *pe.first;
        copy_plane_out(dst->ptr[e.planes[pe.second]], dst->stride[e.planes[pe.second]],
                       down + e.dst_off + (size_t)pe.second * e.plane_elems, e.pitch, e.w, e.h);
    }
    for (const Entry &e : f->entries) {
        if (!f->stacked_out()) break;
        for (int i = 0; i < e.nplanes; ++i) {
            if (!((e.proc_mask >> i) & 1)) continue;
            const int p = e.planes[i];
            const float *src = down + e.dst_off + (size_t)i * f->tw * 2 * e.plane_elems;
            copy_plane_out(dst->ptr[p], dst->stride[p], src, e.pitch, e.w, e.h * 2 * f->tw);
        }
    }
    if (f->stacked_out() && f->zero_init) {
        for (int p = 0; p < f->vi.num_planes && p < 3; ++p) {
            if (f->process[p]) continue;
            const int w = p == 0 ? f->vi.width : f->vi.width >> f->vi.subsampling_w;
            const int h = (p == 0 ? f->vi_out.height : f->vi_out.height >> f->vi.subsampling_h);
            for (int y = 0; y < h; ++y) memset((char *)dst->ptr[p] + (ptrdiff_t)y * dst->stride[p], 0, (size_t)w * 4);
        }
    }
    release_slot(f, slot);
    return 0;
}

// BM3Dv2 radius > 0: accumulator stacks of the 2r+1 centres around n (cached on
// the device by centre), then the temporal aggregation.  The stacks and the
// aggregation are those of the composed BM3D + VAggregate chain, so the output
// is the same byte for byte (src/bm3d.zig:481-633).
static int get_frame_temporal(Filter *f, int n, const zb3d_frame *clip_frames, const zb3d_frame *ref_frames,
                              zb3d_frame_out *dst, char *err, size_t errlen) {
    using namespace zb;
    const int r = f->radius, tw = f->tw, nf = f->vi.num_frames;
    int first, last;
    zb3d_frame_range(reinterpret_cast<zb3d_filter *>(f), n, &first, &last);
    const int slot = acquire_slot(f);
    Slot &s = f->slots[slot];
    cudaSetDevice(f->device);
    cudaError_t ce = cudaSuccess;

    // centres and their accumulator stacks
    long long ckeys[kMaxTw];
    int centres[kMaxTw], nc = 0;
    for (int i = 0; i < tw; ++i) {
        const int m = clampi(n - r + i, 0, nf - 1);
        bool dup = false;
        for (int k = 0; k < nc; ++k) dup |= centres[k] == m;
        if (!dup) {
            centres[nc] = m;
            ckeys[nc] = m;
            ++nc;
        }
    }
    int aidx[kMaxTw];
    bool aload[kMaxTw];
    f->acc_cache.acquire(ckeys, nc, aidx, aload);

    // source frames the missing centres need
    long long skeys[4 * kMaxRadius + 1];
    int sframes[4 * kMaxRadius + 1], ns = 0;
    for (int k = 0; k < nc; ++k) {
        if (!aload[k]) continue;
        for (int t = 0; t < tw; ++t) {
            const int idx = clampi(centres[k] - r + t, 0, nf - 1);
            bool dup = false;
            for (int q = 0; q < ns; ++q) dup |= sframes[q] == idx;
            if (!dup) {
                sframes[ns] = idx;
                skeys[ns] = idx;
                ++ns;
            }
        }
    }
    int sidx[4 * kMaxRadius + 1];
    bool sload[4 * kMaxRadius + 1];
    if (ns) f->src_cache.acquire(skeys, ns, sidx, sload);
    for (int q = 0; q < ns && ce == cudaSuccess; ++q) {
        if (!sload[q]) continue;
        const int idx = sframes[q];
        float *stage = s.h_stage;  // one frame at a time through the up-stage
        for (const Entry &e : f->entries)
            for (int c = f->pilot ? 1 : 0; c < f->nclips; ++c) {  // pilot form: step 1 makes clip 0
                const zb3d_frame *frames = (f->final_ && c == 0) ? ref_frames : clip_frames;
                const zb3d_frame &fr = frames[idx - first];
                for (int i = 0; i < e.nplanes; ++i) {
                    const int p = e.planes[i];
                    copy_plane_in(stage + e.frame_off + (size_t)(c * e.nplanes + i) * e.plane_elems, e.pitch,
                                  fr.ptr[p], fr.stride[p], e.w, e.h);
                }
            }
        ce = cudaMemcpyAsync(f->src_cache.buf(sidx[q]), stage, f->frame_elems * sizeof(float), cudaMemcpyHostToDevice,
                             s.cst);
        if (ce == cudaSuccess) ce = cudaEventRecord(f->src_cache.ev(sidx[q]), s.cst);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(s.cst);  // the stage is reused by the next frame
        if (ce == cudaSuccess) f->src_cache.publish(sidx[q]);
    }
    for (int q = 0; q < ns && ce == cudaSuccess; ++q) ce = cudaStreamWaitEvent(s.st, f->src_cache.ev(sidx[q]), 0);

    // compute the missing stacks
    for (int k = 0; k < nc && ce == cudaSuccess; ++k) {
        if (!aload[k]) continue;
        const int m = centres[k];
        for (const Entry &e : f->entries)
            for (int c = 0; c < f->nclips; ++c)
                for (int i = 0; i < e.nplanes; ++i)
                    for (int t = 0; t < tw && ce == cudaSuccess; ++t) {
                        const int idx = clampi(m - r + t, 0, nf - 1);
                        int q = 0;
                        while (sframes[q] != idx) ++q;
                        const float *from = (const float *)f->src_cache.buf(sidx[q]) + e.frame_off +
                                            (size_t)(c * e.nplanes + i) * e.plane_elems;
                        float *to = s.d_src + e.src_off + ((size_t)(c * e.nplanes + i) * tw + t) * e.plane_elems;
                        ce = cudaMemcpyAsync(to, from, e.plane_elems * sizeof(float), cudaMemcpyDeviceToDevice, s.st);
                    }
        if (ce != cudaSuccess) break;
        // the window's stacked accumulators go straight into the cache slot
        float *stack = (float *)f->acc_cache.buf(aidx[k]);
        ce = run_window(f, s, s.d_src, stack);
        if (ce == cudaSuccess) ce = cudaEventRecord(f->acc_cache.ev(aidx[k]), s.st);
        if (ce == cudaSuccess) f->acc_cache.publish(aidx[k]);
    }
    for (int k = 0; k < nc && ce == cudaSuccess; ++k) ce = cudaStreamWaitEvent(s.st, f->acc_cache.ev(aidx[k]), 0);

    // temporal aggregation of frame n
    float *down = s.h_stage + s.stage_up;
    for (const Entry &e : f->entries) {
        if (ce != cudaSuccess) break;
        const float *ptrs[kMaxTw];
        int zs[kMaxTw];
        for (int i = 0; i < tw; ++i) {
            const int m = clampi(n - r + i, 0, nf - 1);
            int k = 0;
            while (centres[k] != m) ++k;
            ptrs[i] = (const float *)f->acc_cache.buf(aidx[k]) + e.dst_off;
            zs[i] = zb3d_agg_z(i, n, nf, r);
        }
        ce = launch_vagg(ptrs, zs, tw, e.w, e.h, e.pitch, e.nplanes, e.proc_mask, s.d_dst + e.out_off, e.pitch,
                         (long long)e.plane_elems, s.st);
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(down, s.d_dst, f->sum_out * sizeof(float), cudaMemcpyDeviceToHost, s.st);
    if (ce == cudaSuccess && s.dev_status)
        ce = cudaMemcpyAsync(s.h_dev_status, s.dev_status, sizeof(int), cudaMemcpyDeviceToHost, s.st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s.st);
    if (ce == cudaSuccess && s.h_dev_status && *s.h_dev_status != 0) {
        *s.h_dev_status = 0;
        cudaMemsetAsync(s.dev_status, 0, sizeof(int), s.st);
        ce = cudaErrorLaunchTimeout;  // a tensor-core pipeline wait ran out: the frame is incomplete
    }
    // claims are dropped only after the streams drained (released slots may be reloaded at once)
    if (ce != cudaSuccess) {
        cudaStreamSynchronize(s.cst);
        cudaStreamSynchronize(s.st);
        for (int q = 0; q < ns; ++q)
            if (sload[q]) f->src_cache.abandon(sidx[q]);
        if (ns) f->src_cache.release(sidx, ns);
        for (int k = 0; k < nc; ++k)
            if (aload[k]) f->acc_cache.abandon(aidx[k]);
        f->acc_cache.release(aidx, nc);
        release_slot(f, slot);
        set_err(err, errlen, "BM3Dv2: process frame failed. (%s)", cudaGetErrorString(ce));
        return -1;
    }
    if (ns) f->src_cache.release(sidx, ns);
    f->acc_cache.release(aidx, nc);
    for (const Entry &e : f->entries)
        for (int i = 0; i < e.nplanes; ++i) {
            if (!((e.proc_mask >> i) & 1)) continue;
            const int p = e.planes[i];
            copy_plane_out(dst->ptr[p], dst->stride[p], down + e.out_off + (size_t)i * e.plane_elems, e.pitch, e.w,
                           e.h);
        }
    release_slot(f, slot);
    return 0;
}

int zb3d_get_frame(zb3d_filter *fp, int n, const zb3d_frame *clip_frames, const zb3d_frame *ref_frames,
                   zb3d_frame_out *dst, char *err, size_t errlen) {
    Filter *f = reinterpret_cast<Filter *>(fp);
    if (n < 0 || n >= f->vi.num_frames) {
        zb::set_err(err, errlen, "BM3D: frame %d out of range.", n);
        return -1;
    }
    if (f->passthrough) {
        int first, last;
        zb3d_frame_range(fp, n, &first, &last);
        const zb3d_frame &fr = clip_frames[n - first];
        for (int p = 0; p < f->vi.num_planes && p < 3; ++p) {
            const int w = p == 0 ? f->vi.width : f->vi.width >> f->vi.subsampling_w;
            const int h = p == 0 ? f->vi.height : f->vi.height >> f->vi.subsampling_h;
            for (int y = 0; y < h; ++y)
                memcpy((char *)dst->ptr[p] + (ptrdiff_t)y * dst->stride[p],
                       (const char *)fr.ptr[p] + (ptrdiff_t)y * fr.stride[p], (size_t)w * 4);
        }
        return 0;
    }
    if (f->final_ && !f->pilot && !ref_frames) {
        zb::set_err(err, errlen, "BM3D: ref frames are required.");
        return -1;
    }
    if (f->v2 && f->radius > 0) return get_frame_temporal(f, n, clip_frames, ref_frames, dst, err, errlen);
    return get_frame_window(f, n, clip_frames, ref_frames, dst, err, errlen);
}

void zb3d_free(zb3d_filter *fp) {
    Filter *f = reinterpret_cast<Filter *>(fp);
    if (!f) return;
    if (!f->passthrough) {
        cudaSetDevice(f->device);
        cudaDeviceSynchronize();
        for (auto &kv : f->graphs) cudaGraphExecDestroy(kv.second);
        f->graphs.clear();
        for (auto &s : f->slots) {
            if (s.st) cudaStreamSynchronize(s.st);
            if (s.cst) cudaStreamSynchronize(s.cst);
            s.destroy();
        }
        f->src_cache.clear();
        f->acc_cache.clear();
    }
    delete f;
}

// ---- VAggregate -----------------------------------------------------------

struct zb3d_vagg {
    zb3d_video_info vi;       // src
    int radius;
    bool process[3];
    int device;
    std::mutex mu;
    float *d_in = nullptr, *d_out = nullptr, *h_stage = nullptr;
    size_t in_elems = 0, out_elems = 0;
    cudaStream_t st = nullptr;
};

zb3d_vagg *zb3d_vaggregate_create(const zb3d_video_info *clip, const zb3d_video_info *src, const int *planes,
                                  int n_planes, char *err, size_t errlen) {
    using namespace zb;
    if (src->height <= 0 || src->sample_type != ZB3D_FLOAT || src->bits_per_sample != 32) {
        set_err(err, errlen, "VAggregate: \"src\" must be 32 bit float.");
        return nullptr;
    }
    if (clip->color_family != src->color_family || clip->sample_type != src->sample_type ||
        clip->bits_per_sample != src->bits_per_sample || clip->subsampling_w != src->subsampling_w ||
        clip->subsampling_h != src->subsampling_h || clip->num_frames != src->num_frames) {
        set_err(err, errlen, "VAggregate: \"clip\" must have the same format and frame count as \"src\".");
        return nullptr;
    }
    const int ratio = clip->height / src->height;
    if (ratio < 6 || (ratio - 2) % 4 != 0 || clip->height % src->height != 0 || clip->width != src->width) {
        set_err(err, errlen, "VAggregate: \"clip\" is not a BM3D stacked clip of \"src\" (radius >= 1).");
        return nullptr;
    }
    const int radius = (ratio - 2) / 4;
    if (radius > kMaxRadius) {
        set_err(err, errlen, "VAggregate: radius too large.");
        return nullptr;
    }
    bool proc[3] = {false, false, false};
    for (int i = 0; i < n_planes; ++i) {
        if (planes[i] < 0 || planes[i] > 2) {
            set_err(err, errlen, "VAggregate: \"planes\" must be 0..2.");
            return nullptr;
        }
        proc[planes[i]] = true;
    }
    if (n_planes == 0) {
        set_err(err, errlen, "VAggregate: \"planes\" is required.");
        return nullptr;
    }
    zb3d_vagg *v = new zb3d_vagg();
    v->vi = *src;
    v->radius = radius;
    for (int i = 0; i < 3; ++i) v->process[i] = proc[i];
    cudaGetDevice(&v->device);
    return v;
}

void zb3d_vaggregate_output_info(const zb3d_vagg *v, zb3d_video_info *out) { *out = v->vi; }

void zb3d_vaggregate_frame_range(const zb3d_vagg *v, int n, int *first, int *last) {
    *first = std::max(n - v->radius, 0);
    *last = std::min(n + v->radius, v->vi.num_frames - 1);
}

int zb3d_vaggregate_get_frame(zb3d_vagg *v, int n, const zb3d_frame *stacks, zb3d_frame_out *dst, char *err,
                              size_t errlen) {
    using namespace zb;
    std::lock_guard<std::mutex> lk(v->mu);
    const int r = v->radius, tw = 2 * r + 1, nf = v->vi.num_frames;
    int first, last;
    zb3d_vaggregate_frame_range(v, n, &first, &last);
    cudaSetDevice(v->device);
    // device layout per plane: tw stacks of [tw][2][h][pitch] (one plane at a time)
    const int W = v->vi.width, H = v->vi.height;
    const int pitch = round_up(W, 32);
    const size_t stack_elems = (size_t)tw * 2 * H * pitch;
    if (!v->st && cudaStreamCreateWithFlags(&v->st, cudaStreamNonBlocking) != cudaSuccess) {
        set_err(err, errlen, "VAggregate: CUDA initialization failed.");
        return -1;
    }
    if (v->in_elems < stack_elems * tw) {
        cudaFree(v->d_in);
        cudaFree(v->d_out);
        if (v->h_stage) cudaFreeHost(v->h_stage);
        v->in_elems = stack_elems * tw;
        v->out_elems = (size_t)H * pitch;
        if (cudaMalloc(&v->d_in, v->in_elems * 4) != cudaSuccess ||
            cudaMalloc(&v->d_out, v->out_elems * 4) != cudaSuccess ||
            cudaHostAlloc((void **)&v->h_stage, (v->in_elems + v->out_elems) * 4, cudaHostAllocDefault) != cudaSuccess) {
            v->in_elems = 0;
            set_err(err, errlen, "VAggregate: out of device memory.");
            return -1;
        }
    }
    for (int p = 0; p < v->vi.num_planes && p < 3; ++p) {
        if (!v->process[p]) continue;
        const int w = p == 0 ? W : W >> v->vi.subsampling_w;
        const int h = p == 0 ? H : H >> v->vi.subsampling_h;
        const int pp = round_up(w, 32);
        const size_t se = (size_t)tw * 2 * h * pp;
        const float *ptrs[kMaxTw];
        int zs[kMaxTw];
        for (int i = 0; i < tw; ++i) {
            const int idx = clampi(n - r + i, 0, nf - 1);
            const zb3d_frame &fr = stacks[idx - first];
            copy_plane_in(v->h_stage + i * se, pp, fr.ptr[p], fr.stride[p], w, h * 2 * tw);
            ptrs[i] = v->d_in + i * se;
            zs[i] = zb3d_agg_z(i, n, nf, r);
        }
        cudaError_t ce = cudaMemcpyAsync(v->d_in, v->h_stage, se * tw * 4, cudaMemcpyHostToDevice, v->st);
        if (ce == cudaSuccess)
            ce = launch_vagg(ptrs, zs, tw, w, h, pp, 1, 1u, v->d_out, pp, (long long)h * pp, v->st);
        float *down = v->h_stage + v->in_elems;
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(down, v->d_out, (size_t)h * pp * 4, cudaMemcpyDeviceToHost, v->st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(v->st);
        if (ce != cudaSuccess) {
            set_err(err, errlen, "VAggregate: process frame failed. (%s)", cudaGetErrorString(ce));
            return -1;
        }
        copy_plane_out(dst->ptr[p], dst->stride[p], down, pp, w, h);
    }
    return 0;
}

void zb3d_vaggregate_free(zb3d_vagg *v) {
    if (!v) return;
    cudaSetDevice(v->device);
    if (v->st) cudaStreamSynchronize(v->st), cudaStreamDestroy(v->st);
    cudaFree(v->d_in);
    cudaFree(v->d_out);
    if (v->h_stage) cudaFreeHost(v->h_stage);
    delete v;
}

}  // extern "C"
