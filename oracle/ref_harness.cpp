// Reference-kernel harness — TEST INFRASTRUCTURE ONLY.
//
// Loads a cubin that oracle/build_ref.py compiled from the reference's own
// src/bm3d.cu (or src/bm3d_vagg.cu) and replays the reference host's launch
// sequence on device memory owned by the caller:
//   memsetD8(res, 0) ; bm3d<<<(ceil(ceil(W/(4bs))/WARPS), ceil(H/bs)), 32*WARPS>>>(res, src)
//   aggregate<<<(ceil(W/32), ceil(H/8), planes), (32, 8)>>>(dst, res)          (radius 0)
// (vszipcu src/bm3d.zig:375-401), and the fused temporal aggregation
//   vaggregate<<<(ceil(W/32), ceil(H/8), planes), (32, 8)>>>(dst, AggSrc)   (src/bm3d.zig:608-630).
// Pointers are CUDA device addresses passed as integers; the stream handle too.
#include <cuda.h>

#include <cstdint>
#include <cstdio>
#include <cstring>

namespace {

struct RefModule {
    CUmodule mod = nullptr;
    CUfunction bm3d = nullptr;
    CUfunction aggregate = nullptr;
    CUfunction vaggregate = nullptr;
};

// AggSrc of src/bm3d_vagg.cu:7-16, passed by value (400 bytes, 8-byte aligned).
struct AggSrc {
    unsigned long long p[33];
    int z[33];
};
static_assert(sizeof(AggSrc) == 400, "AggSrc layout");

int fail(char *err, int errlen, const char *what, CUresult r) {
    if (err && errlen > 0) {
        const char *s = nullptr;
        cuGetErrorString(r, &s);
        snprintf(err, errlen, "%s: %s", what, s ? s : "unknown CUDA error");
    }
    return (int)r ? (int)r : -1;
}

unsigned ceil_div(unsigned a, unsigned b) { return (a + b - 1) / b; }

bool ensure_context(char *err, int errlen) {
    if (cuInit(0) != CUDA_SUCCESS) {
        if (err) snprintf(err, errlen, "cuInit failed");
        return false;
    }
    CUcontext ctx = nullptr;
    cuCtxGetCurrent(&ctx);
    if (ctx) return true;
    CUdevice dev;
    if (cuDeviceGet(&dev, 0) != CUDA_SUCCESS || cuDevicePrimaryCtxRetain(&ctx, dev) != CUDA_SUCCESS ||
        cuCtxSetCurrent(ctx) != CUDA_SUCCESS) {
        if (err) snprintf(err, errlen, "could not make the primary context current");
        return false;
    }
    return true;
}

}  // namespace

extern "C" {

void *refh_load(const char *path, char *err, int errlen) {
    if (!ensure_context(err, errlen)) return nullptr;
    RefModule *m = new RefModule();
    CUresult r = cuModuleLoad(&m->mod, path);
    if (r != CUDA_SUCCESS) {
        fail(err, errlen, "cuModuleLoad", r);
        delete m;
        return nullptr;
    }
    if (cuModuleGetFunction(&m->bm3d, m->mod, "bm3d") != CUDA_SUCCESS) m->bm3d = nullptr;
    if (cuModuleGetFunction(&m->aggregate, m->mod, "aggregate") != CUDA_SUCCESS) m->aggregate = nullptr;
    if (cuModuleGetFunction(&m->vaggregate, m->mod, "vaggregate") != CUDA_SUCCESS) m->vaggregate = nullptr;
    return m;
}

void refh_unload(void *h) {
    RefModule *m = (RefModule *)h;
    if (!m) return;
    if (m->mod) cuModuleUnload(m->mod);
    delete m;
}

// Sets the dump pointer of a dump-variant module (int[nby][nbx][8][3]).
int refh_set_dump(void *h, unsigned long long dptr, char *err, int errlen) {
    RefModule *m = (RefModule *)h;
    CUdeviceptr sym;
    size_t bytes;
    CUresult r = cuModuleGetGlobal(&sym, &bytes, m->mod, "zb_ref_dump");
    if (r != CUDA_SUCCESS) return fail(err, errlen, "zb_ref_dump symbol", r);
    r = cuMemcpyHtoD(sym, &dptr, sizeof dptr);
    if (r != CUDA_SUCCESS) return fail(err, errlen, "set dump pointer", r);
    return 0;
}

// Sets the distance dump pointer of a dump-variant module (float[nby][nbx][8]; 0 = off).
int refh_set_dump_err(void *h, unsigned long long dptr, char *err, int errlen) {
    RefModule *m = (RefModule *)h;
    CUdeviceptr sym;
    size_t bytes;
    CUresult r = cuModuleGetGlobal(&sym, &bytes, m->mod, "zb_ref_dump_err");
    if (r != CUDA_SUCCESS) return fail(err, errlen, "zb_ref_dump_err symbol", r);
    r = cuMemcpyHtoD(sym, &dptr, sizeof dptr);
    if (r != CUDA_SUCCESS) return fail(err, errlen, "set distance dump pointer", r);
    return 0;
}

// memset(res) + bm3d (+ aggregate when dst != 0) on `stream`.
int refh_bm3d(void *h, unsigned long long res, unsigned long long src, unsigned long long dst, size_t res_bytes,
              int w, int hgt, int block_step, int warps, int agg_planes, unsigned long long stream, char *err,
              int errlen) {
    RefModule *m = (RefModule *)h;
    CUstream st = (CUstream)(uintptr_t)stream;
    CUresult r = cuMemsetD8Async((CUdeviceptr)res, 0, res_bytes, st);
    if (r != CUDA_SUCCESS) return fail(err, errlen, "memset res", r);
    unsigned groups_x = ceil_div((unsigned)w, 4u * (unsigned)block_step);
    void *args[] = {&res, &src};
    r = cuLaunchKernel(m->bm3d, ceil_div(groups_x, (unsigned)warps), ceil_div((unsigned)hgt, (unsigned)block_step), 1,
                       32u * (unsigned)warps, 1, 1, 0, st, args, nullptr);
    if (r != CUDA_SUCCESS) return fail(err, errlen, "launch bm3d", r);
    if (dst) {
        void *aargs[] = {&dst, &res};
        r = cuLaunchKernel(m->aggregate, ceil_div((unsigned)w, 32u), ceil_div((unsigned)hgt, 8u), (unsigned)agg_planes,
                           32, 8, 1, 0, st, aargs, nullptr);
        if (r != CUDA_SUCCESS) return fail(err, errlen, "launch aggregate", r);
    }
    return 0;
}

// vaggregate over tw accumulator stacks: ptrs[t] = stack base, z[t] = slot.
int refh_vagg(void *h, unsigned long long dst, const unsigned long long *ptrs, const int *z, int tw, int w, int hgt,
              int nplanes, unsigned long long stream, char *err, int errlen) {
    RefModule *m = (RefModule *)h;
    AggSrc s;
    memset(&s, 0, sizeof s);
    for (int t = 0; t < tw && t < 33; ++t) {
        s.p[t] = ptrs[t];
        s.z[t] = z[t];
    }
    void *args[] = {&dst, &s};
    CUresult r = cuLaunchKernel(m->vaggregate, ceil_div((unsigned)w, 32u), ceil_div((unsigned)hgt, 8u),
                                (unsigned)nplanes, 32, 8, 1, 0, (CUstream)(uintptr_t)stream, args, nullptr);
    if (r != CUDA_SUCCESS) return fail(err, errlen, "launch vaggregate", r);
    return 0;
}

int refh_bm3d_registers(void *h, int *regs, int *smem) {
    RefModule *m = (RefModule *)h;
    cuFuncGetAttribute(regs, CU_FUNC_ATTRIBUTE_NUM_REGS, m->bm3d);
    cuFuncGetAttribute(smem, CU_FUNC_ATTRIBUTE_SHARED_SIZE_BYTES, m->bm3d);
    return 0;
}

}  // extern "C"
