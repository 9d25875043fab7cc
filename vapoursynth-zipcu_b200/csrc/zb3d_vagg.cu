// Temporal aggregation of accumulator stacks (VAggregate / fused BM3Dv2).
//
// Compiled WITHOUT -use_fast_math: no flush-to-zero, IEEE division — the
// reference's vaggregate (vszipcu src/bm3d_vagg.cu:1-48) and its CPU aggPlane
// (src/bm3d.zig:1284-1317) both sum the 2r+1 slots in ascending order in FP32 and
// divide once, so composed and fused outputs are byte-identical.
#include <cuda_runtime.h>

namespace zb {

struct VaggArgs {
    const float *p[33];        // stacked entry buffer of window frame t
    int z[33];                 // slot of that stack holding this frame
    int tw, w, h, pitch;
    long long stack_plane_stride;  // floats between planes of a stack (tw*2*h*pitch)
    unsigned proc_mask;
    float *dst;
    int dst_pitch;
    long long dst_plane_stride;
};

__global__ void __launch_bounds__(256) zb_vagg(VaggArgs a) {
    const int x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
    const int plane = blockIdx.z;
    if (x >= a.w || y >= a.h || !((a.proc_mask >> plane) & 1)) return;
    const long long i = (long long)y * a.pitch + x;
    const long long ts = (long long)a.h * a.pitch;
    float sv = 0.0f, sw = 0.0f;
    for (int t = 0; t < a.tw; ++t) {
        const float *s = a.p[t] + plane * a.stack_plane_stride + (long long)a.z[t] * 2 * ts;
        sv = __fadd_rn(sv, s[i]);
        sw = __fadd_rn(sw, s[ts + i]);
    }
    a.dst[plane * a.dst_plane_stride + (long long)y * a.dst_pitch + x] = __fdiv_rn(sv, sw);
}

cudaError_t launch_vagg(const float *const *stacks, const int *z, int tw, int w, int h, int pitch, int nplanes,
                        unsigned proc_mask, float *dst, int dst_pitch, long long dst_plane_stride, cudaStream_t st) {
    if (tw < 1 || tw > 33) return cudaErrorInvalidValue;
    VaggArgs a;
    for (int t = 0; t < 33; ++t) {
        a.p[t] = t < tw ? stacks[t] : nullptr;
        a.z[t] = t < tw ? z[t] : 0;
    }
    a.tw = tw;
    a.w = w;
    a.h = h;
    a.pitch = pitch;
    a.stack_plane_stride = (long long)tw * 2 * h * pitch;
    a.proc_mask = proc_mask;
    a.dst = dst;
    a.dst_pitch = dst_pitch;
    a.dst_plane_stride = dst_plane_stride;
    zb_vagg<<<dim3((w + 31) / 32, (h + 7) / 8, nplanes), dim3(32, 8), 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace zb
