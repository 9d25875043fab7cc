// Match-list helpers shared by the matching kernels (zb3d_kernels.cu, zb3d_match_tc.cu).
#pragma once
#include <cuda_runtime.h>

#include "zb3d_args.h"

namespace zb {

#define ZB_FLT_MAX 3.402823466e+38f
#define ZB_FLT_EPS 1.192092896e-07f

// ---------------------------------------------------------------------------
// Top-8 list: sorted by distance; a candidate enters before the first strictly
// larger entry (vszipcu src/bm3d.cu:641-653), so ties keep scan order.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void top8_insert(float (&e)[8], int (&q)[8], float err, int pos) {
#pragma unroll
    for (int i = 7; i > 0; --i) {
        const bool ci = err < e[i];
        const bool cp = err < e[i - 1];
        e[i] = cp ? e[i - 1] : (ci ? err : e[i]);
        q[i] = cp ? q[i - 1] : (ci ? pos : q[i]);
    }
    if (err < e[0]) {
        e[0] = err;
        q[0] = pos;
    }
}

// The same strict-less insertion into a list of K entries.  Its entries are the first K
// of the 8-entry list that the same candidates would build (stable in scan order).
template <int K>
__device__ __forceinline__ void topk_insert(float (&e)[K], int (&q)[K], float err, int pos) {
#pragma unroll
    for (int i = K - 1; i > 0; --i) {
        const bool ci = err < e[i];
        const bool cp = err < e[i - 1];
        e[i] = cp ? e[i - 1] : (ci ? err : e[i]);
        q[i] = cp ? q[i - 1] : (ci ? pos : q[i]);
    }
    if (err < e[0]) {
        e[0] = err;
        q[0] = pos;
    }
}

__device__ __forceinline__ void top8_insert_z(float (&e)[8], int (&q)[8], int (&z)[8], float err, int pos, int zz) {
#pragma unroll
    for (int i = 7; i > 0; --i) {
        const bool ci = err < e[i];
        const bool cp = err < e[i - 1];
        e[i] = cp ? e[i - 1] : (ci ? err : e[i]);
        q[i] = cp ? q[i - 1] : (ci ? pos : q[i]);
        z[i] = cp ? z[i - 1] : (ci ? zz : z[i]);
    }
    if (err < e[0]) {
        e[0] = err;
        q[0] = pos;
        z[0] = zz;
    }
}

__device__ __forceinline__ int pack_pos(int x, int y) { return x | (y << 16); }
__device__ __forceinline__ int pos_x(int p) { return p & 0xffff; }
__device__ __forceinline__ int pos_y(int p) { return (int)((unsigned)p >> 16); }

// Writes a finished list (with self inclusion at radius 0) and its distances.
__device__ __forceinline__ void store_list(const MatchArgs &a, long long bi, int xb, int y, float (&e)[8],
                                           int (&q)[8]) {
    const int self = pack_pos(xb, y);
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
    int2 *out = a.list + bi * 8;
    const int zr = a.radius << 24;
#pragma unroll
    for (int i = 0; i < 8; ++i) out[i] = make_int2(pos_x(q[i]), pos_y(q[i]) | zr);
    if (a.errs) {
#pragma unroll
        for (int i = 0; i < 8; ++i) a.errs[bi * 8 + i] = e[i];
    }
}

}  // namespace zb
