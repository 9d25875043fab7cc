/*
 * ORACLE — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the vszipcu BM3D path (BM3D / BM3Dv2 / VAggregate) used to
 * check the CUDA product path and, timed, as the CPU baseline.  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arms may load it.
 * The product never links, loads or calls anything in this directory.
 *
 * Two precisions, on purpose:
 *   - Block matching is restated in FP32 with the exact operation order and FMA
 *     contraction of the reference kernel, under flush-to-zero (the reference is
 *     compiled with -use_fast_math), so match indices can be compared bit for bit.
 *   - The 3D transforms, shrinkage and aggregation run in FP64 from the
 *     mathematical definition of each transform: this is the FP64 oracle against
 *     which the FP32 GPU output error is stated.
 *
 * Reference citations (paths inside the vszipcu project):
 *   distances          src/bm3d.cu:282-390
 *   block geometry     src/bm3d.cu:585-595
 *   spatial search     src/bm3d.cu:614-660
 *   temporal search    src/bm3d.cu:663-756
 *   self inclusion     src/bm3d.cu:758-788
 *   transforms         src/bm3d.cu:32-280 (linear maps restated in FP64)
 *   hard threshold     src/bm3d.cu:415-478
 *   Wiener             src/bm3d.cu:480-546
 *   aggregation        src/bm3d.cu:861-922
 *   VAggregate / aggZ  src/bm3d.zig:46-48, 1284-1317
 */
#include <float.h>
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <xmmintrin.h>

enum { OC_SSD = 0, OC_SAD = 1, OC_ZSSD = 2, OC_ZSAD = 3, OC_SSD_NORM = 4 };
enum { OC_DCT = 0, OC_HAAR = 1, OC_WHT = 2, OC_BIOR15 = 3 };

#define OC_FLT_MAX 3.402823466e+38f
#define OC_FLT_EPS 1.192092896e-07f

/* One filter invocation over one "entry" (a plane, or Y+U+V for CBM3D). */
typedef struct oc_cfg {
    int w, h, stride;      /* plane geometry, stride in elements */
    int nplanes;           /* 1, or 3 when chroma */
    int radius;            /* temporal radius r; tw = 2r+1 */
    int final_;            /* 1: clip 0 = ref (basic estimate), clip 1 = noisy */
    int chroma;
    float sigma[3];        /* already multiplied by the hard/Wiener factor */
    int bs, range, ps_num, ps_range;
    int bm_error, t2d, t1d;
    int nthreads;
    float extractor;       /* 2^extractor_exp, or 0 (src/bm3d.zig:1056-1057) */
} oc_cfg;

/* ------------------------------------------------------------------------- */
/* FP32 exact-order distances (src/bm3d.cu:282-390).                          */
/* A lane of the reference holds one patch column; rows i are accumulated in   */
/* two interleaved partials (even rows, odd rows), the column result is        */
/* e0+e1 and the 8 columns are summed by an xor butterfly 1,2,4, i.e.          */
/* ((s0+s1)+(s2+s3))+((s4+s5)+(s6+s7)).                                        */
/* ------------------------------------------------------------------------- */
static inline float tree8(const float s[8]) {
    return ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
}

static inline float col_sum8(const float *p, int stride) {
    /* (((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7))) down one column (src/bm3d.cu:319) */
    return ((p[0] + p[stride]) + (p[2 * stride] + p[3 * stride])) +
           ((p[4 * stride] + p[5 * stride]) + (p[6 * stride] + p[7 * stride]));
}

static float dist_ssd(const float *a, const float *b, int stride) {
    float s[8];
    for (int j = 0; j < 8; ++j) {
        float d[8];
        for (int i = 0; i < 8; ++i) d[i] = a[i * stride + j] - b[i * stride + j];
        float e0 = d[0] * d[0];
        float e1 = d[1] * d[1];
        e0 = fmaf(d[2], d[2], e0);
        e1 = fmaf(d[3], d[3], e1);
        e0 = fmaf(d[4], d[4], e0);
        e1 = fmaf(d[5], d[5], e1);
        e0 = fmaf(d[6], d[6], e0);
        e1 = fmaf(d[7], d[7], e1);
        s[j] = e0 + e1;
    }
    return tree8(s);
}

static float dist_sad(const float *a, const float *b, int stride) {
    float s[8];
    for (int j = 0; j < 8; ++j) {
        float e0 = 0.0f, e1 = 0.0f;
        for (int i = 0; i < 8; i += 2) {
            e0 += fabsf(a[i * stride + j] - b[i * stride + j]);
            e1 += fabsf(a[(i + 1) * stride + j] - b[(i + 1) * stride + j]);
        }
        s[j] = e0 + e1;
    }
    return tree8(s);
}

static float patch_mean(const float *a, int stride) {
    float s[8];
    for (int j = 0; j < 8; ++j) s[j] = col_sum8(a + j, stride);
    return tree8(s) * (1.0f / 64.f);
}

static float dist_zssd(const float *a, const float *b, int stride) {
    float dm = patch_mean(a, stride) - patch_mean(b, stride);
    float s[8];
    for (int j = 0; j < 8; ++j) {
        float v[8];
        for (int i = 0; i < 8; ++i) v[i] = (a[i * stride + j] - b[i * stride + j]) - dm;
        float e0 = v[0] * v[0];
        float e1 = v[1] * v[1];
        e0 = fmaf(v[2], v[2], e0);
        e1 = fmaf(v[3], v[3], e1);
        e0 = fmaf(v[4], v[4], e0);
        e1 = fmaf(v[5], v[5], e1);
        e0 = fmaf(v[6], v[6], e0);
        e1 = fmaf(v[7], v[7], e1);
        s[j] = e0 + e1;
    }
    return tree8(s);
}

static float dist_zsad(const float *a, const float *b, int stride) {
    float dm = patch_mean(a, stride) - patch_mean(b, stride);
    float s[8];
    for (int j = 0; j < 8; ++j) {
        float e0 = 0.0f, e1 = 0.0f;
        for (int i = 0; i < 8; i += 2) {
            e0 += fabsf((a[i * stride + j] - b[i * stride + j]) - dm);
            e1 += fabsf((a[(i + 1) * stride + j] - b[(i + 1) * stride + j]) - dm);
        }
        s[j] = e0 + e1;
    }
    return tree8(s);
}

static float sq_norm(const float *a, int stride) {
    float s[8];
    for (int j = 0; j < 8; ++j) {
        float e0 = a[j] * a[j];
        float e1 = a[stride + j] * a[stride + j];
        for (int i = 2; i < 8; i += 2) {
            e0 = fmaf(a[i * stride + j], a[i * stride + j], e0);
            e1 = fmaf(a[(i + 1) * stride + j], a[(i + 1) * stride + j], e1);
        }
        s[j] = e0 + e1;
    }
    return tree8(s);
}

/* ssd/norm: the reference computes sqrt and the final division with the GPU's
 * approximate instructions; IEEE sqrtf / division here, so indices for this
 * metric are approximate (documented). */
static float dist_ssd_norm(const float *a, const float *b, int stride) {
    float na = sqrtf(sq_norm(a, stride));
    float nb = sqrtf(sq_norm(b, stride));
    float s[8];
    for (int j = 0; j < 8; ++j) {
        float e0 = a[j] * b[j];
        float e1 = a[stride + j] * b[stride + j];
        for (int i = 2; i < 8; i += 2) {
            e0 = fmaf(a[i * stride + j], b[i * stride + j], e0);
            e1 = fmaf(a[(i + 1) * stride + j], b[(i + 1) * stride + j], e1);
        }
        s[j] = e0 + e1;
    }
    return 2.0f - 2.0f * tree8(s) / fmaf(na, nb, OC_FLT_EPS);
}

static inline float dist(int metric, const float *a, const float *b, int stride) {
    switch (metric) {
    case OC_SAD: return dist_sad(a, b, stride);
    case OC_ZSSD: return dist_zssd(a, b, stride);
    case OC_ZSAD: return dist_zsad(a, b, stride);
    case OC_SSD_NORM: return dist_ssd_norm(a, b, stride);
    default: return dist_ssd(a, b, stride);
    }
}

/* ------------------------------------------------------------------------- */
/* Sorted top-8 list with the reference's insertion rule (src/bm3d.cu:641-653):*/
/* a candidate enters at the first slot whose error is strictly greater, later */
/* slots shift down and the last one drops.                                    */
/* ------------------------------------------------------------------------- */
typedef struct { float e[8]; int x[8], y[8], z[8]; } top8;

static inline void top8_init(top8 *l, int z) {
    for (int i = 0; i < 8; ++i) { l->e[i] = OC_FLT_MAX; l->x[i] = 0; l->y[i] = 0; l->z[i] = z; }
}

static inline void top8_insert(top8 *l, float err, int x, int y, int z) {
    if (!(err < l->e[7])) return;
    int s = 0;
    while (!(err < l->e[s])) ++s;
    for (int i = 7; i > s; --i) { l->e[i] = l->e[i - 1]; l->x[i] = l->x[i - 1]; l->y[i] = l->y[i - 1]; l->z[i] = l->z[i - 1]; }
    l->e[s] = err; l->x[s] = x; l->y[s] = y; l->z[s] = z;
}

static inline int imax(int a, int b) { return a > b ? a : b; }
static inline int imin(int a, int b) { return a < b ? a : b; }

/* Block matching for the reference block at (x, y); planes[t] = matching plane of frame t.
 * Cloned for x86-64-v3 so fmaf() becomes one FMA instruction where the CPU has it. */
__attribute__((target_clones("arch=x86-64-v3", "default")))
static void match_block(const oc_cfg *c, const float *const *mplanes, int x, int y, top8 *out) {
    const int W = c->w, H = c->h, S = c->stride, R = c->range, r = c->radius;
    const float *cur = mplanes[r] + (size_t)y * S + x;
    top8 l;
    top8_init(&l, r);
    {
        int left = imax(x - R, 0), right = imin(x + R, W - 8);
        int top = imax(y - R, 0), bottom = imin(y + R, H - 8);
        for (int row = top; row <= bottom; ++row)
            for (int col = left; col <= right; ++col) {
                float e = dist(c->bm_error, cur, mplanes[r] + (size_t)row * S + col, S);
                top8_insert(&l, e, col, row, r);
            }
    }
    if (r > 0) {
        top8 centre = l;
        for (int dir = -1; dir <= 1; dir += 2) {
            top8 last = centre;
            for (int t = 1; t <= r; ++t) {
                int zt = r + dir * t;
                top8 fl;
                top8_init(&fl, 0);
                for (int i = 0; i < c->ps_num; ++i) {
                    int xx = last.x[i], yy = last.y[i];
                    int left = imax(xx - c->ps_range, 0), right = imin(xx + c->ps_range, W - 8);
                    int top = imax(yy - c->ps_range, 0), bottom = imin(yy + c->ps_range, H - 8);
                    for (int row = top; row <= bottom; ++row)
                        for (int col = left; col <= right; ++col) {
                            float e = dist(c->bm_error, cur, mplanes[zt] + (size_t)row * S + col, S);
                            top8_insert(&fl, e, col, row, 0);
                        }
                }
                for (int i = 0; i < c->ps_num; ++i) top8_insert(&l, fl.e[i], fl.x[i], fl.y[i], zt);
                last = fl;
            }
        }
    }
    /* self inclusion (src/bm3d.cu:758-788) */
    int found = 0;
    for (int i = 0; i < 8; ++i)
        if (l.x[i] == x && l.y[i] == y && l.z[i] == r) found = 1;
    if (!found) {
        for (int i = 7; i > 0; --i) { l.e[i] = l.e[i - 1]; l.x[i] = l.x[i - 1]; l.y[i] = l.y[i - 1]; l.z[i] = l.z[i - 1]; }
        l.e[0] = 0.0f; l.x[0] = x; l.y[0] = y; l.z[0] = r;
    }
    *out = l;
}

/* ------------------------------------------------------------------------- */
/* FP64 transforms.  Each 8-point transform of the reference is an            */
/* unnormalised linear map; the oracle builds its 8x8 matrix once in FP64.     */
/* DCT: 4 x orthonormal DCT-II forward, 4 x orthonormal DCT-III inverse.       */
/* Haar / WHT / bior1.5: the reference's own linear maps (src/bm3d.cu:125-280),*/
/* restated from their output formulas, including the reference's inverse Haar */
/* (which reuses coefficients 2 and 4 for every detail term).                  */
/* ------------------------------------------------------------------------- */
static void fwd_haar(const double x[8], double v[8]) {
    const double s2 = sqrt(2.0);
    double t1 = x[0] + x[1], t2 = x[0] - x[1], t3 = x[2] + x[3], t4 = x[2] - x[3];
    double t5 = x[4] + x[5], t6 = x[4] - x[5], t7 = x[6] + x[7], t8 = x[6] - x[7];
    double t9 = t1 + t3, t10 = s2 * (t1 - t3), t11 = t5 + t7, t12 = s2 * (t5 - t7);
    v[0] = s2 * (t9 + t11); v[1] = s2 * (t9 - t11); v[2] = s2 * t10; v[3] = s2 * t12;
    v[4] = 2 * s2 * t2; v[5] = 2 * s2 * t4; v[6] = 2 * s2 * t6; v[7] = 2 * s2 * t8;
}
static void inv_haar(const double v[8], double x[8]) {
    const double s2 = sqrt(2.0);
    double t1 = v[0] + v[1], t2 = v[0] - v[1];
    double a = s2 * v[2], b = 2 * v[4];
    x[0] = s2 * (t1 + (a + b)); x[1] = s2 * (t1 + (a - b));
    x[2] = s2 * (t1 + (-a + b)); x[3] = s2 * (t1 + (-a - b));
    x[4] = s2 * (t2 + (a + b)); x[5] = s2 * (t2 + (a - b));
    x[6] = s2 * (t2 + (-a + b)); x[7] = s2 * (t2 + (-a - b));
}
static void wht8(const double x[8], double v[8]) {
    const double s2 = sqrt(2.0);
    double t1 = x[0] + x[1], t2 = x[0] - x[1], t3 = x[2] + x[3], t4 = x[2] - x[3];
    double t5 = x[4] + x[5], t6 = x[4] - x[5], t7 = x[6] + x[7], t8 = x[6] - x[7];
    double t9 = t1 + t3, t10 = t1 - t3, t11 = t2 + t4, t12 = t2 - t4;
    double t13 = t5 + t7, t14 = t5 - t7, t15 = t6 + t8, t16 = t6 - t8;
    v[0] = s2 * (t9 + t13); v[1] = s2 * (t9 - t13); v[2] = s2 * (t10 - t14); v[3] = s2 * (t10 + t14);
    v[4] = s2 * (t12 + t16); v[5] = s2 * (t12 - t16); v[6] = s2 * (t11 - t15); v[7] = s2 * (t11 + t15);
}
/* bior1.5 analysis / synthesis weights, restated in FP64 from src/bm3d.cu:215-279. */
static void fwd_bior(const double x[8], double v[8]) {
    const double a0 = 1.414213562373095048801688724209698078569671875;
    const double a1 = 0.877670597010003062405456290501163901200537360;
    const double a2 = 1.797135031972863413496886690073811797696338403;
    const double a3 = 2.277437593371384746027611934034934695963515886;
    const double a4 = 1.609389232649111887192845766718020518480884560;
    const double a5 = 0.334024180361136429417383083658457088741315663;
    const double a6 = 2.828427124746190097603377448419396157139343751;
    double t1 = x[0] + x[3], t2 = x[0] - x[3], t3 = x[1] + x[2], t4 = x[1] - x[2];
    double t5 = x[4] + x[7], t6 = x[4] - x[7], t7 = x[5] + x[6], t8 = x[5] - x[6];
    v[0] = a0 * (t1 + t5 + t3 + t7);
    v[1] = a1 * (t1 - t5) + a2 * (t3 - t7);
    v[2] = a3 * t2 + a4 * t4 + a5 * (t8 - t6);
    v[3] = a3 * t6 + a4 * t8 + a5 * (t4 - t2);
    v[4] = a6 * (x[0] - x[1]); v[5] = a6 * (x[2] - x[3]);
    v[6] = a6 * (x[4] - x[5]); v[7] = a6 * (x[6] - x[7]);
}
static void inv_bior(const double v[8], double x[8]) {
    const double b0 = 1.414213562373095048801688724209698078569671875;
    const double b1 = 1.495435764250674860795011090214036706658653686;
    const double b2 = 2.058234225009388964222454285384072231477027482;
    const double b3 = 0.486135912065751423025580498947083714508324707;
    const double b4 = 2.828427124746190097603377448419396157139343751;
    double t1 = b0 * v[0], t2 = b1 * v[1], t3 = b2 * v[2], t4 = b2 * v[3];
    double t5 = b4 * v[4], t6 = b3 * v[4], t7 = b4 * v[5], t8 = b3 * v[5];
    double t9 = b4 * v[6], t10 = b3 * v[6], t11 = b4 * v[7], t12 = b3 * v[7];
    double t13 = t1 + t2, t14 = t1 - t2, t15 = t8 - t12, t16 = t6 - t10;
    x[0] = (t13 + t3) + (t5 - t15); x[1] = (t13 + t3) - (t5 + t15);
    x[2] = (t13 - t3) + (t16 + t7); x[3] = (t13 - t3) + (t16 - t7);
    x[4] = (t14 + t4) + (t15 + t9); x[5] = (t14 + t4) + (t15 - t9);
    x[6] = (t14 - t4) - (t16 - t11); x[7] = (t14 - t4) - (t16 + t11);
}

static double g_fwd[4][8][8], g_inv[4][8][8];
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

static void build_matrices(void) {
    const double pi = 3.14159265358979323846264338327950288;
    for (int k = 0; k < 8; ++k)
        for (int n = 0; n < 8; ++n) {
            double a = (k == 0) ? sqrt(1.0 / 8.0) : sqrt(2.0 / 8.0);
            double c = a * cos(pi * (2 * n + 1) * k / 16.0);
            g_fwd[OC_DCT][k][n] = 4.0 * c;
            g_inv[OC_DCT][n][k] = 4.0 * c;
        }
    for (int n = 0; n < 8; ++n) {
        double e[8] = {0}, o[8];
        e[n] = 1.0;
        fwd_haar(e, o); for (int k = 0; k < 8; ++k) g_fwd[OC_HAAR][k][n] = o[k];
        inv_haar(e, o); for (int k = 0; k < 8; ++k) g_inv[OC_HAAR][k][n] = o[k];
        wht8(e, o);     for (int k = 0; k < 8; ++k) { g_fwd[OC_WHT][k][n] = o[k]; g_inv[OC_WHT][k][n] = o[k]; }
        fwd_bior(e, o); for (int k = 0; k < 8; ++k) g_fwd[OC_BIOR15][k][n] = o[k];
        inv_bior(e, o); for (int k = 0; k < 8; ++k) g_inv[OC_BIOR15][k][n] = o[k];
    }
}

/* g[i][r][c]: apply m along axis (0 = patch index, 1 = row, 2 = column). */
static void apply_axis(double g[8][8][8], const double m[8][8], int axis) {
    double in[8], out[8];
    for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b) {
            for (int n = 0; n < 8; ++n)
                in[n] = axis == 0 ? g[n][a][b] : axis == 1 ? g[a][n][b] : g[a][b][n];
            for (int k = 0; k < 8; ++k) {
                double s = 0.0;
                for (int n = 0; n < 8; ++n) s += m[k][n] * in[n];
                out[k] = s;
            }
            for (int k = 0; k < 8; ++k) {
                if (axis == 0) g[k][a][b] = out[k];
                else if (axis == 1) g[a][k][b] = out[k];
                else g[a][b][k] = out[k];
            }
        }
}

static void fwd3(double g[8][8][8], int t2d, int t1d) {
    apply_axis(g, g_fwd[t2d], 1);
    apply_axis(g, g_fwd[t2d], 2);
    apply_axis(g, g_fwd[t1d], 0);
}
static void inv3(double g[8][8][8], int t2d, int t1d) {
    apply_axis(g, g_inv[t2d], 1);
    apply_axis(g, g_inv[t2d], 2);
    apply_axis(g, g_inv[t1d], 0);
}

/* ------------------------------------------------------------------------- */
/* Driver: match every block, filter its group in FP64, aggregate.            */
/* ------------------------------------------------------------------------- */
typedef struct {
    const oc_cfg *c;
    const float *const *src;   /* [clip][plane][t] plane pointers */
    int nbx, nby;
    int32_t *matches;          /* [nby][nbx][8][3] or NULL */
    /* per-chunk group results */
    int chunk_begin, chunk_end;
    double *gvals;             /* [chunk][nplanes][512] */
    double *gw;                /* [chunk][nplanes] */
    int8_t *gdone;             /* [chunk][nplanes] processed flag */
    top8 *glist;               /* [chunk] */
    int next;                  /* work counter (atomic) */
} oc_job;

static void block_xy(const oc_cfg *c, int bi, int nbx, int *x, int *y) {
    int kx = bi % nbx, ky = bi / nbx;
    *x = imin(kx * c->bs, c->w - 8);
    *y = imin(ky * c->bs, c->h - 8);
}

static void filter_block(oc_job *j, int local) {
    const oc_cfg *c = j->c;
    const int S = c->stride, tw = 2 * c->radius + 1, np = c->nplanes;
    int bi = j->chunk_begin + local;
    int x, y;
    block_xy(c, bi, j->nbx, &x, &y);
    const float *mplanes[33];
    for (int t = 0; t < tw; ++t) mplanes[t] = j->src[(0 * np + 0) * tw + t];
    top8 l;
    match_block(c, mplanes, x, y, &l);
    j->glist[local] = l;
    if (j->matches) {
        int32_t *m = j->matches + (size_t)bi * 24;
        for (int i = 0; i < 8; ++i) { m[3 * i] = l.x[i]; m[3 * i + 1] = l.y[i]; m[3 * i + 2] = l.z[i]; }
    }
    static const double inv4096 = 1.0 / 4096.0;
    for (int p = 0; p < np; ++p) {
        double sigma = (double)c->sigma[p];
        double *out = j->gvals + ((size_t)local * np + p) * 512;
        j->gdone[(size_t)local * np + p] = 0;
        if (c->chroma && c->sigma[p] < OC_FLT_EPS) continue;
        double g[8][8][8], rg[8][8][8];
        int nclip = c->final_ ? 1 : 0;
        for (int i = 0; i < 8; ++i) {
            const float *sp = j->src[(nclip * np + p) * tw + l.z[i]] + (size_t)l.y[i] * S + l.x[i];
            const float *rp = j->src[(0 * np + p) * tw + l.z[i]] + (size_t)l.y[i] * S + l.x[i];
            for (int r = 0; r < 8; ++r)
                for (int q = 0; q < 8; ++q) {
                    g[i][r][q] = sp[r * S + q];
                    rg[i][r][q] = rp[r * S + q];
                }
        }
        double weight;
        fwd3(g, c->t2d, c->t1d);
        if (!c->final_) {
            double k = 0.0;
            for (int i = 0; i < 8; ++i)
                for (int r = 0; r < 8; ++r)
                    for (int q = 0; q < 8; ++q) {
                        double thr = (i == 0 && r == 0 && q == 0) ? 0.0 : sigma;
                        int keep = fabs(g[i][r][q]) >= thr;
                        k += keep;
                        g[i][r][q] = keep ? g[i][r][q] * inv4096 : 0.0;
                    }
            weight = 1.0 / k;
        } else {
            fwd3(rg, c->t2d, c->t1d);
            double k = 0.0, s2 = sigma * sigma;
            for (int i = 0; i < 8; ++i)
                for (int r = 0; r < 8; ++r)
                    for (int q = 0; q < 8; ++q) {
                        double rv = rg[i][r][q];
                        double coeff = (rv * rv) / (rv * rv + s2);
                        if (i == 0 && r == 0 && q == 0) coeff = 1.0;
                        k += coeff * coeff;
                        g[i][r][q] = g[i][r][q] * coeff * inv4096;
                    }
            weight = 1.0 / k;
        }
        inv3(g, c->t2d, c->t1d);
        for (int i = 0; i < 8; ++i)
            for (int r = 0; r < 8; ++r)
                for (int q = 0; q < 8; ++q) out[(i * 8 + r) * 8 + q] = g[i][r][q];
        j->gw[(size_t)local * np + p] = weight;
        j->gdone[(size_t)local * np + p] = 1;
    }
}

static void *worker(void *arg) {
    oc_job *j = (oc_job *)arg;
    /* The reference is built with -use_fast_math: FP32 results and inputs are
     * flushed to zero.  FTZ|DAZ reproduces that for the FP32 matching; the FP64
     * filtering is unaffected at any magnitude it reaches. */
    _mm_setcsr(_mm_getcsr() | 0x8040);
    int n = j->chunk_end - j->chunk_begin;
    for (;;) {
        int i = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (i >= n) break;
        filter_block(j, i);
    }
    return NULL;
}

/*
 * Run one BM3D pass over one entry.
 *   src   : [clip][plane][t] plane pointers; clip 0 is the matching clip
 *           (the noisy clip, or the basic estimate when final_).
 *   num,den: [plane][t][h][w] FP64 accumulators, zeroed by the caller.
 *   matches: optional [nby][nbx][8][3] (x, y, z) match lists.
 * Returns the number of reference blocks.
 */
int oracle_bm3d_pass(const oc_cfg *c, const float *const *src, double *num, double *den, int32_t *matches) {
    pthread_once(&g_once, build_matrices);
    const int W = c->w, H = c->h, tw = 2 * c->radius + 1, np = c->nplanes;
    int nbx = (W - 8 + c->bs - 1) / c->bs + 1;
    int nby = (H - 8 + c->bs - 1) / c->bs + 1;
    int nblocks = nbx * nby;
    int nthreads = c->nthreads > 0 ? c->nthreads : 1;
    if (nthreads > 256) nthreads = 256;
    const int CHUNK = 4096;
    oc_job j;
    memset(&j, 0, sizeof j);
    j.c = c; j.src = src; j.nbx = nbx; j.nby = nby; j.matches = matches;
    j.gvals = (double *)malloc(sizeof(double) * CHUNK * np * 512);
    j.gw = (double *)malloc(sizeof(double) * CHUNK * np);
    j.gdone = (int8_t *)malloc(CHUNK * np);
    j.glist = (top8 *)malloc(sizeof(top8) * CHUNK);
    if (!j.gvals || !j.gw || !j.gdone || !j.glist) {
        free(j.gvals); free(j.gw); free(j.gdone); free(j.glist);
        return -1;
    }
    pthread_t th[256];
    for (int b0 = 0; b0 < nblocks; b0 += CHUNK) {
        j.chunk_begin = b0;
        j.chunk_end = imin(b0 + CHUNK, nblocks);
        j.next = 0;
        for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, worker, &j);
        for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
        /* deterministic, sequential aggregation in block order.  With an
         * extractor E the reference rounds every contribution to the float grid
         * around E, (v + E) - E (src/bm3d.cu:884-885); modelled here as
         * f32(v + E) - E so the FP64 oracle shares that quantisation. */
        for (int b = 0; b < j.chunk_end - j.chunk_begin; ++b) {
            const top8 *l = &j.glist[b];
            for (int p = 0; p < np; ++p) {
                if (!j.gdone[(size_t)b * np + p]) continue;
                const double *v = j.gvals + ((size_t)b * np + p) * 512;
                double w = j.gw[(size_t)b * np + p];
                double E = (double)c->extractor;
                double wq = E != 0.0 ? (double)(float)(w + E) - E : w;
                for (int i = 0; i < 8; ++i) {
                    size_t base = ((size_t)(p * tw + l->z[i]) * H + l->y[i]) * W + l->x[i];
                    for (int r = 0; r < 8; ++r)
                        for (int q = 0; q < 8; ++q) {
                            double val = w * v[(i * 8 + r) * 8 + q];
                            if (E != 0.0) val = (double)(float)(val + E) - E;
                            num[base + (size_t)r * W + q] += val;
                            den[base + (size_t)r * W + q] += wq;
                        }
                }
            }
        }
    }
    free(j.gvals); free(j.gw); free(j.gdone); free(j.glist);
    return nblocks;
}

/* Only the matching stage, FP32 exact order, for index parity. */
typedef struct { const oc_cfg *c; const float *const *mplanes; int nbx, nblocks; int32_t *matches; int next; } oc_mjob;

static void *match_worker(void *arg) {
    oc_mjob *j = (oc_mjob *)arg;
    _mm_setcsr(_mm_getcsr() | 0x8040);
    for (;;) {
        int bi = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (bi >= j->nblocks) break;
        int x, y;
        block_xy(j->c, bi, j->nbx, &x, &y);
        top8 l;
        match_block(j->c, j->mplanes, x, y, &l);
        int32_t *m = j->matches + (size_t)bi * 24;
        for (int i = 0; i < 8; ++i) { m[3 * i] = l.x[i]; m[3 * i + 1] = l.y[i]; m[3 * i + 2] = l.z[i]; }
    }
    return NULL;
}

int oracle_match(const oc_cfg *c, const float *const *mplanes, int32_t *matches) {
    int nbx = (c->w - 8 + c->bs - 1) / c->bs + 1;
    int nby = (c->h - 8 + c->bs - 1) / c->bs + 1;
    oc_mjob j = {c, mplanes, nbx, nbx * nby, matches, 0};
    int nthreads = c->nthreads > 0 ? (c->nthreads > 256 ? 256 : c->nthreads) : 1;
    pthread_t th[256];
    for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, match_worker, &j);
    for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
    return nbx * nby;
}

/* Error of one candidate, exposed for unit tests of the distance order. */
float oracle_distance(int metric, const float *a, const float *b, int stride) {
    unsigned int old = _mm_getcsr();
    _mm_setcsr(old | 0x8040);
    float e = dist(metric, a, b, stride);
    _mm_setcsr(old);
    return e;
}

/* aggZ (src/bm3d.zig:46-48) */
int oracle_agg_z(int i, int n, int nframes, int radius) {
    return imin(imax(2 * radius - i, n - nframes + 1 + radius), n + radius);
}

/*
 * VAggregate of one plane (src/bm3d.zig:1284-1317): stacks[i] is the stacked
 * BM3D output of frame clamp(n-r+i) (height h*2*tw, FP32); ascending float sums,
 * IEEE division.  No flush-to-zero, like the reference's CPU path.
 */
void oracle_vaggregate_plane(float *dst, const float *const *stacks, int w, int h, int stride,
                             int radius, int n, int nframes) {
    int tw = 2 * radius + 1;
    for (int y = 0; y < h; ++y) {
        const float *rows[33], *wts[33];
        for (int i = 0; i < tw; ++i) {
            int z = oracle_agg_z(i, n, nframes, radius);
            size_t base = ((size_t)z * 2 * h + y) * stride;
            rows[i] = stacks[i] + base;
            wts[i] = stacks[i] + base + (size_t)h * stride;
        }
        for (int x = 0; x < w; ++x) {
            float acc = 0.0f, acw = 0.0f;
            for (int i = 0; i < tw; ++i) { acc += rows[i][x]; acw += wts[i][x]; }
            dst[(size_t)y * stride + x] = acc / acw;
        }
    }
}
