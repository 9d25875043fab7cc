// 8-point transforms of the BM3D 3D stack (forward and inverse).
//
// These are the unnormalised FFTW-style factorisations the reference uses
// (vszipcu src/bm3d.cu:32-280): DCT-II / DCT-III with gain 4 per axis, the
// reference's Haar pair (its inverse reuses coefficients 2 and 4 for every detail
// term, which is kept because the output must equal the reference's), the
// Walsh-Hadamard map (its own inverse) and bior1.5.  The arithmetic is restated
// with the same operation order so that, compiled with -use_fast_math like the
// reference, every coefficient comes out bit-identical; `a * b + c` is written
// where the reference writes its FMA/FMS/FNMS macros.
#pragma once

namespace zb {

enum Transform { T_DCT = 0, T_HAAR = 1, T_WHT = 2, T_BIOR15 = 3 };

struct Dct8 {
    static __device__ __forceinline__ void fwd(float *v) {
        const float k414 = (float)0.414213562373095048801688724209698078569671875;
        const float k1847 = (float)1.847759065022573512256366378793576573644833252;
        const float k198 = (float)0.198912367379658006911597622644676228597850501;
        const float k1961 = (float)1.961570560806460898252364472268478073947867462;
        const float k1414 = (float)1.414213562373095048801688724209698078569671875;
        const float k668 = (float)0.668178637919298919997757686523080761552472251;
        const float k1662 = (float)1.662939224605090474157576755235811513477121624;
        const float k707 = (float)0.707106781186547524400844362104849039284835938;
        float d07 = v[0] - v[7], s07 = v[0] + v[7];
        float d43 = v[4] - v[3], s43 = v[4] + v[3];
        float d25 = v[2] - v[5];
        float d16 = v[1] - v[6];
        float a = d25 + d16, s16 = v[1] + v[6];
        float b = d25 - d16, s25 = v[2] + v[5];
        float p = d07 - k707 * a;
        float q = d43 - k707 * b;
        v[3] = k1662 * (k668 * q + p);
        v[5] = -(k1662 * (q - k668 * p));
        float e = s07 + s43, f = s25 + s16;
        v[4] = k1414 * (e - f);
        v[0] = k1414 * (e + f);
        float g = k707 * a + d07;
        float h = k707 * b + d43;
        v[1] = k1961 * (g - k198 * h);
        v[7] = k1961 * (k198 * g + h);
        float m = s07 - s43, n = s25 - s16;
        v[2] = k1847 * (m - k414 * n);
        v[6] = k1847 * (k414 * m + n);
    }
    static __device__ __forceinline__ void inv(float *v) {
        const float k1662 = (float)1.662939224605090474157576755235811513477121624;
        const float k668 = (float)0.668178637919298919997757686523080761552472251;
        const float k1961 = (float)1.961570560806460898252364472268478073947867462;
        const float k198 = (float)0.198912367379658006911597622644676228597850501;
        const float k1847 = (float)1.847759065022573512256366378793576573644833252;
        const float k707 = (float)0.707106781186547524400844362104849039284835938;
        const float k414 = (float)0.414213562373095048801688724209698078569671875;
        const float k1414 = (float)1.414213562373095048801688724209698078569671875;
        float dc = v[0] * k1414;
        float c4 = v[4];
        float e0 = k1414 * c4 + dc;
        float e1 = dc - k1414 * c4;
        float c2 = v[2], c6 = v[6];
        float o0 = k414 * c6 + c2;
        float o1 = k414 * c2 - c6;
        float c1 = v[1], c7 = v[7], c5 = v[5], c3 = v[3];
        float s53 = c5 + c3, d35 = c3 - c5;
        float u = k707 * s53 + c1;
        float t = c7 - k707 * d35;
        float r = k707 * d35 + c7;
        float w = c1 - k707 * s53;
        float a0 = k1847 * o0 + e0;
        float b0 = k198 * r + u;
        v[7] = a0 - k1961 * b0;
        v[0] = k1961 * b0 + a0;
        float a1 = e1 - k1847 * o1;
        float b1 = k668 * w + t;
        v[5] = a1 - k1662 * b1;
        v[2] = k1662 * b1 + a1;
        float a2 = e0 - k1847 * o0;
        float b2 = r - k198 * u;
        v[3] = a2 - k1961 * b2;
        v[4] = k1961 * b2 + a2;
        float a3 = k1847 * o1 + e1;
        float b3 = w - k668 * t;
        v[6] = a3 - k1662 * b3;
        v[1] = k1662 * b3 + a3;
    }
};

struct Haar8 {
    static __device__ __forceinline__ void fwd(float *v) {
        const float r2 = (float)1.414213562373095048801688724209698078569671875;
        const float two = (float)2.0;
        float p01 = v[0] + v[1], m01 = v[0] - v[1];
        float p23 = v[2] + v[3], m23 = v[2] - v[3];
        float p45 = v[4] + v[5], m45 = v[4] - v[5];
        float p67 = v[6] + v[7], m67 = v[6] - v[7];
        float lo0 = p01 + p23, hi0 = r2 * (p01 - p23);
        float lo1 = p45 + p67, hi1 = r2 * (p45 - p67);
        const float s = r2;
        v[0] = s * (lo0 + lo1);
        v[1] = s * (lo0 - lo1);
        v[2] = s * hi0;
        v[3] = s * hi1;
        v[4] = s * two * m01;
        v[5] = s * two * m23;
        v[6] = s * two * m45;
        v[7] = s * two * m67;
    }
    static __device__ __forceinline__ void inv(float *v) {
        const float r2 = (float)1.414213562373095048801688724209698078569671875;
        const float two = (float)2.0;
        float sum = v[0] + v[1], dif = v[0] - v[1];
        float a = r2 * v[2] + two * v[4];
        float b = r2 * v[2] - two * v[4];
        float c = -r2 * v[2] + two * v[4];
        float d = -r2 * v[2] - two * v[4];
        float e = r2 * v[2] + two * v[4];
        float f = r2 * v[2] - two * v[4];
        float g = -r2 * v[2] + two * v[4];
        float h = -r2 * v[2] - two * v[4];
        const float s = r2;
        v[0] = s * (sum + a);
        v[1] = s * (sum + b);
        v[2] = s * (sum + c);
        v[3] = s * (sum + d);
        v[4] = s * (dif + e);
        v[5] = s * (dif + f);
        v[6] = s * (dif + g);
        v[7] = s * (dif + h);
    }
};

struct Wht8 {
    static __device__ __forceinline__ void apply(float *v) {
        const float r2 = (float)1.414213562373095048801688724209698078569671875;
        float a0 = v[0] + v[1], a1 = v[0] - v[1];
        float a2 = v[2] + v[3], a3 = v[2] - v[3];
        float a4 = v[4] + v[5], a5 = v[4] - v[5];
        float a6 = v[6] + v[7], a7 = v[6] - v[7];
        float b0 = a0 + a2, b1 = a0 - a2, b2 = a1 + a3, b3 = a1 - a3;
        float b4 = a4 + a6, b5 = a4 - a6, b6 = a5 + a7, b7 = a5 - a7;
        const float s = r2;
        v[0] = s * (b0 + b4);
        v[1] = s * (b0 - b4);
        v[2] = s * (b1 - b5);
        v[3] = s * (b1 + b5);
        v[4] = s * (b3 + b7);
        v[5] = s * (b3 - b7);
        v[6] = s * (b2 - b6);
        v[7] = s * (b2 + b6);
    }
    static __device__ __forceinline__ void fwd(float *v) { apply(v); }
    static __device__ __forceinline__ void inv(float *v) { apply(v); }
};

struct Bior15 {
    static __device__ __forceinline__ void fwd(float *v) {
        const float c0 = (float)1.414213562373095048801688724209698078569671875;
        const float c1 = (float)0.877670597010003062405456290501163901200537360;
        const float c2 = (float)1.797135031972863413496886690073811797696338403;
        const float c3 = (float)2.277437593371384746027611934034934695963515886;
        const float c4 = (float)1.609389232649111887192845766718020518480884560;
        const float c5 = (float)0.334024180361136429417383083658457088741315663;
        const float c6 = (float)2.828427124746190097603377448419396157139343751;
        float s03 = v[0] + v[3], d03 = v[0] - v[3];
        float s12 = v[1] + v[2], d12 = v[1] - v[2];
        float s47 = v[4] + v[7], d47 = v[4] - v[7];
        float s56 = v[5] + v[6], d56 = v[5] - v[6];
        float h0 = v[0] - v[1], h1 = v[2] - v[3];
        float h2 = v[4] - v[5], h3 = v[6] - v[7];
        v[0] = c0 * (s03 + s47 + s12 + s56);
        v[1] = c1 * (s03 - s47) + c2 * (s12 - s56);
        v[2] = c3 * d03 + c4 * d12 + c5 * (d56 - d47);
        v[3] = c3 * d47 + c4 * d56 + c5 * (d12 - d03);
        v[4] = c6 * h0;
        v[5] = c6 * h1;
        v[6] = c6 * h2;
        v[7] = c6 * h3;
    }
    static __device__ __forceinline__ void inv(float *v) {
        const float c0 = (float)1.414213562373095048801688724209698078569671875;
        const float c1 = (float)1.495435764250674860795011090214036706658653686;
        const float c2 = (float)2.058234225009388964222454285384072231477027482;
        const float c3 = (float)0.486135912065751423025580498947083714508324707;
        const float c4 = (float)2.828427124746190097603377448419396157139343751;
        float l0 = c0 * v[0];
        float l1 = c1 * v[1];
        float l2 = c2 * v[2];
        float l3 = c2 * v[3];
        float e4 = c4 * v[4], f4 = c3 * v[4];
        float e5 = c4 * v[5], f5 = c3 * v[5];
        float e6 = c4 * v[6], f6 = c3 * v[6];
        float e7 = c4 * v[7], f7 = c3 * v[7];
        float p = l0 + l1, m = l0 - l1;
        float q = f5 - f7, r = f4 - f6;
        v[0] = (p + l2) + (e4 - q);
        v[1] = (p + l2) - (e4 + q);
        v[2] = (p - l2) + (r + e5);
        v[3] = (p - l2) + (r - e5);
        v[4] = (m + l3) + (q + e6);
        v[5] = (m + l3) + (q - e6);
        v[6] = (m - l3) - (r - e7);
        v[7] = (m - l3) - (r + e7);
    }
};

template <int T> struct TransformOf;
template <> struct TransformOf<T_DCT> { using type = Dct8; };
template <> struct TransformOf<T_HAAR> { using type = Haar8; };
template <> struct TransformOf<T_WHT> { using type = Wht8; };
template <> struct TransformOf<T_BIOR15> { using type = Bior15; };

}  // namespace zb
