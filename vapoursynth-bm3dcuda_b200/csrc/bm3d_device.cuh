// Device building blocks of the BM3D / V-BM3D pipeline for sm_100a.
//
// Every floating-point step that decides a result (block distances, the
// transform, the shrinkage, the group weights) is written with explicit
// round-to-nearest intrinsics (__fadd_rn, __fmul_rn, __fmaf_rn, __fdiv_rn), so
// nvcc cannot contract or reorder it and the values are bit-identical to the
// reference's CPU implementation (cpu_source/source.cpp) built with an exact
// reciprocal. Only the order of the final scatter additions differs (atomics).
#pragma once

#include <cfloat>
#include <cstdint>

namespace bm3d {

// ---------------------------------------------------------------------------
// Packed block coordinates: x (14 bits) | y (14 bits) | z (4 bits, temporal slot)
// ---------------------------------------------------------------------------
constexpr int kCoordBits = 14;
constexpr int kMaxDim = (1 << kCoordBits) - 1;
constexpr int kMaxRadius = 7;

__host__ __device__ __forceinline__ int pack_pos(int x, int y, int z) {
    return x | (y << kCoordBits) | (z << (2 * kCoordBits));
}
__host__ __device__ __forceinline__ int pos_x(int p) { return p & kMaxDim; }
__host__ __device__ __forceinline__ int pos_y(int p) { return (p >> kCoordBits) & kMaxDim; }
__host__ __device__ __forceinline__ int pos_z(int p) { return (unsigned)p >> (2 * kCoordBits); }

// ---------------------------------------------------------------------------
// 8-point scaled DCT-II / DCT-III, FFTW-derived factorisation (FFTW 3.3.9
// e10_8 / e01_8) as the reference uses it (source/kernel.cu:84-176,
// cpu_source/source.cpp:441-536), with the fused multiply-adds placed exactly
// where the reference's CPU code places them. fwd(inv(x)) = 16 x.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void dct8_fwd(float v[8]) {
    const float KP414213562 = 0.414213562373095048801688724209698078569671875f;
    const float KP1_847759065 = 1.847759065022573512256366378793576573644833252f;
    const float KP198912367 = 0.198912367379658006911597622644676228597850501f;
    const float KP1_961570560 = 1.961570560806460898252364472268478073947867462f;
    const float KP1_414213562 = 1.414213562373095048801688724209698078569671875f;
    const float KP668178637 = 0.668178637919298919997757686523080761552472251f;
    const float KP1_662939224 = 1.662939224605090474157576755235811513477121624f;
    const float KP707106781 = 0.707106781186547524400844362104849039284835938f;
    float T3 = __fsub_rn(v[0], v[7]), Tj = __fadd_rn(v[0], v[7]);
    float Te = __fsub_rn(v[4], v[3]), Tk = __fadd_rn(v[4], v[3]);
    float T6 = __fsub_rn(v[2], v[5]);
    float T9 = __fsub_rn(v[1], v[6]);
    float Ta = __fadd_rn(T6, T9), Tn = __fadd_rn(v[1], v[6]);
    float Tf = __fsub_rn(T6, T9), Tm = __fadd_rn(v[2], v[5]);
    float Tb = __fmaf_rn(-KP707106781, Ta, T3);
    float Tg = __fmaf_rn(-KP707106781, Tf, Te);
    float o3 = __fmul_rn(KP1_662939224, __fmaf_rn(KP668178637, Tg, Tb));
    float o5 = -__fmul_rn(KP1_662939224, __fmaf_rn(-KP668178637, Tb, Tg));
    float Tp = __fadd_rn(Tj, Tk), Tq = __fadd_rn(Tm, Tn);
    float o4 = __fmul_rn(KP1_414213562, __fsub_rn(Tp, Tq));
    float o0 = __fmul_rn(KP1_414213562, __fadd_rn(Tp, Tq));
    float Th = __fmaf_rn(KP707106781, Ta, T3);
    float Ti = __fmaf_rn(KP707106781, Tf, Te);
    float o1 = __fmul_rn(KP1_961570560, __fmaf_rn(-KP198912367, Ti, Th));
    float o7 = __fmul_rn(KP1_961570560, __fmaf_rn(KP198912367, Th, Ti));
    float Tl = __fsub_rn(Tj, Tk), To = __fsub_rn(Tm, Tn);
    float o2 = __fmul_rn(KP1_847759065, __fmaf_rn(-KP414213562, To, Tl));
    float o6 = __fmul_rn(KP1_847759065, __fmaf_rn(KP414213562, Tl, To));
    v[0] = o0; v[1] = o1; v[2] = o2; v[3] = o3;
    v[4] = o4; v[5] = o5; v[6] = o6; v[7] = o7;
}

__device__ __forceinline__ void dct8_inv(float v[8]) {
    const float KP1_662939224 = 1.662939224605090474157576755235811513477121624f;
    const float KP668178637 = 0.668178637919298919997757686523080761552472251f;
    const float KP1_961570560 = 1.961570560806460898252364472268478073947867462f;
    const float KP198912367 = 0.198912367379658006911597622644676228597850501f;
    const float KP1_847759065 = 1.847759065022573512256366378793576573644833252f;
    const float KP707106781 = 0.707106781186547524400844362104849039284835938f;
    const float KP414213562 = 0.414213562373095048801688724209698078569671875f;
    const float KP1_414213562 = 1.414213562373095048801688724209698078569671875f;
    float T1 = __fmul_rn(KP1_414213562, v[0]);
    float T3 = __fmaf_rn(KP1_414213562, v[4], T1);
    float Tj = __fmaf_rn(-KP1_414213562, v[4], T1);
    float T6 = __fmaf_rn(KP414213562, v[6], v[2]);
    float Tk = __fmaf_rn(KP414213562, v[2], -v[6]);
    float Tb = __fadd_rn(v[5], v[3]), Te = __fsub_rn(v[3], v[5]);
    float Tc = __fmaf_rn(KP707106781, Tb, v[1]);
    float Tn = __fmaf_rn(-KP707106781, Te, v[7]);
    float Tf = __fmaf_rn(KP707106781, Te, v[7]);
    float Tm = __fmaf_rn(-KP707106781, Tb, v[1]);
    float T7 = __fmaf_rn(KP1_847759065, T6, T3);
    float Tg = __fmaf_rn(KP198912367, Tf, Tc);
    float o7 = __fmaf_rn(-KP1_961570560, Tg, T7);
    float o0 = __fmaf_rn(KP1_961570560, Tg, T7);
    float Tp = __fmaf_rn(-KP1_847759065, Tk, Tj);
    float Tq = __fmaf_rn(KP668178637, Tm, Tn);
    float o5 = __fmaf_rn(-KP1_662939224, Tq, Tp);
    float o2 = __fmaf_rn(KP1_662939224, Tq, Tp);
    float Th = __fmaf_rn(-KP1_847759065, T6, T3);
    float Ti = __fmaf_rn(-KP198912367, Tc, Tf);
    float o3 = __fmaf_rn(-KP1_961570560, Ti, Th);
    float o4 = __fmaf_rn(KP1_961570560, Ti, Th);
    float Tl = __fmaf_rn(KP1_847759065, Tk, Tj);
    float To = __fmaf_rn(-KP668178637, Tn, Tm);
    float o6 = __fmaf_rn(-KP1_662939224, To, Tl);
    float o1 = __fmaf_rn(KP1_662939224, To, Tl);
    v[0] = o0; v[1] = o1; v[2] = o2; v[3] = o3;
    v[4] = o4; v[5] = o5; v[6] = o6; v[7] = o7;
}

// ---------------------------------------------------------------------------
// Transforms of the run-time-compiled plugin variant (bm3dcuda_rtc,
// rtc_source/kernel.hpp:200-380): Haar, Walsh-Hadamard and biorthogonal
// spline 1.5, scaled like the DCT. The coefficients are the reference's; each
// product is rounded on its own and sums run left to right (the same
// sequence as the oracle's restatement). The reference's inverse Haar reads
// only coefficients 0, 1, 2 and 4 (rtc_source/kernel.hpp:226-252), which a
// drop-in reproduces.
// ---------------------------------------------------------------------------
enum TxKind { kTxDct = 0, kTxHaar = 1, kTxWht = 2, kTxBior = 3 };

__device__ __forceinline__ void haar8(float v[8], bool forward) {
    const float S = 1.414213562373095048801688724209698078569671875f;
    const float S2 = __fmul_rn(S, 2.0f);
    if (forward) {
        const float T1 = __fadd_rn(v[0], v[1]), T2 = __fsub_rn(v[0], v[1]);
        const float T3 = __fadd_rn(v[2], v[3]), T4 = __fsub_rn(v[2], v[3]);
        const float T5 = __fadd_rn(v[4], v[5]), T6 = __fsub_rn(v[4], v[5]);
        const float T7 = __fadd_rn(v[6], v[7]), T8 = __fsub_rn(v[6], v[7]);
        const float T9 = __fadd_rn(T1, T3), T10 = __fmul_rn(S, __fsub_rn(T1, T3));
        const float T11 = __fadd_rn(T5, T7), T12 = __fmul_rn(S, __fsub_rn(T5, T7));
        v[0] = __fmul_rn(S, __fadd_rn(T9, T11));
        v[1] = __fmul_rn(S, __fsub_rn(T9, T11));
        v[2] = __fmul_rn(S, T10);
        v[3] = __fmul_rn(S, T12);
        v[4] = __fmul_rn(S2, T2);
        v[5] = __fmul_rn(S2, T4);
        v[6] = __fmul_rn(S2, T6);
        v[7] = __fmul_rn(S2, T8);
    } else {
        const float T1 = __fadd_rn(v[0], v[1]), T2 = __fsub_rn(v[0], v[1]);
        const float a = __fmul_rn(S, v[2]), b = __fmul_rn(2.0f, v[4]);
        const float P = __fadd_rn(a, b), Q = __fsub_rn(a, b);
        const float R = __fadd_rn(-a, b), U = __fsub_rn(-a, b);
        v[0] = __fmul_rn(S, __fadd_rn(T1, P));
        v[1] = __fmul_rn(S, __fadd_rn(T1, Q));
        v[2] = __fmul_rn(S, __fadd_rn(T1, R));
        v[3] = __fmul_rn(S, __fadd_rn(T1, U));
        v[4] = __fmul_rn(S, __fadd_rn(T2, P));
        v[5] = __fmul_rn(S, __fadd_rn(T2, Q));
        v[6] = __fmul_rn(S, __fadd_rn(T2, R));
        v[7] = __fmul_rn(S, __fadd_rn(T2, U));
    }
}

__device__ __forceinline__ void wht8(float v[8]) {
    const float S = 1.414213562373095048801688724209698078569671875f;
    const float T1 = __fadd_rn(v[0], v[1]), T2 = __fsub_rn(v[0], v[1]);
    const float T3 = __fadd_rn(v[2], v[3]), T4 = __fsub_rn(v[2], v[3]);
    const float T5 = __fadd_rn(v[4], v[5]), T6 = __fsub_rn(v[4], v[5]);
    const float T7 = __fadd_rn(v[6], v[7]), T8 = __fsub_rn(v[6], v[7]);
    const float T9 = __fadd_rn(T1, T3), T10 = __fsub_rn(T1, T3);
    const float T11 = __fadd_rn(T2, T4), T12 = __fsub_rn(T2, T4);
    const float T13 = __fadd_rn(T5, T7), T14 = __fsub_rn(T5, T7);
    const float T15 = __fadd_rn(T6, T8), T16 = __fsub_rn(T6, T8);
    v[0] = __fmul_rn(S, __fadd_rn(T9, T13));
    v[1] = __fmul_rn(S, __fsub_rn(T9, T13));
    v[2] = __fmul_rn(S, __fsub_rn(T10, T14));
    v[3] = __fmul_rn(S, __fadd_rn(T10, T14));
    v[4] = __fmul_rn(S, __fadd_rn(T12, T16));
    v[5] = __fmul_rn(S, __fsub_rn(T12, T16));
    v[6] = __fmul_rn(S, __fsub_rn(T11, T15));
    v[7] = __fmul_rn(S, __fadd_rn(T11, T15));
}

__device__ __forceinline__ void bior8(float v[8], bool forward) {
    const float S = 1.414213562373095048801688724209698078569671875f;
    const float C2828 = 2.828427124746190097603377448419396157139343751f;
    if (forward) {
        const float C877 = 0.877670597010003062405456290501163901200537360f;
        const float C1797 = 1.797135031972863413496886690073811797696338403f;
        const float C2277 = 2.277437593371384746027611934034934695963515886f;
        const float C1609 = 1.609389232649111887192845766718020518480884560f;
        const float C334 = 0.334024180361136429417383083658457088741315663f;
        const float T1 = __fadd_rn(v[0], v[3]), T2 = __fsub_rn(v[0], v[3]);
        const float T3 = __fadd_rn(v[1], v[2]), T4 = __fsub_rn(v[1], v[2]);
        const float T5 = __fadd_rn(v[4], v[7]), T6 = __fsub_rn(v[4], v[7]);
        const float T7 = __fadd_rn(v[5], v[6]), T8 = __fsub_rn(v[5], v[6]);
        const float T9 = __fsub_rn(v[0], v[1]), T10 = __fsub_rn(v[2], v[3]);
        const float T11 = __fsub_rn(v[4], v[5]), T12 = __fsub_rn(v[6], v[7]);
        v[0] = __fmul_rn(S, __fadd_rn(__fadd_rn(__fadd_rn(T1, T5), T3), T7));
        v[1] = __fadd_rn(__fmul_rn(C877, __fsub_rn(T1, T5)), __fmul_rn(C1797, __fsub_rn(T3, T7)));
        v[2] = __fadd_rn(__fadd_rn(__fmul_rn(C2277, T2), __fmul_rn(C1609, T4)),
                         __fmul_rn(C334, __fsub_rn(T8, T6)));
        v[3] = __fadd_rn(__fadd_rn(__fmul_rn(C2277, T6), __fmul_rn(C1609, T8)),
                         __fmul_rn(C334, __fsub_rn(T4, T2)));
        v[4] = __fmul_rn(C2828, T9);
        v[5] = __fmul_rn(C2828, T10);
        v[6] = __fmul_rn(C2828, T11);
        v[7] = __fmul_rn(C2828, T12);
    } else {
        const float C1495 = 1.495435764250674860795011090214036706658653686f;
        const float C2058 = 2.058234225009388964222454285384072231477027482f;
        const float C486 = 0.486135912065751423025580498947083714508324707f;
        const float T1 = __fmul_rn(S, v[0]), T2 = __fmul_rn(C1495, v[1]);
        const float T3 = __fmul_rn(C2058, v[2]), T4 = __fmul_rn(C2058, v[3]);
        const float T5 = __fmul_rn(C2828, v[4]), T6 = __fmul_rn(C486, v[4]);
        const float T7 = __fmul_rn(C2828, v[5]), T8 = __fmul_rn(C486, v[5]);
        const float T9 = __fmul_rn(C2828, v[6]), T10 = __fmul_rn(C486, v[6]);
        const float T11 = __fmul_rn(C2828, v[7]), T12 = __fmul_rn(C486, v[7]);
        const float T13 = __fadd_rn(T1, T2), T14 = __fsub_rn(T1, T2);
        const float T15 = __fsub_rn(T8, T12), T16 = __fsub_rn(T6, T10);
        v[0] = __fadd_rn(__fadd_rn(T13, T3), __fsub_rn(T5, T15));
        v[1] = __fsub_rn(__fadd_rn(T13, T3), __fadd_rn(T5, T15));
        v[2] = __fadd_rn(__fsub_rn(T13, T3), __fadd_rn(T16, T7));
        v[3] = __fadd_rn(__fsub_rn(T13, T3), __fsub_rn(T16, T7));
        v[4] = __fadd_rn(__fadd_rn(T14, T4), __fadd_rn(T15, T9));
        v[5] = __fadd_rn(__fadd_rn(T14, T4), __fsub_rn(T15, T9));
        v[6] = __fsub_rn(__fsub_rn(T14, T4), __fsub_rn(T16, T11));
        v[7] = __fsub_rn(__fsub_rn(T14, T4), __fadd_rn(T16, T11));
    }
}

// Any of the four 8-point transforms; `kind` is warp-uniform.
__device__ __forceinline__ void tx8(float v[8], int kind, bool forward) {
    switch (kind) {
        case kTxHaar: haar8(v, forward); break;
        case kTxWht: wht8(v); break;
        case kTxBior: bior8(v, forward); break;
        default:
            if (forward) dct8_fwd(v); else dct8_inv(v);
    }
}

// Device-wide nanosecond clock (for per-clip latency stamps).
__device__ __forceinline__ unsigned long long globaltimer_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---------------------------------------------------------------------------
// Correctly rounded reciprocal for normal a whose reciprocal is normal
// (2^-126 <= |a| < 2^126), without a slow-path call: hardware approximation,
// one Newton-Raphson step, then Markstein's correction y + y * (1 - a * y)
// with the residual formed exactly by an FMA (P. Markstein, "IA-64 and
// Elementary Functions", Prentice Hall 2000, ch. 8). Checked bit-exact against
// the IEEE reciprocal over every float of that range by
// bm3d_b200_selftest_reciprocal.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float rcp_rn_normal(float a) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
    float e = __fmaf_rn(-a, y, 1.0f);
    y = __fmaf_rn(e, y, y);
    e = __fmaf_rn(-a, y, 1.0f);
    return __fmaf_rn(e, y, y);
}

// ---------------------------------------------------------------------------
// Packed FP32x2 arithmetic (sm_100: add/sub/mul/fma.rn.f32x2). Each lane is
// an ordinary IEEE round-to-nearest single-precision operation, so results are
// bit-identical to two scalar operations; one instruction issues both.
// ---------------------------------------------------------------------------
typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pack2(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void unpack2(f32x2 v, float &lo, float &hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

__device__ __forceinline__ f32x2 splat2(float k) { return pack2(k, k); }
__device__ __forceinline__ float lo2(f32x2 v) {
    float a, b;
    unpack2(v, a, b);
    return a;
}
__device__ __forceinline__ float hi2(f32x2 v) {
    float a, b;
    unpack2(v, a, b);
    return b;
}
// The hardware reciprocal approximation that rcp_rn_normal starts from.
__device__ __forceinline__ float rcp_approx(float a) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(a));
    return y;
}
__device__ __forceinline__ f32x2 neg2(f32x2 a) { return a ^ 0x8000000080000000ull; }

// dct8_fwd / dct8_inv on two lines at once: lane 0 of every value is one
// line, lane 1 the other, and each packed instruction is the scalar codelet's
// operation in the same order (bit-identical results, half the instructions).
__device__ __forceinline__ void dct8_fwd2(f32x2 v[8]) {
    const float KP414213562 = 0.414213562373095048801688724209698078569671875f;
    const float KP1_847759065 = 1.847759065022573512256366378793576573644833252f;
    const float KP198912367 = 0.198912367379658006911597622644676228597850501f;
    const float KP1_961570560 = 1.961570560806460898252364472268478073947867462f;
    const float KP1_414213562 = 1.414213562373095048801688724209698078569671875f;
    const float KP668178637 = 0.668178637919298919997757686523080761552472251f;
    const float KP1_662939224 = 1.662939224605090474157576755235811513477121624f;
    const float KP707106781 = 0.707106781186547524400844362104849039284835938f;
    f32x2 T3 = sub2(v[0], v[7]), Tj = add2(v[0], v[7]);
    f32x2 Te = sub2(v[4], v[3]), Tk = add2(v[4], v[3]);
    f32x2 T6 = sub2(v[2], v[5]);
    f32x2 T9 = sub2(v[1], v[6]);
    f32x2 Ta = add2(T6, T9), Tn = add2(v[1], v[6]);
    f32x2 Tf = sub2(T6, T9), Tm = add2(v[2], v[5]);
    f32x2 Tb = fma2(splat2(-KP707106781), Ta, T3);
    f32x2 Tg = fma2(splat2(-KP707106781), Tf, Te);
    f32x2 o3 = mul2(splat2(KP1_662939224), fma2(splat2(KP668178637), Tg, Tb));
    f32x2 o5 = mul2(splat2(-KP1_662939224), fma2(splat2(-KP668178637), Tb, Tg));
    f32x2 Tp = add2(Tj, Tk), Tq = add2(Tm, Tn);
    f32x2 o4 = mul2(splat2(KP1_414213562), sub2(Tp, Tq));
    f32x2 o0 = mul2(splat2(KP1_414213562), add2(Tp, Tq));
    f32x2 Th = fma2(splat2(KP707106781), Ta, T3);
    f32x2 Ti = fma2(splat2(KP707106781), Tf, Te);
    f32x2 o1 = mul2(splat2(KP1_961570560), fma2(splat2(-KP198912367), Ti, Th));
    f32x2 o7 = mul2(splat2(KP1_961570560), fma2(splat2(KP198912367), Th, Ti));
    f32x2 Tl = sub2(Tj, Tk), To = sub2(Tm, Tn);
    f32x2 o2 = mul2(splat2(KP1_847759065), fma2(splat2(-KP414213562), To, Tl));
    f32x2 o6 = mul2(splat2(KP1_847759065), fma2(splat2(KP414213562), Tl, To));
    v[0] = o0; v[1] = o1; v[2] = o2; v[3] = o3;
    v[4] = o4; v[5] = o5; v[6] = o6; v[7] = o7;
}

__device__ __forceinline__ void dct8_inv2(f32x2 v[8]) {
    const float KP1_662939224 = 1.662939224605090474157576755235811513477121624f;
    const float KP668178637 = 0.668178637919298919997757686523080761552472251f;
    const float KP1_961570560 = 1.961570560806460898252364472268478073947867462f;
    const float KP198912367 = 0.198912367379658006911597622644676228597850501f;
    const float KP1_847759065 = 1.847759065022573512256366378793576573644833252f;
    const float KP707106781 = 0.707106781186547524400844362104849039284835938f;
    const float KP414213562 = 0.414213562373095048801688724209698078569671875f;
    const float KP1_414213562 = 1.414213562373095048801688724209698078569671875f;
    f32x2 T1 = mul2(splat2(KP1_414213562), v[0]);
    f32x2 T3 = fma2(splat2(KP1_414213562), v[4], T1);
    f32x2 Tj = fma2(splat2(-KP1_414213562), v[4], T1);
    f32x2 T6 = fma2(splat2(KP414213562), v[6], v[2]);
    f32x2 Tk = fma2(splat2(KP414213562), v[2], neg2(v[6]));
    f32x2 Tb = add2(v[5], v[3]), Te = sub2(v[3], v[5]);
    f32x2 Tc = fma2(splat2(KP707106781), Tb, v[1]);
    f32x2 Tn = fma2(splat2(-KP707106781), Te, v[7]);
    f32x2 Tf = fma2(splat2(KP707106781), Te, v[7]);
    f32x2 Tm = fma2(splat2(-KP707106781), Tb, v[1]);
    f32x2 T7 = fma2(splat2(KP1_847759065), T6, T3);
    f32x2 Tg = fma2(splat2(KP198912367), Tf, Tc);
    f32x2 o7 = fma2(splat2(-KP1_961570560), Tg, T7);
    f32x2 o0 = fma2(splat2(KP1_961570560), Tg, T7);
    f32x2 Tp = fma2(splat2(-KP1_847759065), Tk, Tj);
    f32x2 Tq = fma2(splat2(KP668178637), Tm, Tn);
    f32x2 o5 = fma2(splat2(-KP1_662939224), Tq, Tp);
    f32x2 o2 = fma2(splat2(KP1_662939224), Tq, Tp);
    f32x2 Th = fma2(splat2(-KP1_847759065), T6, T3);
    f32x2 Ti = fma2(splat2(-KP198912367), Tc, Tf);
    f32x2 o3 = fma2(splat2(-KP1_961570560), Ti, Th);
    f32x2 o4 = fma2(splat2(KP1_961570560), Ti, Th);
    f32x2 Tl = fma2(splat2(KP1_847759065), Tk, Tj);
    f32x2 To = fma2(splat2(-KP668178637), Tn, Tm);
    f32x2 o6 = fma2(splat2(-KP1_662939224), To, Tl);
    f32x2 o1 = fma2(splat2(KP1_662939224), To, Tl);
    v[0] = o0; v[1] = o1; v[2] = o2; v[3] = o3;
    v[4] = o4; v[5] = o5; v[6] = o6; v[7] = o7;
}

// ---------------------------------------------------------------------------
// Block distance of K horizontally adjacent candidates.
//
// The reference sums a candidate's squared differences per column in two FMA
// chains (even rows, odd rows), adds the chains, and then adds the 8 column
// sums as ((c0+c1)+(c2+c3))+((c4+c5)+(c6+c7)) (cpu_source/source.cpp:97-136;
// source/kernel.cu:455-471 is the same tree with shuffles). Here one thread
// evaluates the whole 64-term distance for K candidates at once: it walks the
// K+7 pixel columns of the candidate strip, and each loaded column feeds
// column j = m - k of every candidate k that overlaps it, so every pixel
// loaded from shared memory serves up to 8 candidates. Rows 2q and 2q+1 of a
// column travel as one packed pair, so the pair's low lane is the even-row
// chain and its high lane the odd-row chain: 8 packed instructions per column
// instead of 16. The column sums are folded into the tree in column order
// (A: c0..c3, B: c2..c7, C: c6..c7).
//
// refp[q][j] = (ref[2q][j], ref[2q+1][j]); row[r] are shared-memory word
// offsets of the strip's 8 pixel rows at the strip's first column.
// ---------------------------------------------------------------------------
template <int K>
__device__ __forceinline__ void ssd_strip(const f32x2 (&refp)[4][8], const float *tile,
                                          const int (&row)[8], float (&err)[K]) {
    float A[K], B[K], C[K];
#pragma unroll
    for (int m = 0; m < K + 7; ++m) {
        f32x2 px[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) px[q] = pack2(tile[row[2 * q] + m], tile[row[2 * q + 1] + m]);
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int j = m - k;
            if (j >= 0 && j < 8) {
                f32x2 d = sub2(refp[0][j], px[0]);
                f32x2 e = mul2(d, d);
                d = sub2(refp[1][j], px[1]);
                e = fma2(d, d, e);
                d = sub2(refp[2][j], px[2]);
                e = fma2(d, d, e);
                d = sub2(refp[3][j], px[3]);
                e = fma2(d, d, e);
                float e0, e1;
                unpack2(e, e0, e1);
                const float c = __fadd_rn(e0, e1);
                if (j == 0) {
                    A[k] = c;
                } else if (j == 1) {
                    A[k] = __fadd_rn(A[k], c);
                } else if (j == 2) {
                    B[k] = c;
                } else if (j == 3) {
                    B[k] = __fadd_rn(B[k], c);
                    A[k] = __fadd_rn(A[k], B[k]);
                } else if (j == 4) {
                    B[k] = c;
                } else if (j == 5) {
                    B[k] = __fadd_rn(B[k], c);
                } else if (j == 6) {
                    C[k] = c;
                } else {
                    C[k] = __fadd_rn(C[k], c);
                    B[k] = __fadd_rn(B[k], C[k]);
                    err[k] = __fadd_rn(A[k], B[k]);
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Sorted 8-entry match list with the reference's insertion rule
// (source/kernel.cu:473-485, cpu_source/source.cpp:179-204): a candidate goes
// in front of every entry whose error is strictly larger, so among equal
// errors the earlier-scanned candidate stays first. Callers feed candidates
// in the reference's scan order, which makes the result identical.
// ---------------------------------------------------------------------------
struct List8 {
    float e[8];
    int p[8];
};

__device__ __forceinline__ void list_init(List8 &l, float e, int p) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        l.e[i] = e;
        l.p[i] = p;
    }
}

__device__ __forceinline__ void list_insert(List8 &l, float err, int pos) {
#pragma unroll
    for (int i = 7; i > 0; --i) {
        const bool shift = err < l.e[i - 1];
        const bool here = !shift && err < l.e[i];
        l.e[i] = shift ? l.e[i - 1] : (here ? err : l.e[i]);
        l.p[i] = shift ? l.p[i - 1] : (here ? pos : l.p[i]);
    }
    if (err < l.e[0]) {
        l.e[0] = err;
        l.p[0] = pos;
    }
}

// Register-array element at a runtime index without local-memory indexing.
template <int N, typename T>
__device__ __forceinline__ T pick(const T (&a)[N], int i) {
    T v = a[0];
#pragma unroll
    for (int k = 1; k < N; ++k) v = (i == k) ? a[k] : v;
    return v;
}

// ---------------------------------------------------------------------------
// Shared-memory pixel tiles of the block matchers: rows skewed by
// (row / 8) mod 8 words, which makes the 32 threads of a warp (4 x 8
// reference blocks, block_step 8) hit 32 distinct banks.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int skewed(int ty, int tx, int pitch) {
    return ty * pitch + ((ty >> 3) & 7) + tx;
}

// Stage the pixel rectangle [y0, y0+th) x [x0, x0+tw) of `plane` into the
// tile; pixels outside the image read as 0 (they are never ranked). Every
// word is an asynchronous global->shared copy (cp.async), so all of a
// thread's copies are in flight together; the thread waits for its own copies
// before returning, and the caller's barrier publishes the tile. A warp copies
// one row at a time: rows that lie inside the image copy four words per lane
// and iteration with immediate offsets; border rows check every word
// (zero-filled when outside the image, then from the plane's first word).
__device__ __forceinline__ void load_tile(float *tile, const float *__restrict__ plane, int width,
                                          int height, int stride, int x0, int y0, int tw, int th,
                                          int pitch) {
    const int nwarps = blockDim.x >> 5;
    const int lane = threadIdx.x & 31;
    const bool cols_inside = x0 >= 0 && x0 + tw <= width;
    for (int ty = threadIdx.x >> 5; ty < th; ty += nwarps) {
        const int gy = y0 + ty;
        const bool row_ok = gy >= 0 && gy < height;
        const float *src = plane + (size_t)(row_ok ? gy : 0) * stride;
        const unsigned dst =
            (unsigned)__cvta_generic_to_shared(tile + ty * pitch + ((ty >> 3) & 7));
        if (row_ok && cols_inside) {
            const float *s = src + x0 + lane;
            unsigned d = dst + 4u * lane;
            int tx = lane;
            for (; tx + 96 < tw; tx += 128, s += 128, d += 512u)
                asm volatile(
                    "cp.async.ca.shared.global [%0], [%1], 4;\n\t"
                    "cp.async.ca.shared.global [%0+128], [%1+128], 4;\n\t"
                    "cp.async.ca.shared.global [%0+256], [%1+256], 4;\n\t"
                    "cp.async.ca.shared.global [%0+384], [%1+384], 4;" ::"r"(d),
                    "l"(s)
                    : "memory");
            for (; tx < tw; tx += 32, s += 32, d += 128u)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(s) : "memory");
        } else {
            for (int tx = lane; tx < tw; tx += 32) {
                const int gx = x0 + tx;
                const bool ok = row_ok && gx >= 0 && gx < width;
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst + 4u * tx),
                             "l"(ok ? src + gx : plane), "r"(ok ? 4 : 0)
                             : "memory");
            }
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Block distances of the run-time-compiled plugin variant
// (rtc_source/kernel.hpp:392-504): 1 SAD, 2 ZSSD, 3 ZSAD, 4 SSD/NORM (0 is
// the SSD of ssd_strip). Column c of the block plays the reference's lane:
// per column two accumulators over even and odd rows, then the butterfly
// across columns; means are the butterfly of the per-column pairwise sums
// times 1/64.
// ---------------------------------------------------------------------------
struct RefStats {
    float mean;  // zero-mean distances: mean of the reference block
    float norm;  // SSD/NORM: l2 norm of the reference block
};

__device__ __forceinline__ float tree8(const float (&c)[8]) {
    return __fadd_rn(__fadd_rn(__fadd_rn(c[0], c[1]), __fadd_rn(c[2], c[3])),
                     __fadd_rn(__fadd_rn(c[4], c[5]), __fadd_rn(c[6], c[7])));
}

// Column c of the reference block, rows 0..7 (refp holds row pairs packed).
__device__ __forceinline__ void ref_column(const f32x2 (&refp)[4][8], int c, float (&a)[8]) {
#pragma unroll
    for (int q = 0; q < 4; ++q) unpack2(refp[q][c], a[2 * q], a[2 * q + 1]);
}

template <int M>
__device__ __forceinline__ RefStats ref_stats(const f32x2 (&refp)[4][8]) {
    RefStats rs{0.0f, 0.0f};
    float col[8];
    if (M == 2 || M == 3) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float a[8];
            ref_column(refp, c, a);
            col[c] = tree8(a);
        }
        rs.mean = __fmul_rn(tree8(col), 1.0f / 64.0f);
    } else if (M == 4) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float a[8];
            ref_column(refp, c, a);
            float e0 = 0.0f, e1 = 0.0f;
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                e0 = __fmaf_rn(a[r], a[r], e0);
                e1 = __fmaf_rn(a[r + 1], a[r + 1], e1);
            }
            col[c] = __fadd_rn(e0, e1);
        }
        rs.norm = __fsqrt_rn(tree8(col));
    }
    return rs;
}

// Distance of the reference block to the candidate whose row r starts at
// tile[row[r] + off].
template <int M>
__device__ __forceinline__ float metric_dist(const f32x2 (&refp)[4][8], const RefStats &rs,
                                             const float *tile, const int (&row)[8], int off) {
    float col[8];
    if (M == 1) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float a[8];
            ref_column(refp, c, a);
            float e0 = 0.0f, e1 = 0.0f;
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                e0 = __fadd_rn(e0, fabsf(__fsub_rn(a[r], tile[row[r] + off + c])));
                e1 = __fadd_rn(e1, fabsf(__fsub_rn(a[r + 1], tile[row[r + 1] + off + c])));
            }
            col[c] = __fadd_rn(e0, e1);
        }
        return tree8(col);
    } else if (M == 2 || M == 3) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float n[8];
#pragma unroll
            for (int r = 0; r < 8; ++r) n[r] = tile[row[r] + off + c];
            col[c] = tree8(n);
        }
        const float dm = __fsub_rn(rs.mean, __fmul_rn(tree8(col), 1.0f / 64.0f));
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float a[8];
            ref_column(refp, c, a);
            float e0 = 0.0f, e1 = 0.0f;
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const float d0 = __fsub_rn(__fsub_rn(a[r], tile[row[r] + off + c]), dm);
                const float d1 = __fsub_rn(__fsub_rn(a[r + 1], tile[row[r + 1] + off + c]), dm);
                if (M == 2) {
                    e0 = __fmaf_rn(d0, d0, e0);
                    e1 = __fmaf_rn(d1, d1, e1);
                } else {
                    e0 = __fadd_rn(e0, fabsf(d0));
                    e1 = __fadd_rn(e1, fabsf(d1));
                }
            }
            col[c] = __fadd_rn(e0, e1);
        }
        return tree8(col);
    } else {
        float nn[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            float a[8];
            ref_column(refp, c, a);
            float b0 = 0.0f, b1 = 0.0f, d0 = 0.0f, d1 = 0.0f;
#pragma unroll
            for (int r = 0; r < 8; r += 2) {
                const float n0 = tile[row[r] + off + c], n1 = tile[row[r + 1] + off + c];
                b0 = __fmaf_rn(n0, n0, b0);
                b1 = __fmaf_rn(n1, n1, b1);
                d0 = __fmaf_rn(a[r], n0, d0);
                d1 = __fmaf_rn(a[r + 1], n1, d1);
            }
            nn[c] = __fadd_rn(b0, b1);
            col[c] = __fadd_rn(d0, d1);
        }
        const float den = __fmaf_rn(rs.norm, __fsqrt_rn(tree8(nn)), FLT_EPSILON);
        return __fsub_rn(2.0f, __fdiv_rn(__fmul_rn(2.0f, tree8(col)), den));
    }
}

}  // namespace bm3d
