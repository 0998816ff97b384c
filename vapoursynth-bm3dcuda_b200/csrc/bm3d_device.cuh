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
// word is an asynchronous global->shared copy (cp.async, zero-filled when
// outside the image, then from the plane's first word), so all of a thread's
// copies are in flight together; the thread waits for its own copies before
// returning, and the caller's barrier publishes the tile.
__device__ __forceinline__ void load_tile(float *tile, const float *__restrict__ plane, int width,
                                          int height, int stride, int x0, int y0, int tw, int th,
                                          int pitch) {
    const int nwarps = blockDim.x >> 5;
    for (int ty = threadIdx.x >> 5; ty < th; ty += nwarps) {
        const int gy = y0 + ty;
        const bool row_ok = gy >= 0 && gy < height;
        const float *src = plane + (size_t)(row_ok ? gy : 0) * stride;
        const unsigned dst =
            (unsigned)__cvta_generic_to_shared(tile + ty * pitch + ((ty >> 3) & 7));
        for (int tx = threadIdx.x & 31; tx < tw; tx += 32) {
            const int gx = x0 + tx;
            const bool ok = row_ok && gx >= 0 && gx < width;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst + 4u * tx),
                         "l"(ok ? src + gx : plane), "r"(ok ? 4 : 0)
                         : "memory");
        }
    }
    asm volatile("cp.async.wait_all;" ::: "memory");
}

}  // namespace bm3d
