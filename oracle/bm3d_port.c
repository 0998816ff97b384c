/*
 * Test infrastructure only (the oracle). Exported C entry points of the CPU
 * restatement in bm3d_port_impl.h, in an FP32 and an FP64 instantiation.
 * Used by tests/, __graft_entry__.smoke() and bench.py's CPU baseline as the
 * checker; the product never links it.
 *
 * port_bm3d_f32: bit-identical to bm3dcpu (cpu_source/source.cpp) built with an
 *                exact reciprocal, when extractor == 0; with extractor > 0 the
 *                accumulation follows the CUDA kernel's pre-rounding
 *                (source/kernel.cu:740-742).
 * port_bm3d_f64: the same algorithm in double precision (FP64 oracle).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define REAL float
#define SFX _f32
#define RFMA(a, b, c) fmaf((a), (b), (c))
#define RABS(a) fabsf(a)
#define RSQRT(a) sqrtf(a)
#define AGG_DIVIDE(a, b) ((a) * (1.0f / (b)))
#include "bm3d_port_impl.h"
#undef REAL
#undef SFX
#undef RFMA
#undef RABS
#undef RSQRT
#undef AGG_DIVIDE

#define REAL double
#define SFX _f64
#define RFMA(a, b, c) fma((a), (b), (c))
#define RABS(a) fabs(a)
#define RSQRT(a) sqrt(a)
#define AGG_DIVIDE(a, b) ((a) / (b))
#include "bm3d_port_impl.h"
#undef REAL
#undef SFX
#undef RFMA
#undef RABS
#undef RSQRT
#undef AGG_DIVIDE

/* sigma scaling of BM3DCreate (source/source.cpp:520-523,
 * cpu_source/source.cpp:1323-1326), in float as the reference computes it. */
float port_scale_sigma(float sigma_user, int final_) {
    float s = sigma_user;
    s *= (3.f / 4.f) / 255.f * 64.f * (final_ ? 1.0f : 2.7f);
    return s;
}

static int check_args(int width, int height, int stride, int block_step, int bm_range,
                      int radius, int ps_num, int ps_range) {
    if (width < 8 || height < 8 || stride < width) return -1;
    if (block_step < 1 || block_step > 8 || bm_range < 1 || radius < 0) return -1;
    if (ps_num < 1 || ps_num > 8 || ps_range < 1) return -1;
    return 0;
}

/* Number of reference blocks of a plane (cpu_source/source.cpp:787-791). */
int port_num_blocks(int width, int height, int block_step) {
    int nx = 0, ny = 0;
    for (int x = 0; x < width - 8 + block_step; x += block_step) ++nx;
    for (int y = 0; y < height - 8 + block_step; y += block_step) ++ny;
    return nx * ny;
}

int port_bm3d_f32(float *const *acc, float *const *out, const float *const *srcps,
                  const float *const *refps, int width, int height, int stride,
                  const float *sigma_user, int block_step, int bm_range, int radius,
                  int ps_num, int ps_range, int chroma, float extractor,
                  const int *match_in, int *match_out) {
    if (check_args(width, height, stride, block_step, bm_range, radius, ps_num, ps_range))
        return -1;
    float sigma[3];
    for (int p = 0; p < (chroma ? 3 : 1); ++p) sigma[p] = port_scale_sigma(sigma_user[p], refps != NULL);
    return bm3d_window_f32(acc, out, srcps, refps, width, height, stride, sigma, block_step,
                           bm_range, radius, ps_num, ps_range, chroma, extractor, match_in,
                           match_out, 0, 0, 0);
}

/* The run-time-compiled plugin variant (bm3dcuda_rtc): block distance
 * `metric` (0 SSD, 1 SAD, 2 ZSSD, 3 ZSAD, 4 SSD/NORM) and transforms t2d
 * (rows, columns) and t1d (group) (0 DCT, 1 Haar, 2 WHT, 3 bior1.5). */
int port_bm3d_rtc_f32(float *const *acc, float *const *out, const float *const *srcps,
                      const float *const *refps, int width, int height, int stride,
                      const float *sigma_user, int block_step, int bm_range, int radius,
                      int ps_num, int ps_range, int chroma, float extractor, int metric,
                      int t2d, int t1d, const int *match_in, int *match_out) {
    if (check_args(width, height, stride, block_step, bm_range, radius, ps_num, ps_range))
        return -1;
    if (metric < 0 || metric > 4 || t2d < 0 || t2d > 3 || t1d < 0 || t1d > 3) return -1;
    float sigma[3];
    for (int p = 0; p < (chroma ? 3 : 1); ++p) sigma[p] = port_scale_sigma(sigma_user[p], refps != NULL);
    return bm3d_window_f32(acc, out, srcps, refps, width, height, stride, sigma, block_step,
                           bm_range, radius, ps_num, ps_range, chroma, extractor, match_in,
                           match_out, metric, t2d, t1d);
}

int port_bm3d_f64(double *const *acc, double *const *out, const float *const *srcps,
                  const float *const *refps, int width, int height, int stride,
                  const float *sigma_user, int block_step, int bm_range, int radius,
                  int ps_num, int ps_range, int chroma, const int *match_in, int *match_out) {
    if (check_args(width, height, stride, block_step, bm_range, radius, ps_num, ps_range))
        return -1;
    double sigma[3];
    for (int p = 0; p < (chroma ? 3 : 1); ++p)
        sigma[p] = (double)sigma_user[p] * (0.75 / 255.0 * 64.0 * (refps != NULL ? 1.0 : 2.7));
    return bm3d_window_f64(acc, out, srcps, refps, width, height, stride, sigma, block_step,
                           bm_range, radius, ps_num, ps_range, chroma, 0.0, match_in, match_out,
                           0, 0, 0);
}

void port_vaggregate_f32(float *dst, const float *const *vframes, int width, int height,
                         int stride, int radius, int n, int num_frames) {
    vaggregate_f32(dst, vframes, width, height, stride, radius, n, num_frames);
}

void port_vaggregate_f64(double *dst, const double *const *vframes, int width, int height,
                         int stride, int radius, int n, int num_frames) {
    vaggregate_f64(dst, vframes, width, height, stride, radius, n, num_frames);
}

/* 1-D 8-point transforms, exported for known-answer tests (fwd then inv = x16). */
void port_rescore_f32(int *xyz, const float *const *planes, int width, int height, int stride,
                      int block_step, int radius) {
    rescore_f32(xyz, planes, width, height, stride, block_step, radius);
}

void port_dct8_f32(float *v, int forward) {
    if (forward) dct8_fwd_f32(v); else dct8_inv_f32(v);
}
void port_dct8_f64(double *v, int forward) {
    if (forward) dct8_fwd_f64(v); else dct8_inv_f64(v);
}

/* Any of the four 8-point transforms (kind 0 DCT, 1 Haar, 2 WHT, 3 bior1.5). */
void port_tx8_f32(float *v, int kind, int forward) { tx8_f32(v, kind, forward); }
void port_tx8_f64(double *v, int kind, int forward) { tx8_f64(v, kind, forward); }
