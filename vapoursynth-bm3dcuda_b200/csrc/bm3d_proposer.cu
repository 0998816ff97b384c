// Learned match proposal for BM3D / V-BM3D on sm_100a (no counterpart in the
// reference).
//
// A small CNN - three 3x3 convolutions, 1 -> 16 -> 16 -> 16 channels, ReLU
// after the first two, zero padding - maps the 2x-downsampled plane to a
// 16-channel embedding per half-resolution pixel. A full-resolution block
// origin (u, v) belongs to the cell (u/2, v/2), and a cell's embedding is the
// network output at half-resolution pixel (u/2 + 2, v/2 + 2), the middle of
// the block's 4x4 half-resolution footprint. The learned block matcher
// (bm3d_learned.cu) ranks candidate cells by squared embedding distance to
// the reference block's own cell and scores only the best cells exactly.
//
// Two implementations of the network live here:
//   * training: FP32 forward / backward kernels over a batch of frames, the
//     listwise proposal loss and Adam, all written for this project;
//   * inference: one fused kernel per frame tile, the three layers on the
//     5th-generation tensor cores (tcgen05.mma with M = 128, N = 16, BF16
//     operands from shared memory, FP32 accumulators in tensor memory)
//     with the activations held in shared memory, writing 8-bit embeddings
//     (16 bytes per cell; one scale and 16 offsets calibrated on the
//     embeddings of sample frames, see calibrate()).
//
// Parameters: one FP32 vector of 4800 values, w1 [3][3][1][16], b1 [16],
// w2 [3][3][16][16], b2 [16], w3 [3][3][16][16], b3 [16]; w[dy][dx][ci][co]
// multiplies input pixel (y + dy - 1, x + dx - 1).
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <new>
#include <vector>

#include "bm3d_b200.h"
#include "bm3d_device.cuh"
#include "bm3d_internal.h"
#include "bm3d_umma.cuh"

namespace bm3d {

int abi_fail(int code, const char *msg);

constexpr int kCh = 16;
constexpr int kOffW1 = 0, kOffB1 = 144, kOffW2 = 160, kOffB2 = 2464, kOffW3 = 2480,
              kOffB3 = 4784;
static_assert(kOffB3 + kCh == BM3D_B200_PROPOSER_PARAMS, "parameter layout");

namespace {

// ===========================================================================
// training kernels (FP32)
// ===========================================================================

// 2x2 mean of each frame [height][stride] -> [h2][w2].
__global__ void downsample2_kernel(const float *__restrict__ src, long long frame_floats,
                                   int stride, int w2, int h2, float *__restrict__ dst) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int f = blockIdx.z;
    if (x >= w2) return;
    const float *s = src + f * frame_floats + (size_t)(2 * y) * stride + 2 * x;
    dst[((size_t)f * h2 + y) * w2 + x] = 0.25f * ((s[0] + s[1]) + (s[stride] + s[stride + 1]));
}

// out[f][y][x][co] = b[co] + sum in[f][y+dy-1][x+dx-1][ci] * w[dy][dx][ci][co]
template <int CIN, int COUT>
__global__ void conv3x3_fwd_kernel(const float *__restrict__ in, const float *__restrict__ w,
                                   const float *__restrict__ b, float *__restrict__ out,
                                   int width, int height, int nframes, int relu) {
    __shared__ float ws[9 * CIN * COUT + COUT];
    for (int i = threadIdx.x; i < 9 * CIN * COUT; i += blockDim.x) ws[i] = w[i];
    for (int i = threadIdx.x; i < COUT; i += blockDim.x) ws[9 * CIN * COUT + i] = b[i];
    __syncthreads();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long npix = (long long)width * height;
    if (idx >= npix * nframes) return;
    const int f = (int)(idx / npix);
    const int pix = (int)(idx % npix);
    const int x = pix % width, y = pix / width;
    const float *fin = in + (size_t)f * npix * CIN;
    float acc[COUT];
#pragma unroll
    for (int c = 0; c < COUT; ++c) acc[c] = ws[9 * CIN * COUT + c];
#pragma unroll
    for (int dy = 0; dy < 3; ++dy) {
        const int yy = y + dy - 1;
        if (yy < 0 || yy >= height) continue;
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
            const int xx = x + dx - 1;
            if (xx < 0 || xx >= width) continue;
            const float *pin = fin + ((size_t)yy * width + xx) * CIN;
            const float *pw = ws + (dy * 3 + dx) * CIN * COUT;
#pragma unroll
            for (int ci = 0; ci < CIN; ++ci) {
                const float v = pin[ci];
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] = fmaf(v, pw[ci * COUT + c], acc[c]);
            }
        }
    }
    float *po = out + (size_t)idx * COUT;
#pragma unroll
    for (int c = 0; c < COUT; ++c) po[c] = relu ? fmaxf(acc[c], 0.0f) : acc[c];
}

// Input gradient of conv3x3 (+ ReLU applied to `out`, when relu):
//   g = dout * (out > 0);  din[y][x][ci] = sum g[y-dy+1][x-dx+1][co] * w[dy][dx][ci][co]
template <int CIN, int COUT>
__global__ void conv3x3_bwd_data_kernel(const float *__restrict__ dout,
                                        const float *__restrict__ out,
                                        const float *__restrict__ w, float *__restrict__ din,
                                        int width, int height, int nframes, int relu) {
    __shared__ float ws[9 * CIN * COUT];
    for (int i = threadIdx.x; i < 9 * CIN * COUT; i += blockDim.x) ws[i] = w[i];
    __syncthreads();
    const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long npix = (long long)width * height;
    if (idx >= npix * nframes) return;
    const int f = (int)(idx / npix);
    const int pix = (int)(idx % npix);
    const int x = pix % width, y = pix / width;
    const size_t fo = (size_t)f * npix * COUT;
    float acc[CIN];
#pragma unroll
    for (int ci = 0; ci < CIN; ++ci) acc[ci] = 0.0f;
#pragma unroll
    for (int dy = 0; dy < 3; ++dy) {
        const int yy = y - dy + 1;
        if (yy < 0 || yy >= height) continue;
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
            const int xx = x - dx + 1;
            if (xx < 0 || xx >= width) continue;
            const size_t o = fo + ((size_t)yy * width + xx) * COUT;
            const float *pw = ws + (dy * 3 + dx) * CIN * COUT;
#pragma unroll
            for (int c = 0; c < COUT; ++c) {
                float g = dout[o + c];
                if (relu && !(out[o + c] > 0.0f)) g = 0.0f;
#pragma unroll
                for (int ci = 0; ci < CIN; ++ci) acc[ci] = fmaf(g, pw[ci * COUT + c], acc[ci]);
            }
        }
    }
#pragma unroll
    for (int ci = 0; ci < CIN; ++ci) din[(size_t)idx * CIN + ci] = acc[ci];
}

// Weight gradient: dw[dy][dx][ci][co] += sum in[y+dy-1][x+dx-1][ci] * g[y][x][co],
// db[co] += sum g. One CTA row per (tap, ci); the CTAs of a row stride over
// all pixels of all frames, reduce, and add one atomic per weight.
template <int CIN, int COUT>
__global__ void conv3x3_bwd_weight_kernel(const float *__restrict__ in,
                                          const float *__restrict__ dout,
                                          const float *__restrict__ out, float *__restrict__ dw,
                                          float *__restrict__ db, int width, int height,
                                          int nframes, int relu) {
    const int tap = blockIdx.x / CIN, ci = blockIdx.x % CIN;
    const int dy = tap / 3, dx = tap % 3;
    const bool do_bias = tap == 0 && ci == 0;
    const long long npix = (long long)width * height;
    float acc[COUT], accb[COUT];
#pragma unroll
    for (int c = 0; c < COUT; ++c) acc[c] = accb[c] = 0.0f;
    for (long long idx = (long long)blockIdx.y * blockDim.x + threadIdx.x; idx < npix * nframes;
         idx += (long long)gridDim.y * blockDim.x) {
        const int f = (int)(idx / npix);
        const int pix = (int)(idx % npix);
        const int x = pix % width, y = pix / width;
        const int yy = y + dy - 1, xx = x + dx - 1;
        const bool inside = yy >= 0 && yy < height && xx >= 0 && xx < width;
        const float v =
            inside ? in[((size_t)f * npix + (size_t)yy * width + xx) * CIN + ci] : 0.0f;
        const size_t o = (size_t)idx * COUT;
#pragma unroll
        for (int c = 0; c < COUT; ++c) {
            float g = dout[o + c];
            if (relu && !(out[o + c] > 0.0f)) g = 0.0f;
            acc[c] = fmaf(v, g, acc[c]);
            accb[c] += g;
        }
    }
    __shared__ float red[COUT][2][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c < COUT; ++c) {
        float s = acc[c], sb = accb[c];
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            sb += __shfl_xor_sync(0xffffffffu, sb, o);
        }
        if (lane == 0) {
            red[c][0][warp] = s;
            red[c][1][warp] = sb;
        }
    }
    __syncthreads();
    if (threadIdx.x < COUT) {
        const int c = threadIdx.x;
        float s = 0.0f, sb = 0.0f;
        for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) {
            s += red[c][0][wi];
            sb += red[c][1][wi];
        }
        atomicAdd(dw + ((size_t)tap * CIN + ci) * COUT + c, s);
        if (do_bias) atomicAdd(db + c, sb);
    }
}

// Teacher distances of the training samples: for sample (fc, fz, x, y) and
// each candidate cell (x/2 + u, y/2 + v), |u|, |v| <= U, of frame fz, the
// smallest exact block distance (sum of squared differences) between the
// reference block at (x, y) of frame fc and the cell's block origins in the
// plane - the distances the exhaustive search ranks. +inf for cells without
// an origin in the plane and for samples outside the frames or the plane.
// One warp per sample, lanes over cells.
__global__ void teacher_kernel(const float *__restrict__ frames, long long frame_floats,
                               int stride, const int4 *__restrict__ samples, int nsamples,
                               int nframes, int width, int height, int U,
                               float *__restrict__ teacher) {
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (b >= nsamples) return;
    const int4 smp = samples[b];
    const int x = smp.z, y = smp.w;
    const int side = 2 * U + 1, ncand = side * side;
    float *out = teacher + (size_t)b * ncand;
    const bool ok = smp.x >= 0 && smp.x < nframes && smp.y >= 0 && smp.y < nframes && x >= 0 &&
                    y >= 0 && x <= width - 8 && y <= height - 8;
    const float *rf = frames + smp.x * frame_floats + (size_t)y * stride + x;
    const float *cf = frames + smp.y * frame_floats;
    for (int c = lane; c < ncand; c += 32) {
        float best = INFINITY;
        if (ok) {
            const int gx = (x >> 1) + c % side - U, gy = (y >> 1) + c / side - U;
            for (int dv = 0; dv < 2; ++dv)
                for (int du = 0; du < 2; ++du) {
                    const int u = 2 * gx + du, v = 2 * gy + dv;
                    if (u < 0 || v < 0 || u > width - 8 || v > height - 8) continue;
                    const float *q = cf + (size_t)v * stride + u;
                    float e = 0.0f;
                    for (int r = 0; r < 8; ++r)
                        for (int k = 0; k < 8; ++k) {
                            const float d = rf[r * stride + k] - q[r * stride + k];
                            e = fmaf(d, d, e);
                        }
                    best = fminf(best, e);
                }
        }
        out[c] = best;
    }
}

// Distillation loss, one warp per sample: the student's distribution over
// the sample's candidate cells is p = softmax(-d), d the squared embedding
// distance to the reference cell's embedding (frame fc); the teacher's is
// q = softmax(-(s - min s) / T) over the teacher distances s (cells with
// s = +inf excluded). loss = (1/n) sum over samples of KL(q || p);
// d loss / d d_c = (q_c - p_c) / n. Adds the loss to *loss and its gradient
// to demb (both zeroed before).
__global__ void proposal_loss_kernel(const float *__restrict__ emb, int w2, int h2,
                                     const int4 *__restrict__ samples,
                                     const float *__restrict__ teacher, int nsamples,
                                     int nframes, int width, int height, int U, float inv_t,
                                     float inv_n, float *__restrict__ demb,
                                     float *__restrict__ loss) {
    const int lane = threadIdx.x & 31;
    const int b = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (b >= nsamples) return;
    const int4 smp = samples[b];
    const int x = smp.z, y = smp.w;
    // samples outside the frames or the plane carry no signal (and are not read)
    if (smp.x < 0 || smp.x >= nframes || smp.y < 0 || smp.y >= nframes || x < 0 || y < 0 ||
        x > width - 8 || y > height - 8)
        return;
    const int cx = x / 2, cy = y / 2;
    const size_t fstride = (size_t)w2 * h2 * kCh;
    const float *ec_base = emb + (size_t)smp.y * fstride;
    float *gc_base = demb + (size_t)smp.y * fstride;
    const int side = 2 * U + 1, ncand = side * side;
    const float *ts = teacher + (size_t)b * ncand;
    float er[kCh];
    const size_t ro = (size_t)smp.x * fstride + ((size_t)(cy + 2) * w2 + (cx + 2)) * kCh;
#pragma unroll
    for (int k = 0; k < kCh; ++k) er[k] = emb[ro + k];
    auto cell = [&](int c) {
        return ((size_t)(cy + c / side - U + 2) * w2 + (cx + c % side - U + 2)) * kCh;
    };
    auto dist = [&](size_t oc) {
        float d = 0.0f;
#pragma unroll
        for (int k = 0; k < kCh; ++k) {
            const float t = er[k] - ec_base[oc + k];
            d = fmaf(t, t, d);
        }
        return d;
    };
    float mx = -FLT_MAX, smin = INFINITY;
    for (int c = lane; c < ncand; c += 32) {
        const float sc = ts[c];
        if (!(sc < INFINITY)) continue;
        mx = fmaxf(mx, -dist(cell(c)));
        smin = fminf(smin, sc);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        smin = fminf(smin, __shfl_xor_sync(0xffffffffu, smin, o));
    }
    if (!(smin < INFINITY)) return;  // no candidate cell: no signal
    float sa = 0.0f, sq = 0.0f, sqd = 0.0f, sqs = 0.0f;
    for (int c = lane; c < ncand; c += 32) {
        const float sc = ts[c];
        if (!(sc < INFINITY)) continue;
        const float d = dist(cell(c));
        const float z = (sc - smin) * inv_t;
        const float w = expf(-z);
        sa += expf(-d - mx);
        sq += w;
        sqd += w * d;
        sqs += w * z;
    }
    for (int o = 16; o > 0; o >>= 1) {
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sq += __shfl_xor_sync(0xffffffffu, sq, o);
        sqd += __shfl_xor_sync(0xffffffffu, sqd, o);
        sqs += __shfl_xor_sync(0xffffffffu, sqs, o);
    }
    // KL = sum q d + logsumexp(-d) + sum q log q,  sum q log q = -sqs/sq - log sq
    if (lane == 0) atomicAdd(loss, (sqd / sq + mx + logf(sa) - sqs / sq - logf(sq)) * inv_n);
    float gr[kCh];
#pragma unroll
    for (int k = 0; k < kCh; ++k) gr[k] = 0.0f;
    for (int c = lane; c < ncand; c += 32) {
        const float sc = ts[c];
        if (!(sc < INFINITY)) continue;
        const size_t oc = cell(c);
        float t[kCh], d = 0.0f;
#pragma unroll
        for (int k = 0; k < kCh; ++k) {
            t[k] = er[k] - ec_base[oc + k];
            d = fmaf(t[k], t[k], d);
        }
        const float pc = expf(-d - mx) / sa;
        const float qc = expf(-(sc - smin) * inv_t) / sq;
        const float gd = (qc - pc) * inv_n;  // d loss / d distance
#pragma unroll
        for (int k = 0; k < kCh; ++k) {
            const float g = 2.0f * gd * t[k];  // d d / d er = 2 t, d d / d ec = -2 t
            gr[k] += g;
            atomicAdd(gc_base + oc + k, -g);
        }
    }
#pragma unroll
    for (int k = 0; k < kCh; ++k) {
        float g = gr[k];
        for (int o = 16; o > 0; o >>= 1) g += __shfl_xor_sync(0xffffffffu, g, o);
        if (lane == 0) atomicAdd(demb + ro + k, g);
    }
}

// Counts the samples that enter the loss (the loss's n): inside the frames
// and the plane, with at least one candidate cell.
__global__ void count_samples_kernel(const int4 *__restrict__ samples,
                                     const float *__restrict__ teacher, int nsamples,
                                     int nframes, int width, int height, int U,
                                     int *__restrict__ count) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nsamples) return;
    const int4 s = samples[i];
    if (s.x < 0 || s.x >= nframes || s.y < 0 || s.y >= nframes || s.z < 0 || s.w < 0 ||
        s.z > width - 8 || s.w > height - 8)
        return;
    const int ncand = (2 * U + 1) * (2 * U + 1);
    bool any = false;
    for (int c = 0; c < ncand && !any; ++c) any = teacher[(size_t)i * ncand + c] < INFINITY;
    if (any) atomicAdd(count, 1);
}

// Adam (Kingma & Ba 2015) with the bias corrections of step *step.
__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, int n, float lr,
                            const int *__restrict__ step) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float b1 = 0.9f, b2 = 0.999f;
    const float t = (float)*step;
    const float c1 = 1.0f - powf(b1, t), c2 = 1.0f - powf(b2, t);
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + 1e-8f);
}

__global__ void step_kernel(int *step) { *step += 1; }

// ===========================================================================
// inference helpers
// ===========================================================================

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

// BF16 pair of max(lo, 0), max(hi, 0), rounded to nearest (lo in the low half)
__device__ __forceinline__ uint32_t bf16x2_relu(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}

// FP32 biases [3][16] of the inference kernel (the quantisation follows them).
__global__ void pack_bias_kernel(const float *__restrict__ prm, float *__restrict__ bias) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 48) bias[i] = prm[(i < 16 ? kOffB1 : i < 32 ? kOffB2 : kOffB3) + (i & 15)];
}

// Embedding quantisation to 8 bits: v * qs + qo (one rounding), rounded to
// the nearest integer (ties to even) and saturated to [0, 255].
__device__ __forceinline__ uint32_t quantize_u8(float v, float qs, float qo) {
    uint32_t r;
    asm("cvt.rni.sat.u8.f32 %0, %1;" : "=r"(r) : "f"(__fmaf_rn(v, qs, qo)));
    return r;
}

// ===========================================================================
// inference on the 5th-generation tensor cores (tcgen05, accumulators in TMEM)
// ===========================================================================
//
// Same network as the training kernels, with the layers as tcgen05.mma
// (kind::f16, BF16 operands from shared memory, FP32 accumulators in tensor
// memory):
//   * a CTA computes kUTY x kUTX outputs of one frame with flat pitch kUP =
//     128, so one M = 128 MMA covers one row of a layer's region and a 3x3 tap
//     (dy, dx) of output index f reads input index f + dy*kUP + dx: the A
//     operand of a tap is the activation array shifted by that many pixels,
//     i.e. the same matrix descriptor with another start address (no im2col);
//   * BF16 activations are kept as two planes of 16 bytes per pixel
//     (channels 0-7, channels 8-15), which is the canonical K-major layout
//     without swizzle: core matrices of 8 pixels x 16 bytes, 8-pixel groups
//     128 bytes apart (SBO), the two channel halves one plane apart (LBO);
//   * weights: per tap a 16 x 16 operand (N = output channels, K = input
//     channels) in the same canonical layout, 512 bytes;
//   * layer 1 (one input channel) multiplies a 9-tap row per pixel (padded
//     to K = 16) built in the activation buffer;
//   * the layers run as a pipeline of 128-pixel chunks (one row each): one
//     thread of the last warp issues the MMAs (a chunk accumulates its 9
//     taps in one of 8 slots of 16 TMEM columns, taken in issue order) and
//     commits each chunk to its own mbarrier; eight epilogue warps (two warpgroups, alternate chunks;
//     warp w reads TMEM lanes 32(w%4) .. +31) take each finished chunk, add
//     the bias, apply ReLU and the zero padding, write the next layer's BF16
//     activations into the same buffer and arrive on that row's "written"
//     barrier; the next layer's chunk c is issued once rows c .. c+3 of its
//     input are written, so the tensor core works on one layer while the
//     epilogue warps drain the previous one. The last layer quantises to 8
//     bits straight to global memory.
//     In-place reuse is safe because an epilogue overwrites row c only after
//     every MMA reading row c has completed (a commit covers all earlier
//     MMAs, later chunks read rows above c), and a TMEM slot is reused only
//     after the epilogue of the chunk that last used it has read it back.
//     With 9 output rows per CTA (71.8 KB of shared memory, 128 TMEM
//     columns) three CTAs share an SM.
// Columns past a layer's valid width are computed but feed no valid output.
// Every wait on the mbarrier is bounded in time: on expiry the CTA records
// an error in *err, releases its tensor memory and returns.
constexpr int kUP = 128;                        // flat pitch (pixels)
constexpr int kUTY = 9;                         // output rows per CTA
constexpr int kUTX = kUP - 6;                   // 122 output columns per CTA
constexpr int kUC1 = 13, kUC2 = 11, kUC3 = 9;   // 128-pixel chunks of layers 1, 2, 3
constexpr int kUN1 = kUC1 * 128;                // layer-1 outputs (rows oy-2 .. oy+10)
constexpr int kUN3 = kUC3 * 128;                // layer-3 outputs (rows oy .. oy+8)
constexpr int kUAct = kUN1 + 8;                 // pixels per activation plane
constexpr int kUX0 = (kUTY + 6) * kUP + 8;      // input floats (rows oy-3 .. oy+11)
constexpr int kUTiles = 19;                     // weight operands: layer 1, 9 + 9 taps
constexpr int kUTileBytes = 512;
constexpr uint32_t kUmmaWords = kUTiles * kUTileBytes / 4;
constexpr size_t kUActBytes = (size_t)2 * kUAct * 16;
constexpr int kUBars = 2 * (kUC1 + kUC2 + kUC3);  // per-chunk mbarriers
constexpr size_t kUEmbedSmem = kUActBytes + (size_t)kUTiles * kUTileBytes + (size_t)kUX0 * 4 +
                               80 * 4 + 8 * kUBars + 16;
constexpr int kUEpiWarps = 8;                     // two warpgroups of epilogue warps
constexpr int kUThreads = 32 * (kUEpiWarps + 1);  // + the warp that issues the MMAs
constexpr int kUSlots = 8;                       // accumulator slots of 16 TMEM columns
constexpr int kUTmemCols = 16 * kUSlots;         // 128 columns: three CTAs per SM fit
static_assert(kUN3 == kUTY * kUP, "layer-3 rows");
static_assert(kUC2 * 128 >= kUN3 + 2 * kUP, "layer-2 extent");
static_assert(kUN1 >= kUC2 * 128 + 2 * kUP, "layer-1 extent");
static_assert(kUAct >= kUN1 + 2, "layer-2 taps of the last outputs stay inside the buffer");
static_assert(kUX0 >= kUN1 + 2 * kUP + 2, "layer-1 taps stay inside the input");
static_assert(kUSlots * 16 == kUTmemCols, "accumulator ring");
static_assert(kUEmbedSmem < (1u << 18), "descriptor start addresses fit their 14-bit field");
// kind::f16, A and B BF16, D FP32, both K-major, N = 16, M = 128
constexpr uint32_t kUIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((16u >> 3) << 17) |
                             ((128u >> 4) << 24);

// Weight operands in the canonical K-major layout: element (n, k) of a tile
// at byte (k / 8) * 256 + (n / 8) * 128 + (n % 8) * 16 + (k % 8) * 2.
__global__ void pack_umma_kernel(const float *__restrict__ prm, uint32_t *__restrict__ tiles) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;  // word: elements k, k + 1
    if (i >= (int)kUmmaWords) return;
    const int tile = i / (kUTileBytes / 4), b = 4 * (i % (kUTileBytes / 4));
    const int n = ((b >> 7) & 1) * 8 + ((b >> 4) & 7);
    const int k = (b >> 8) * 8 + ((b >> 1) & 7);
    float v[2];
    for (int j = 0; j < 2; ++j) {
        const int kk = k + j;
        if (tile == 0) {
            v[j] = kk < 9 ? prm[kOffW1 + kk * kCh + n] : 0.0f;  // w1[tap = kk][0][n]
        } else {
            const int tap = (tile - 1) % 9;
            const int off = tile <= 9 ? kOffW2 : kOffW3;
            v[j] = prm[off + (tap * kCh + kk) * kCh + n];
        }
    }
    tiles[i] = bf16x2(v[0], v[1]);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                          uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(kUIdesc), "r"(accumulate), "r"(z));
}

// The 9 tap MMAs of chunk c of a 16-channel layer into the accumulator at
// TMEM address d. adesc / wdesc: descriptors of the input activations and of
// the layer's first weight operand; a tap moves the start-address field
// (16-byte units, shared addresses stay below 256 KB so the field never
// carries).
__device__ __forceinline__ void umma_chunk16(uint32_t d, uint64_t adesc, uint64_t wdesc, int c) {
#pragma unroll
    for (int tap = 0; tap < 9; ++tap)
        umma_bf16(d,
                  adesc + (uint64_t)(c * 128 + (tap / 3) * kUP + tap % 3),
                  wdesc + (uint64_t)(tap * (kUTileBytes / 16)), tap > 0);
}

// ReLU epilogue of chunk c of a 16-channel layer whose output f is
// half-resolution pixel (oy + org + f / kUP, ox + org + f % kUP): BF16 into
// the activation planes, zero outside the plane (INSIDE: the layer's whole
// region lies inside the plane, no test). ta: this warp's TMEM lanes of the
// chunk's accumulator slot; b: the biases (16 floats, 8-byte aligned).
template <bool INSIDE>
__device__ __forceinline__ void umma_epilogue_relu(uint32_t ta, unsigned char *act,
                                                   const float *b, int c, int oy, int ox,
                                                   int org, int w2, int h2) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float v[16];
    tmem_ld16(ta, v);
    const int f = c * 128 + 32 * (warp & 3) + lane;
    bool in = true;
    if (!INSIDE) {
        const int yy = oy + org + f / kUP, xx = ox + org + f % kUP;
        in = yy >= 0 && yy < h2 && xx >= 0 && xx < w2;
    }
    const f32x2 *bp = reinterpret_cast<const f32x2 *>(b);
    uint32_t h[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        float lo, hi;
        unpack2(add2(pack2(v[2 * k], v[2 * k + 1]), bp[k]), lo, hi);
        h[k] = in ? bf16x2_relu(lo, hi) : 0u;
    }
    *reinterpret_cast<uint4 *>(act + 16 * f) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4 *>(act + kUAct * 16 + 16 * f) = make_uint4(h[4], h[5], h[6], h[7]);
}

// Whether the rows x 128 region of a layer starting at (y0, x0) lies inside
// the h2 x w2 plane.
__device__ __forceinline__ bool region_inside(int y0, int x0, int rows, int w2, int h2) {
    return y0 >= 0 && x0 >= 0 && y0 + rows <= h2 && x0 + kUP <= w2;
}

__global__ void __launch_bounds__(kUThreads, 3)
    embed_umma_kernel(const float *__restrict__ src, long long frame_floats, int width,
                      int height, int stride, const uint4 *__restrict__ wtiles,
                      const float *__restrict__ bias, uint8_t *__restrict__ emb,
                      long long emb_frame, unsigned *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char usmem[];
    unsigned char *act = usmem;
    unsigned char *wts = act + kUActBytes;
    float *x0 = reinterpret_cast<float *>(wts + kUTiles * kUTileBytes);
    float *sb = x0 + kUX0;  // [48] biases, qscale, [16] qoffsets
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sb + 80);  // [kUBars]
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + kUBars);
    const uint32_t act_s = (uint32_t)__cvta_generic_to_shared(act);
    const uint32_t wts_s = (uint32_t)__cvta_generic_to_shared(wts);
    const uint32_t mbar_s = (uint32_t)__cvta_generic_to_shared(mbar);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int w2 = width / 2, h2 = height / 2;
    const int oy = blockIdx.y * kUTY, ox = blockIdx.x * kUTX;
    src += blockIdx.z * frame_floats;
    emb += blockIdx.z * emb_frame;

    // barriers: done1[13], done2[11], done3[9] (one commit each), then
    // written1[13], written2[11], read3[9] (one arrival per epilogue warp of
    // the chunk's warpgroup). Chunks take accumulator slots in issue order
    // (sequence number n: layer-1 chunks, then layer 2, then layer 3; slot
    // n % 8); chunk n is issued once chunk n - 8's epilogue has read its slot.
    const uint32_t done1 = mbar_s, done2 = done1 + 8u * kUC1, done3 = done2 + 8u * kUC2;
    const uint32_t wr1 = done3 + 8u * kUC3, wr2 = wr1 + 8u * kUC1, rd3 = wr2 + 8u * kUC2;
    auto slot = [&](int n) { return 16u * (uint32_t)(n % kUSlots); };
    // the barrier that marks chunk n's accumulator as read
    auto read_bar = [&](int n) {
        return n < kUC1 ? wr1 + 8u * n
                        : n < kUC1 + kUC2 ? wr2 + 8u * (n - kUC1) : rd3 + 8u * (n - kUC1 - kUC2);
    };
    if (warp == kUEpiWarps) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tslot)),
                     "r"(kUTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid < kUBars) mbar_init(mbar_s + 8u * tid, tid < kUC1 + kUC2 + kUC3 ? 1u : 4u);
    // All of a thread's global loads (weights, its input pixels) are issued
    // before the first shared-memory store: one memory latency, not one per
    // loop iteration. Input pixel f is the 2x2 mean of the frame at
    // (2 yy, 2 xx); horizontal pairs load as float2 when rows are 8-byte
    // aligned.
    constexpr int kUWIter = (kUTiles * kUTileBytes / 16 + kUThreads - 1) / kUThreads;
    constexpr int kUIn = (kUX0 + kUThreads - 1) / kUThreads;
    uint4 wv[kUWIter];
#pragma unroll
    for (int k = 0; k < kUWIter; ++k) {
        const int i = tid + k * kUThreads;
        if (i < kUTiles * kUTileBytes / 16) wv[k] = __ldg(wtiles + i);
    }
    const float bv = tid < 65 ? __ldg(bias + tid) : 0.0f;
    const bool pairs =
        (stride & 1) == 0 && (reinterpret_cast<unsigned long long>(src) & 7ull) == 0;
    float2 ra[kUIn], rb[kUIn];
#pragma unroll
    for (int k = 0; k < kUIn; ++k) {
        const int f = tid + k * kUThreads;
        const int yy = oy - 3 + f / kUP, xx = ox - 3 + f % kUP;
        ra[k] = rb[k] = make_float2(0.0f, 0.0f);
        if (f < kUX0 && yy >= 0 && yy < h2 && xx >= 0 && xx < w2) {
            const float *s = src + (size_t)(2 * yy) * stride + 2 * xx;
            if (pairs) {
                ra[k] = __ldg(reinterpret_cast<const float2 *>(s));
                rb[k] = __ldg(reinterpret_cast<const float2 *>(s + stride));
            } else {
                ra[k] = make_float2(__ldg(s), __ldg(s + 1));
                rb[k] = make_float2(__ldg(s + stride), __ldg(s + stride + 1));
            }
        }
    }
#pragma unroll
    for (int k = 0; k < kUWIter; ++k) {
        const int i = tid + k * kUThreads;
        if (i < kUTiles * kUTileBytes / 16) reinterpret_cast<uint4 *>(wts)[i] = wv[k];
    }
    if (tid < 65) sb[tid] = bv;
    for (int i = tid; i < 2 * (kUAct - kUN1); i += kUThreads)
        *reinterpret_cast<uint4 *>(act + (i / (kUAct - kUN1)) * kUAct * 16 +
                                   16 * (kUN1 + i % (kUAct - kUN1))) = make_uint4(0, 0, 0, 0);
#pragma unroll
    for (int k = 0; k < kUIn; ++k) {
        const int f = tid + k * kUThreads;
        if (f < kUX0) x0[f] = 0.25f * ((ra[k].x + ra[k].y) + (rb[k].x + rb[k].y));
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    // layer-1 operand: row f holds the 9 taps of output f, then zeros
    for (int f = tid; f < kUN1; f += kUThreads) {
        float t[9];
#pragma unroll
        for (int k = 0; k < 9; ++k) t[k] = x0[f + (k / 3) * kUP + k % 3];
        *reinterpret_cast<uint4 *>(act + 16 * f) =
            make_uint4(bf16x2(t[0], t[1]), bf16x2(t[2], t[3]), bf16x2(t[4], t[5]),
                       bf16x2(t[6], t[7]));
        *reinterpret_cast<uint4 *>(act + kUAct * 16 + 16 * f) =
            make_uint4(bf16x2(t[8], 0.0f), 0u, 0u, 0u);
    }
    fence_async_smem();
    __syncthreads();

    bool ok = true;
    if (warp == kUEpiWarps) {
        // the MMA issuer
        if (lane == 0) {
            const uint64_t adesc0 = umma_desc(act_s, kUAct * 16u, 128u);
            tc_fence_after();
            // waits until chunk n's accumulator slot has been read back
            auto slot_free = [&](int n) {
                if (ok && n >= kUSlots) {
                    ok = mbar_wait_bounded(read_bar(n - kUSlots), 0);
                    tc_fence_after();
                }
            };
            for (int c = 0; c < kUC1 && ok; ++c) {
                slot_free(c);
                if (!ok) break;
                umma_bf16(tmem + slot(c), umma_desc(act_s + 16u * c * 128, kUAct * 16u, 128u),
                          umma_desc(wts_s, 256u, 128u), 0u);
                umma_commit(done1 + 8u * c);
            }
            int w = 0;
            for (int c = 0; c < kUC2 && ok; ++c) {
                for (; ok && w <= min(c + 3, kUC1 - 1); ++w)
                    ok = mbar_wait_bounded(wr1 + 8u * w, 0);
                slot_free(kUC1 + c);
                if (!ok) break;
                tc_fence_after();
                umma_chunk16(tmem + slot(kUC1 + c), adesc0,
                             umma_desc(wts_s + kUTileBytes, 256u, 128u), c);
                umma_commit(done2 + 8u * c);
            }
            w = 0;
            for (int c = 0; c < kUC3 && ok; ++c) {
                for (; ok && w <= min(c + 3, kUC2 - 1); ++w)
                    ok = mbar_wait_bounded(wr2 + 8u * w, 0);
                slot_free(kUC1 + kUC2 + c);
                if (!ok) break;
                tc_fence_after();
                umma_chunk16(tmem + slot(kUC1 + kUC2 + c), adesc0,
                             umma_desc(wts_s + 10 * kUTileBytes, 256u, 128u), c);
                umma_commit(done3 + 8u * c);
            }
        }
    } else {
        // epilogue warps: warpgroup g takes chunks g, g + 2, ...
        const int g = warp >> 2;
        const uint32_t tq = tmem + ((uint32_t)(32 * (warp & 3)) << 16);
        const bool inside1 = region_inside(oy - 2, ox - 2, kUC1, w2, h2);
        const bool inside2 = region_inside(oy - 1, ox - 1, kUC2, w2, h2);
        for (int c = g; c < kUC1 && ok; c += 2) {
            ok = __all_sync(0xffffffffu, mbar_wait_bounded(done1 + 8u * c, 0));
            if (!ok) break;
            tc_fence_after();
            if (inside1) umma_epilogue_relu<true>(tq + slot(c), act, sb, c, oy, ox, -2, w2, h2);
            else umma_epilogue_relu<false>(tq + slot(c), act, sb, c, oy, ox, -2, w2, h2);
            fence_async_smem();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(wr1 + 8u * c);
        }
        for (int c = g; c < kUC2 && ok; c += 2) {
            ok = __all_sync(0xffffffffu, mbar_wait_bounded(done2 + 8u * c, 0));
            if (!ok) break;
            tc_fence_after();
            const uint32_t ta = tq + slot(kUC1 + c);
            if (inside2) umma_epilogue_relu<true>(ta, act, sb + 16, c, oy, ox, -1, w2, h2);
            else umma_epilogue_relu<false>(ta, act, sb + 16, c, oy, ox, -1, w2, h2);
            fence_async_smem();
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(wr2 + 8u * c);
        }
        // layer 3, quantised: q = clamp(rint((acc + b3) * qscale + qoff[c]), 0, 255)
        const float qs = sb[48];
        for (int c = g; c < kUC3 && ok; c += 2) {
            ok = __all_sync(0xffffffffu, mbar_wait_bounded(done3 + 8u * c, 0));
            if (!ok) break;
            tc_fence_after();
            float v[16];
            tmem_ld16(tq + slot(kUC1 + kUC2 + c), v);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(rd3 + 8u * c);
            const int f = c * 128 + 32 * (warp & 3) + lane;
            const int i = f / kUP, j = f % kUP;
            const int yy = oy + i, xx = ox + j;
            if (j >= kUTX || yy >= h2 || xx >= w2) continue;
            uint32_t q[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                uint32_t word = 0;
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int ch = 4 * k + e;
                    word |= quantize_u8(__fadd_rn(v[ch], sb[32 + ch]), qs, sb[49 + ch]) << (8 * e);
                }
                q[k] = word;
            }
            *reinterpret_cast<uint4 *>(emb + ((size_t)yy * w2 + xx) * kCh) =
                make_uint4(q[0], q[1], q[2], q[3]);
        }
    }
    tc_fence_before();
    ok = __syncthreads_and(ok);
    if (!ok && tid == 0) atomicOr(err, 1u);
    if (warp == kUEpiWarps) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kUTmemCols)
                     : "memory");
    }
}

}  // namespace

cudaError_t launch_embed(const float *src, long long frame_floats, int nframes, int width,
                         int height, int stride, const uint32_t *frag, const float *bias,
                         uint8_t *emb, long long emb_frame, unsigned *err, cudaStream_t s) {
    if (nframes <= 0) return cudaSuccess;
    static int configured[64] = {0};
    cudaError_t e = raise_smem_limit(configured, (const void *)embed_umma_kernel, kUEmbedSmem);
    if (e != cudaSuccess) return e;
    const int w2 = width / 2, h2 = height / 2;
    dim3 grid((w2 + kUTX - 1) / kUTX, (h2 + kUTY - 1) / kUTY, nframes);
    embed_umma_kernel<<<grid, kUThreads, kUEmbedSmem, s>>>(
        src, frame_floats, width, height, stride, reinterpret_cast<const uint4 *>(frag),
        bias, emb, emb_frame, err);
    return cudaGetLastError();
}

}  // namespace bm3d

// ===========================================================================
// C ABI: the proposer object
// ===========================================================================
using namespace bm3d;

struct bm3d_b200_proposer {
    int device = 0;
    float *d_prm = nullptr;                // [4800] FP32 master parameters
    float *d_grad = nullptr;               // [4800]
    float *d_m = nullptr, *d_v = nullptr;  // Adam moments
    int *d_step = nullptr;                 // Adam step counter
    uint32_t *d_frag = nullptr;            // inference weights (tensor-core operand layout)
    unsigned *h_err = nullptr;             // inference error word (mapped host memory)
    unsigned *d_err = nullptr;             // its device address
    float *d_bias = nullptr;               // [48] biases, then [17] quantisation
    float quant[17] = {};                  // qscale, qoff[16]
    float *d_work = nullptr;               // training activations (grown on demand)
    size_t work_floats = 0;
    float *d_loss = nullptr;
    int *d_count = nullptr;
};

namespace bm3d {

const uint32_t *proposer_frag(const bm3d_b200_proposer *p) { return p->d_frag; }
const float *proposer_bias(const bm3d_b200_proposer *p) { return p->d_bias; }
unsigned *proposer_err(const bm3d_b200_proposer *p) { return p->d_err; }
int proposer_check(const bm3d_b200_proposer *p) {
    if (!p || *(volatile unsigned *)p->h_err == 0) return BM3D_B200_OK;
    return abi_fail(BM3D_B200_ERR_CUDA,
                    "BM3D proposer: an inference tile timed out waiting for its tensor-core work");
}
int proposer_device(const bm3d_b200_proposer *p) { return p->device; }

}  // namespace bm3d

namespace {

int pfail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return bm3d::abi_fail(code, buf);
}

#define PTRY(expr)                                                                       \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return pfail(BM3D_B200_ERR_CUDA, "BM3D proposer: '%s' failed: %s", #expr,   \
                         cudaGetErrorString(e_));                                        \
    } while (0)

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

// Coarse initialisation: channel k = scale * the half-resolution pixel at
// offset (k/4 - 2, k%4 - 2) from the cell + 2 (the block's 4x4 footprint),
// routed through the three layers in steps of at most one pixel.
void coarse_init(std::vector<float> &p, float scale) {
    p.assign(BM3D_B200_PROPOSER_PARAMS, 0.0f);
    for (int c = 0; c < kCh; ++c) p[kOffB1 + c] = 1.0f;  // keeps pixel copies positive
    auto clamp1 = [](int v) { return std::max(-1, std::min(1, v)); };
    for (int k = 0; k < kCh; ++k) {
        const int dy = k / 4 - 2, dx = k % 4 - 2;
        const int s1y = clamp1(dy), s1x = clamp1(dx);
        const int s2y = clamp1(dy - s1y), s2x = clamp1(dx - s1x);
        const int s3y = dy - s1y - s2y, s3x = dx - s1x - s2x;
        p[kOffW1 + ((1 + s1y) * 3 + (1 + s1x)) * kCh + k] = 1.0f;
        p[kOffW2 + (((1 + s2y) * 3 + (1 + s2x)) * kCh + k) * kCh + k] = 1.0f;
        p[kOffW3 + (((1 + s3y) * 3 + (1 + s3x)) * kCh + k) * kCh + k] = scale;
    }
}

int repack(bm3d_b200_proposer *p, cudaStream_t s) {
    pack_bias_kernel<<<1, 64, 0, s>>>(p->d_prm, p->d_bias);
    PTRY(cudaGetLastError());
    pack_umma_kernel<<<(kUmmaWords + 127) / 128, 128, 0, s>>>(p->d_prm, p->d_frag);
    PTRY(cudaGetLastError());
    return BM3D_B200_OK;
}

// Quantisation of the coarse network (outputs 8 * (pixel + 1), pixels about
// [-0.2, 1.2]): q = 20 v - 100 spans [28, 252].
void default_quant(float q[17]) {
    q[0] = 20.0f;
    for (int c = 0; c < kCh; ++c) q[1 + c] = -100.0f;
}

int upload_quant(bm3d_b200_proposer *p, cudaStream_t s) {
    PTRY(cudaMemcpyAsync(p->d_bias + 48, p->quant, 17 * sizeof(float), cudaMemcpyHostToDevice,
                         s));
    PTRY(cudaStreamSynchronize(s));
    return BM3D_B200_OK;
}

// FP32 network embeddings of nframes planes into d_emb ([n][h/2][w/2][16]).
int forward_f32(bm3d_b200_proposer *p, const float *d_frames, int nframes, int width,
                int height, int stride, float *d_emb, cudaStream_t s) {
    const int w2 = width / 2, h2 = height / 2;
    const size_t px = (size_t)nframes * w2 * h2;
    float *tmp = nullptr;
    PTRY(cudaMallocAsync(&tmp, px * (1 + 2 * kCh) * sizeof(float), s));
    float *x0 = tmp, *r1 = tmp + px, *r2 = r1 + px * kCh;
    downsample2_kernel<<<dim3((w2 + 127) / 128, h2, nframes), 128, 0, s>>>(
        d_frames, (long long)height * stride, stride, w2, h2, x0);
    const int grid = (int)((px + 127) / 128);
    const float *prm = p->d_prm;
    conv3x3_fwd_kernel<1, kCh><<<grid, 128, 0, s>>>(x0, prm + kOffW1, prm + kOffB1, r1, w2, h2,
                                                    nframes, 1);
    conv3x3_fwd_kernel<kCh, kCh><<<grid, 128, 0, s>>>(r1, prm + kOffW2, prm + kOffB2, r2, w2, h2,
                                                      nframes, 1);
    conv3x3_fwd_kernel<kCh, kCh><<<grid, 128, 0, s>>>(r2, prm + kOffW3, prm + kOffB3, d_emb, w2,
                                                      h2, nframes, 0);
    PTRY(cudaGetLastError());
    PTRY(cudaFreeAsync(tmp, s));
    return BM3D_B200_OK;
}

// Quantisation from the embeddings of sample frames: one scale that puts
// +-4 standard deviations of the widest channel into [1, 255], offsets that
// centre every channel at 128.
int calibrate(bm3d_b200_proposer *p, const float *d_frames, int nframes, int width, int height,
              int stride, cudaStream_t s) {
    const size_t n = (size_t)nframes * (width / 2) * (height / 2);
    float *d_e = nullptr;
    PTRY(cudaMallocAsync(&d_e, n * kCh * sizeof(float), s));
    std::vector<float> e(n * kCh);
    int rc = forward_f32(p, d_frames, nframes, width, height, stride, d_e, s);
    cudaError_t ce = rc ? cudaSuccess
                        : cudaMemcpyAsync(e.data(), d_e, e.size() * sizeof(float),
                                          cudaMemcpyDeviceToHost, s);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s);
    cudaFreeAsync(d_e, s);
    if (rc) return rc;
    PTRY(ce);
    double mean[kCh] = {}, var[kCh] = {};
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < kCh; ++c) mean[c] += e[i * kCh + c];
    for (int c = 0; c < kCh; ++c) mean[c] /= (double)std::max<size_t>(1, n);
    for (size_t i = 0; i < n; ++i)
        for (int c = 0; c < kCh; ++c) {
            const double d = e[i * kCh + c] - mean[c];
            var[c] += d * d;
        }
    double sd = 0.0;
    for (int c = 0; c < kCh; ++c) sd = std::max(sd, std::sqrt(var[c] / std::max<size_t>(1, n)));
    const double qs = sd > 0.0 ? 127.0 / (4.0 * sd) : 1.0;
    p->quant[0] = (float)qs;
    for (int c = 0; c < kCh; ++c) p->quant[1 + c] = (float)(128.0 - qs * mean[c]);
    return upload_quant(p, s);
}

int check_train_args(int nframes, int width, int height, int stride, int nsamples, int U) {
    if (nframes <= 0 || width < 16 || height < 16 || stride < width || nsamples < 0 || U < 1 ||
        U > 15)
        return pfail(BM3D_B200_ERR_INVALID,
                     "BM3D proposer: invalid training arguments (frames %d, %dx%d, stride %d, "
                     "samples %d, U %d)",
                     nframes, width, height, stride, nsamples, U);
    return BM3D_B200_OK;
}

// Samples with a positive cell (the loss's n).
int count_positive(bm3d_b200_proposer *p, const int *d_samples, const float *d_teacher,
                   int nsamples, int nframes, int width, int height, int U, cudaStream_t s,
                   int *n_pos) {
    *n_pos = 0;
    if (nsamples == 0) return BM3D_B200_OK;
    PTRY(cudaMemsetAsync(p->d_count, 0, sizeof(int), s));
    count_samples_kernel<<<(nsamples + 255) / 256, 256, 0, s>>>(
        reinterpret_cast<const int4 *>(d_samples), d_teacher, nsamples, nframes, width, height, U,
        p->d_count);
    PTRY(cudaGetLastError());
    PTRY(cudaMemcpyAsync(n_pos, p->d_count, sizeof(int), cudaMemcpyDeviceToHost, s));
    PTRY(cudaStreamSynchronize(s));
    return BM3D_B200_OK;
}

// Forward, loss and backward of one training step over all frames; the
// gradient lands in p->d_grad and the loss in p->d_loss.
int loss_grad(bm3d_b200_proposer *p, const float *d_frames, int nframes, int width, int height,
              int stride, const int *d_samples, const float *d_teacher, int nsamples, int U,
              float temperature, int n_pos, cudaStream_t s) {
    const int w2 = width / 2, h2 = height / 2;
    const size_t px = (size_t)nframes * w2 * h2;
    const size_t need = px * (1 + 4 * kCh);
    if (need > p->work_floats) {
        PTRY(cudaStreamSynchronize(s));
        cudaFree(p->d_work);
        p->d_work = nullptr;
        p->work_floats = 0;
        PTRY(cudaMalloc(&p->d_work, need * sizeof(float)));
        p->work_floats = need;
    }
    float *x0 = p->d_work;
    float *r1 = x0 + px;      // relu(conv1)
    float *r2 = r1 + px * kCh;  // relu(conv2)
    float *e = r2 + px * kCh;   // embeddings, later d r2
    float *g = e + px * kCh;    // d e, later d r1
    downsample2_kernel<<<dim3((w2 + 127) / 128, h2, nframes), 128, 0, s>>>(
        d_frames, (long long)height * stride, stride, w2, h2, x0);
    PTRY(cudaGetLastError());
    const int grid = (int)((px + 127) / 128);
    const float *prm = p->d_prm;
    conv3x3_fwd_kernel<1, kCh><<<grid, 128, 0, s>>>(x0, prm + kOffW1, prm + kOffB1, r1, w2, h2,
                                                    nframes, 1);
    conv3x3_fwd_kernel<kCh, kCh><<<grid, 128, 0, s>>>(r1, prm + kOffW2, prm + kOffB2, r2, w2, h2,
                                                      nframes, 1);
    conv3x3_fwd_kernel<kCh, kCh><<<grid, 128, 0, s>>>(r2, prm + kOffW3, prm + kOffB3, e, w2, h2,
                                                      nframes, 0);
    PTRY(cudaGetLastError());
    PTRY(cudaMemsetAsync(g, 0, px * kCh * sizeof(float), s));
    PTRY(cudaMemsetAsync(p->d_loss, 0, sizeof(float), s));
    PTRY(cudaMemsetAsync(p->d_grad, 0, BM3D_B200_PROPOSER_PARAMS * sizeof(float), s));
    if (n_pos > 0) {
        proposal_loss_kernel<<<(nsamples + 3) / 4, 128, 0, s>>>(
            e, w2, h2, reinterpret_cast<const int4 *>(d_samples), d_teacher, nsamples, nframes,
            width, height, U, 1.0f / temperature, 1.0f / n_pos, g, p->d_loss);
        PTRY(cudaGetLastError());
    }
    float *gw = p->d_grad;
    const int wrows = (int)std::min<size_t>(64, (px + 255) / 256);
    // layer 3 (no ReLU): weight gradient from r2 and d e; then d r2 into e
    conv3x3_bwd_weight_kernel<kCh, kCh><<<dim3(9 * kCh, wrows), 256, 0, s>>>(
        r2, g, nullptr, gw + kOffW3, gw + kOffB3, w2, h2, nframes, 0);
    conv3x3_bwd_data_kernel<kCh, kCh><<<grid, 128, 0, s>>>(g, nullptr, prm + kOffW3, e, w2, h2,
                                                           nframes, 0);
    PTRY(cudaGetLastError());
    // layer 2: output gradient d r2 masked by r2 > 0; d r1 into g
    conv3x3_bwd_weight_kernel<kCh, kCh><<<dim3(9 * kCh, wrows), 256, 0, s>>>(
        r1, e, r2, gw + kOffW2, gw + kOffB2, w2, h2, nframes, 1);
    conv3x3_bwd_data_kernel<kCh, kCh><<<grid, 128, 0, s>>>(e, r2, prm + kOffW2, g, w2, h2,
                                                           nframes, 1);
    PTRY(cudaGetLastError());
    // layer 1: output gradient d r1 masked by r1 > 0
    conv3x3_bwd_weight_kernel<1, kCh><<<dim3(9, wrows), 256, 0, s>>>(
        x0, g, r1, gw + kOffW1, gw + kOffB1, w2, h2, nframes, 1);
    PTRY(cudaGetLastError());
    return BM3D_B200_OK;
}

}  // namespace

extern "C" int bm3d_b200_proposer_num_params(void) { return BM3D_B200_PROPOSER_PARAMS; }

extern "C" int bm3d_b200_proposer_create(bm3d_b200_proposer **out, const float *params,
                                         int device) {
    if (!out) return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    *out = nullptr;
    int ndev = 0;
    PTRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev)
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: invalid device ID (%d)", device);
    PTRY(cudaSetDevice(device));
    auto *p = new (std::nothrow) bm3d_b200_proposer;
    if (!p) return pfail(BM3D_B200_ERR_NOMEM, "BM3D proposer: out of host memory");
    p->device = device;
    std::vector<float> init;
    if (!params) coarse_init(init, 8.0f);
    const size_t pb = BM3D_B200_PROPOSER_PARAMS * sizeof(float);
    auto cleanup = [&](int rc) {
        bm3d_b200_proposer_destroy(p);
        return rc;
    };
    if (cudaMalloc(&p->d_prm, pb) != cudaSuccess || cudaMalloc(&p->d_grad, pb) != cudaSuccess ||
        cudaMalloc(&p->d_m, pb) != cudaSuccess || cudaMalloc(&p->d_v, pb) != cudaSuccess ||
        cudaMalloc(&p->d_step, sizeof(int)) != cudaSuccess ||
        cudaMalloc(&p->d_frag, kUmmaWords * sizeof(uint32_t)) != cudaSuccess ||
        cudaHostAlloc(&p->h_err, sizeof(unsigned), cudaHostAllocMapped) != cudaSuccess ||
        cudaHostGetDevicePointer(reinterpret_cast<void **>(&p->d_err), p->h_err, 0) !=
            cudaSuccess ||
        cudaMalloc(&p->d_bias, (48 + 17) * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&p->d_loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&p->d_count, sizeof(int)) != cudaSuccess)
        return cleanup(pfail(BM3D_B200_ERR_NOMEM, "BM3D proposer: device allocation failed"));
    if (cudaMemcpy(p->d_prm, params ? params : init.data(), pb, cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemset(p->d_m, 0, pb) != cudaSuccess || cudaMemset(p->d_v, 0, pb) != cudaSuccess ||
        cudaMemset(p->d_step, 0, sizeof(int)) != cudaSuccess || (*p->h_err = 0, false))
        return cleanup(pfail(BM3D_B200_ERR_CUDA, "BM3D proposer: initialisation failed"));
    if (int rc = repack(p, nullptr)) return cleanup(rc);
    default_quant(p->quant);
    if (int rc = upload_quant(p, nullptr)) return cleanup(rc);
    if (cudaDeviceSynchronize() != cudaSuccess)
        return cleanup(pfail(BM3D_B200_ERR_CUDA, "BM3D proposer: initialisation failed"));
    *out = p;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_proposer_get_quant(bm3d_b200_proposer *p, float *h_quant) {
    if (!p || !h_quant) return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    std::copy(p->quant, p->quant + 17, h_quant);
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_proposer_set_quant(bm3d_b200_proposer *p, const float *h_quant) {
    if (!p) return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    PTRY(cudaSetDevice(p->device));
    if (h_quant) {
        if (!(h_quant[0] > 0.0f) || !std::isfinite(h_quant[0]))
            return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: quantisation scale must be > 0");
        std::copy(h_quant, h_quant + 17, p->quant);
    } else {
        default_quant(p->quant);
    }
    return upload_quant(p, nullptr);
}

extern "C" int bm3d_b200_proposer_calibrate(bm3d_b200_proposer *p, const float *d_frames,
                                            int nframes, int width, int height, int stride,
                                            void *stream) {
    if (!p || !d_frames) return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    if (nframes <= 0 || width < 16 || height < 16 || stride < width)
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: invalid plane %dx%d (stride %d)",
                     width, height, stride);
    PTRY(cudaSetDevice(p->device));
    return calibrate(p, d_frames, nframes, width, height, stride, as_stream(stream));
}

extern "C" void bm3d_b200_proposer_destroy(bm3d_b200_proposer *p) {
    if (!p) return;
    cudaSetDevice(p->device);
    cudaDeviceSynchronize();
    cudaFree(p->d_prm);
    cudaFree(p->d_grad);
    cudaFree(p->d_m);
    cudaFree(p->d_v);
    cudaFree(p->d_step);
    cudaFree(p->d_frag);
    cudaFreeHost(p->h_err);
    cudaFree(p->d_bias);
    cudaFree(p->d_work);
    cudaFree(p->d_loss);
    cudaFree(p->d_count);
    delete p;
}

extern "C" int bm3d_b200_proposer_get_params(bm3d_b200_proposer *p, float *h_params) {
    if (!p || !h_params) return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    PTRY(cudaSetDevice(p->device));
    PTRY(cudaMemcpy(h_params, p->d_prm, BM3D_B200_PROPOSER_PARAMS * sizeof(float),
                    cudaMemcpyDeviceToHost));
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_proposer_set_params(bm3d_b200_proposer *p, const float *h_params) {
    if (!p) return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    PTRY(cudaSetDevice(p->device));
    std::vector<float> init;
    if (!h_params) coarse_init(init, 8.0f);
    PTRY(cudaMemcpy(p->d_prm, h_params ? h_params : init.data(),
                    BM3D_B200_PROPOSER_PARAMS * sizeof(float), cudaMemcpyHostToDevice));
    PTRY(cudaMemset(p->d_m, 0, BM3D_B200_PROPOSER_PARAMS * sizeof(float)));
    PTRY(cudaMemset(p->d_v, 0, BM3D_B200_PROPOSER_PARAMS * sizeof(float)));
    PTRY(cudaMemset(p->d_step, 0, sizeof(int)));
    if (int rc = repack(p, nullptr)) return rc;
    PTRY(cudaDeviceSynchronize());
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_proposer_teacher(const float *d_frames, int nframes, int width,
                                          int height, int stride, const int *d_samples,
                                          int nsamples, int U, float *d_teacher, void *stream) {
    if (!d_frames || (nsamples > 0 && (!d_samples || !d_teacher)))
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    if (int rc = check_train_args(nframes, width, height, stride, nsamples, U)) return rc;
    if (nsamples == 0) return BM3D_B200_OK;
    cudaStream_t s = as_stream(stream);
    teacher_kernel<<<(nsamples + 3) / 4, 128, 0, s>>>(
        d_frames, (long long)height * stride, stride, reinterpret_cast<const int4 *>(d_samples),
        nsamples, nframes, width, height, U, d_teacher);
    PTRY(cudaGetLastError());
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_proposer_loss_grad(bm3d_b200_proposer *p, const float *d_frames,
                                            int nframes, int width, int height, int stride,
                                            const int *d_samples, const float *d_teacher,
                                            int nsamples, int U, float temperature,
                                            float *h_loss, float *h_grad, void *stream) {
    if (!p || !d_frames || (nsamples > 0 && (!d_samples || !d_teacher)))
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    if (int rc = check_train_args(nframes, width, height, stride, nsamples, U)) return rc;
    if (!(temperature > 0.0f))
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: temperature must be positive");
    PTRY(cudaSetDevice(p->device));
    cudaStream_t s = as_stream(stream);
    int n_pos = 0;
    if (int rc = count_positive(p, d_samples, d_teacher, nsamples, nframes, width, height, U, s,
                                &n_pos))
        return rc;
    if (int rc = loss_grad(p, d_frames, nframes, width, height, stride, d_samples, d_teacher,
                           nsamples, U, temperature, n_pos, s))
        return rc;
    if (h_loss) PTRY(cudaMemcpyAsync(h_loss, p->d_loss, sizeof(float), cudaMemcpyDeviceToHost, s));
    if (h_grad)
        PTRY(cudaMemcpyAsync(h_grad, p->d_grad, BM3D_B200_PROPOSER_PARAMS * sizeof(float),
                             cudaMemcpyDeviceToHost, s));
    PTRY(cudaStreamSynchronize(s));
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_proposer_train(bm3d_b200_proposer *p, const float *d_frames,
                                        int nframes, int width, int height, int stride,
                                        const int *d_samples, const float *d_teacher,
                                        int nsamples, int U, float temperature, int steps,
                                        float lr, float *h_losses, void *stream) {
    if (!p || !d_frames || !d_samples || !d_teacher)
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    if (int rc = check_train_args(nframes, width, height, stride, nsamples, U)) return rc;
    if (steps < 0 || !(lr > 0.0f) || !(temperature > 0.0f))
        return pfail(BM3D_B200_ERR_INVALID,
                     "BM3D proposer: invalid steps (%d), learning rate or temperature", steps);
    PTRY(cudaSetDevice(p->device));
    cudaStream_t s = as_stream(stream);
    int n_pos = 0;
    if (int rc = count_positive(p, d_samples, d_teacher, nsamples, nframes, width, height, U, s,
                                &n_pos))
        return rc;
    for (int i = 0; i < steps; ++i) {
        if (int rc = loss_grad(p, d_frames, nframes, width, height, stride, d_samples, d_teacher,
                               nsamples, U, temperature, n_pos, s))
            return rc;
        step_kernel<<<1, 1, 0, s>>>(p->d_step);
        adam_kernel<<<(BM3D_B200_PROPOSER_PARAMS + 255) / 256, 256, 0, s>>>(
            p->d_prm, p->d_grad, p->d_m, p->d_v, BM3D_B200_PROPOSER_PARAMS, lr, p->d_step);
        PTRY(cudaGetLastError());
        if (h_losses)
            PTRY(cudaMemcpyAsync(h_losses + i, p->d_loss, sizeof(float), cudaMemcpyDeviceToHost,
                                 s));
    }
    if (int rc = repack(p, s)) return rc;
    PTRY(cudaStreamSynchronize(s));
    return calibrate(p, d_frames, nframes, width, height, stride, s);
}

extern "C" int bm3d_b200_proposer_embed(bm3d_b200_proposer *p, const float *d_frames,
                                        int nframes, int width, int height, int stride,
                                        void *d_emb, void *stream) {
    if (!p || !d_frames || !d_emb)
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    if (nframes < 0 || width < 16 || height < 16 || stride < width ||
        width > BM3D_B200_MAX_DIM || height > BM3D_B200_MAX_DIM)
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: invalid plane %dx%d (stride %d)",
                     width, height, stride);
    PTRY(cudaSetDevice(p->device));
    const long long ef = (long long)(width / 2) * (height / 2) * kCh;
    PTRY(launch_embed(d_frames, (long long)height * stride, nframes, width, height, stride,
                      p->d_frag, p->d_bias, static_cast<uint8_t *>(d_emb), ef, p->d_err,
                      as_stream(stream)));
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_proposer_status(const bm3d_b200_proposer *p) {
    if (!p) return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    return proposer_check(p);
}

extern "C" int bm3d_b200_proposer_embed_f32(bm3d_b200_proposer *p, const float *d_frames,
                                            int nframes, int width, int height, int stride,
                                            float *d_emb, void *stream) {
    if (!p || !d_frames || !d_emb)
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: null argument");
    if (nframes <= 0 || width < 16 || height < 16 || stride < width)
        return pfail(BM3D_B200_ERR_INVALID, "BM3D proposer: invalid plane %dx%d (stride %d)",
                     width, height, stride);
    PTRY(cudaSetDevice(p->device));
    cudaStream_t s = as_stream(stream);
    if (int rc = forward_f32(p, d_frames, nframes, width, height, stride, d_emb, s)) return rc;
    PTRY(cudaStreamSynchronize(s));
    return BM3D_B200_OK;
}
