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
//     tensor cores (mma.sync m16n8k16, BF16 operands, FP32 accumulation)
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
// inference: fused three-layer network on the tensor cores
// ===========================================================================
//
// A CTA computes the embeddings of a kTY x kTX tile of half-resolution pixels
// of one frame (grid z = frame). Every layer's activations live in shared
// memory as flat arrays with the same row pitch kP = 64 (pixel (i, j) of a
// layer's region at index i*kP + j), so a 3x3 tap (dy, dx) of output index f
// reads input index f + dy*kP + dx and each layer is a GEMM of [outputs x
// (9 taps x 16 channels)] x [144 x 16]: nine m16n8k16 k-steps per 16
// consecutive outputs, two n-tiles. Columns past a layer's valid width are
// computed but never feed a valid output.
//   X0: input, FP32, half-resolution pixel (oy - 3 + i, ox - 3 + j)
//   X1 = relu(conv1(X0)) at (oy - 2 + i, ox - 2 + j), BF16
//   X2 = relu(conv2(X1)) at (oy - 1 + i, ox - 1 + j), BF16
//   out = conv3(X2) at (oy + i, ox + j), quantised to 8 bits per channel
//   (one global scale, a per-channel offset), straight to global memory.
// BF16 activations take 32 bytes per pixel (16 channels), with the two
// 16-byte halves swapped on every other group of four pixels so that the
// eight rows of an ldmatrix phase hit distinct banks. Layer 1 has one input
// channel: its k dimension is the 9 taps (+7 zeros). Pixels outside the
// plane are zero in every layer (the zero padding).
constexpr int kP = 64;
constexpr int kTX = kP - 6;          // 58 output columns
constexpr int kTY = 14;              // output rows
constexpr int kN3 = kTY * kP;        // layer-3 outputs computed (896)
constexpr int kN2 = (kTY + 2) * kP;  // layer-2 outputs (1024)
constexpr int kN1 = 1168;            // layer-1 outputs: >= kN2 + 2*kP + 2, multiple of 16
constexpr int kX0 = 1344;            // input floats: >= kN1 + 2*kP + 2 (21 rows)
constexpr int kX2 = 1040;            // layer-2 storage: >= kN3 + 2*kP + 2, multiple of 16
constexpr size_t kEmbedSmem = (size_t)kX0 * 4 + (size_t)kN1 * 32 + (size_t)kX2 * 32;
constexpr int kEmbedThreads = 256;
static_assert(kN1 >= kN2 + 2 * kP + 2 && kN1 % 16 == 0, "layer-1 extent");
static_assert(kX0 >= kN1 + 2 * kP + 2, "input extent");
static_assert(kX2 >= kN3 + 2 * kP + 2 && kX2 % 16 == 0, "layer-2 extent");

// Fragment-ordered BF16 weights: k-steps [layer 1][layer 2: 9 taps][layer 3:
// 9 taps] x 2 n-tiles x 32 lanes x 2 registers; FP32 biases [3][16] apart.
constexpr int kFragWords = (1 + 9 + 9) * 2 * 32 * 2;

__device__ __forceinline__ uint32_t bf16x2(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

// B fragment of m16n8k16 (.col): lane (g = lane/4, t = lane%4) holds
// B[k = 2t, 2t+1][n = g] and B[k = 2t+8, 2t+9][n = g].
__global__ void pack_weights_kernel(const float *__restrict__ prm, uint32_t *__restrict__ frag,
                                    float *__restrict__ bias) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 48) bias[i] = prm[(i < 16 ? kOffB1 : i < 32 ? kOffB2 : kOffB3) + (i & 15)];
    if (i >= kFragWords / 2) return;
    const int lane = i & 31;
    const int nt = (i >> 5) & 1;
    const int ks = i >> 6;  // 0: layer 1; 1..9: layer 2 taps; 10..18: layer 3 taps
    const int g = lane >> 2, t = lane & 3;
    const int n = nt * 8 + g;
    float v[4];
    for (int j = 0; j < 4; ++j) {
        const int k = (j < 2 ? 2 * t : 2 * t + 8) + (j & 1);
        if (ks == 0) {
            v[j] = k < 9 ? prm[kOffW1 + k * kCh + n] : 0.0f;  // w1[tap = k][0][n]
        } else {
            const int tap = (ks - 1) % 9;
            const int off = ks <= 9 ? kOffW2 : kOffW3;
            v[j] = prm[off + (tap * kCh + k) * kCh + n];
        }
    }
    frag[2 * i] = bf16x2(v[0], v[1]);
    frag[2 * i + 1] = bf16x2(v[2], v[3]);
}

__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
        "{%8,%9}, {%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ void ldmatrix_x4(uint32_t (&a)[4], uint32_t addr) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];"
                 : "=r"(a[0]), "=r"(a[1]), "=r"(a[2]), "=r"(a[3])
                 : "r"(addr));
}

// byte offset of channel half `chunk` of pixel f in a BF16 activation array
__device__ __forceinline__ uint32_t act_off(int f, int chunk) {
    return (uint32_t)f * 32u + (uint32_t)((chunk ^ ((f >> 2) & 1)) << 4);
}

// A layer's B fragments of this lane: [tap][n-tile 0 b0, b1, n-tile 1 b0, b1].
__device__ __forceinline__ void load_layer_frag(uint32_t (&w)[9][4],
                                                const uint32_t *__restrict__ frag, int lane) {
#pragma unroll
    for (int tap = 0; tap < 9; ++tap) {
        const uint32_t *fb = frag + tap * 128 + lane * 2;
        w[tap][0] = __ldg(fb);
        w[tap][1] = __ldg(fb + 1);
        w[tap][2] = __ldg(fb + 64);
        w[tap][3] = __ldg(fb + 65);
    }
}

// One 16-channel 3x3 layer (k-steps = taps) for R output m-tiles of 16
// pixels stacked vertically (f0, f0 + kP, ... f0 + (R-1) kP). ldmatrix.x4
// lanes 0-7 / 8-15 / 16-23 / 24-31 address rows 0-7 / 8-15 of channels 0-7,
// then of channels 8-15, which is the A-fragment order. Every A fragment (one
// source row, one horizontal tap) is loaded once and feeds the up to three
// output rows it is a vertical tap of; each output still accumulates its taps
// in the order 0 .. 8.
template <int R>
__device__ __forceinline__ void conv16_strip(float (&acc)[R][2][4], uint32_t in_base, int f0,
                                             const uint32_t (&w)[9][4], int lane) {
    const int row = lane & 15, chunk = lane >> 4;
#pragma unroll
    for (int so = 0; so < R + 2; ++so) {
#pragma unroll
        for (int dx = 0; dx < 3; ++dx) {
            uint32_t a[4];
            ldmatrix_x4(a, in_base + act_off(f0 + row + so * kP + dx, chunk));
#pragma unroll
            for (int i = 0; i < R; ++i) {
                const int dy = so - i;
                if (dy < 0 || dy > 2) continue;
                const int tap = dy * 3 + dx;
                mma_bf16(acc[i][0], a, w[tap][0], w[tap][1]);
                mma_bf16(acc[i][1], a, w[tap][2], w[tap][3]);
            }
        }
    }
}

// Embedding quantisation to 8 bits, round to nearest even, saturating.
__device__ __forceinline__ int quantize(float v, float qs, float qo) {
    return min(max(__float2int_rn(__fmaf_rn(v, qs, qo)), 0), 255);
}

__global__ void __launch_bounds__(kEmbedThreads, 2)
    embed_kernel(const float *__restrict__ src, long long frame_floats, int width, int height,
                 int stride, const uint32_t *__restrict__ frag, const float *__restrict__ bias,
                 uint8_t *__restrict__ emb, long long emb_frame) {
    extern __shared__ __align__(16) unsigned char smem[];
    float *x0 = reinterpret_cast<float *>(smem);
    unsigned char *x1 = smem + kX0 * 4;
    unsigned char *x2 = x1 + kN1 * 32;
    const uint32_t x1s = (uint32_t)__cvta_generic_to_shared(x1);
    const uint32_t x2s = (uint32_t)__cvta_generic_to_shared(x2);
    const int w2 = width / 2, h2 = height / 2;
    const int oy = blockIdx.y * kTY, ox = blockIdx.x * kTX;  // output tile origin
    src += blockIdx.z * frame_floats;
    emb += blockIdx.z * emb_frame;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = kEmbedThreads / 32;
    const int g = lane >> 2, t = lane & 3;

    for (int f = threadIdx.x; f < kX0; f += kEmbedThreads) {
        const int yy = oy - 3 + f / kP, xx = ox - 3 + f % kP;
        float v = 0.0f;
        if (yy >= 0 && yy < h2 && xx >= 0 && xx < w2) {
            const float *s = src + (size_t)(2 * yy) * stride + 2 * xx;
            v = 0.25f * ((__ldg(s) + __ldg(s + 1)) + (__ldg(s + stride) + __ldg(s + stride + 1)));
        }
        x0[f] = v;
    }
    __syncthreads();

    // layer 1
    {
        const uint32_t *fb = frag + lane * 2;
        const uint32_t b00 = __ldg(fb), b01 = __ldg(fb + 1), b10 = __ldg(fb + 64),
                       b11 = __ldg(fb + 65);
        for (int mt = warp; mt < kN1 / 16; mt += nwarps) {
            const int f0 = mt * 16;
            auto tapv = [&](int f, int k) {
                return k < 9 ? x0[f + (k / 3) * kP + (k % 3)] : 0.0f;
            };
            uint32_t a[4];
            a[0] = bf16x2(tapv(f0 + g, 2 * t), tapv(f0 + g, 2 * t + 1));
            a[1] = bf16x2(tapv(f0 + g + 8, 2 * t), tapv(f0 + g + 8, 2 * t + 1));
            a[2] = bf16x2(tapv(f0 + g, 2 * t + 8), tapv(f0 + g, 2 * t + 9));
            a[3] = bf16x2(tapv(f0 + g + 8, 2 * t + 8), tapv(f0 + g + 8, 2 * t + 9));
            float acc[2][4] = {};
            mma_bf16(acc[0], a, b00, b01);
            mma_bf16(acc[1], a, b10, b11);
#pragma unroll
            for (int h = 0; h < 2; ++h) {  // rows g, g + 8 of the m-tile
                const int f = f0 + g + 8 * h;
                const int yy = oy - 2 + f / kP, xx = ox - 2 + f % kP;
                const bool in = yy >= 0 && yy < h2 && xx >= 0 && xx < w2;
#pragma unroll
                for (int nt = 0; nt < 2; ++nt) {
                    const int c = nt * 8 + 2 * t;
                    const float v0 = in ? fmaxf(acc[nt][2 * h] + bias[c], 0.0f) : 0.0f;
                    const float v1 = in ? fmaxf(acc[nt][2 * h + 1] + bias[c + 1], 0.0f) : 0.0f;
                    *reinterpret_cast<uint32_t *>(x1 + act_off(f, nt) + 4 * t) = bf16x2(v0, v1);
                }
            }
        }
    }
    __syncthreads();

    // layer 2: tasks of 4 output rows x 16 pixels (16 rows x 4 column blocks)
    uint32_t wf[9][4];
    load_layer_frag(wf, frag + 128, lane);
    auto store2 = [&](const float (&acc)[2][4], int f0) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int f = f0 + g + 8 * h;
            const int yy = oy - 1 + f / kP, xx = ox - 1 + f % kP;
            const bool in = f < kN2 && yy >= 0 && yy < h2 && xx >= 0 && xx < w2;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                const int c = nt * 8 + 2 * t;
                const float v0 = in ? fmaxf(acc[nt][2 * h] + bias[16 + c], 0.0f) : 0.0f;
                const float v1 = in ? fmaxf(acc[nt][2 * h + 1] + bias[16 + c + 1], 0.0f) : 0.0f;
                *reinterpret_cast<uint32_t *>(x2 + act_off(f, nt) + 4 * t) = bf16x2(v0, v1);
            }
        }
    };
    static_assert(kN2 == 16 * kP, "layer-2 rows");
    for (int task = warp; task < 16; task += nwarps) {
        const int f0 = (task >> 2) * 4 * kP + (task & 3) * 16;
        float acc[4][2][4] = {};
        conv16_strip<4>(acc, x1s, f0, wf, lane);
#pragma unroll
        for (int i = 0; i < 4; ++i) store2(acc[i], f0 + i * kP);
    }
    // the layer-2 tail past its 16 rows reads as zero in layer 3
    for (int f = kN2 + threadIdx.x; f < kX2; f += kEmbedThreads)
        for (int nt = 0; nt < 2; ++nt)
            *reinterpret_cast<uint4 *>(x2 + act_off(f, nt)) = make_uint4(0, 0, 0, 0);
    __syncthreads();

    // layer 3, quantised: q = clamp(rint((acc + b3) * qscale + qoff[c]), 0, 255);
    // tasks of 4 output rows (the last of 2) x 16 pixels
    const float qs = bias[48];
    load_layer_frag(wf, frag + 128 + 9 * 128, lane);
    auto store3 = [&](const float (&acc)[2][4], int f0) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int f = f0 + g + 8 * h;
            const int i = f / kP, j = f % kP;
            const int yy = oy + i, xx = ox + j;
            if (j >= kTX || yy >= h2 || xx >= w2) continue;
            uint8_t *dst = emb + ((size_t)yy * w2 + xx) * kCh;
#pragma unroll
            for (int nt = 0; nt < 2; ++nt) {
                const int c = nt * 8 + 2 * t;
                const int q0 = quantize(__fadd_rn(acc[nt][2 * h], bias[32 + c]), qs, bias[49 + c]);
                const int q1 = quantize(__fadd_rn(acc[nt][2 * h + 1], bias[33 + c]), qs,
                                        bias[50 + c]);
                *reinterpret_cast<uint16_t *>(dst + c) = (uint16_t)(q0 | (q1 << 8));
            }
        }
    };
    static_assert(kTY == 14, "layer-3 row tasks: 3 x 4 rows + 2 rows");
    for (int task = warp; task < 16; task += nwarps) {
        const int rg = task >> 2, f0 = rg * 4 * kP + (task & 3) * 16;
        if (rg < 3) {
            float acc[4][2][4] = {};
            conv16_strip<4>(acc, x2s, f0, wf, lane);
#pragma unroll
            for (int i = 0; i < 4; ++i) store3(acc[i], f0 + i * kP);
        } else {
            float acc[2][2][4] = {};
            conv16_strip<2>(acc, x2s, f0, wf, lane);
#pragma unroll
            for (int i = 0; i < 2; ++i) store3(acc[i], f0 + i * kP);
        }
    }
}

}  // namespace

cudaError_t launch_embed(const float *src, long long frame_floats, int nframes, int width,
                         int height, int stride, const uint32_t *frag, const float *bias,
                         uint8_t *emb, long long emb_frame, cudaStream_t s) {
    if (nframes <= 0) return cudaSuccess;
    static int configured[64] = {0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || !configured[dev]) {
        e = cudaFuncSetAttribute(embed_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kEmbedSmem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) configured[dev] = 1;
    }
    const int w2 = width / 2, h2 = height / 2;
    dim3 grid((w2 + kTX - 1) / kTX, (h2 + kTY - 1) / kTY, nframes);
    embed_kernel<<<grid, kEmbedThreads, kEmbedSmem, s>>>(src, frame_floats, width, height, stride,
                                                         frag, bias, emb, emb_frame);
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
    uint32_t *d_frag = nullptr;            // inference weights (fragment order)
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
    pack_weights_kernel<<<(kFragWords / 2 + 127) / 128, 128, 0, s>>>(p->d_prm, p->d_frag,
                                                                     p->d_bias);
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
        cudaMalloc(&p->d_frag, kFragWords * sizeof(uint32_t)) != cudaSuccess ||
        cudaMalloc(&p->d_bias, (48 + 17) * sizeof(float)) != cudaSuccess ||
        cudaMalloc(&p->d_loss, sizeof(float)) != cudaSuccess ||
        cudaMalloc(&p->d_count, sizeof(int)) != cudaSuccess)
        return cleanup(pfail(BM3D_B200_ERR_NOMEM, "BM3D proposer: device allocation failed"));
    if (cudaMemcpy(p->d_prm, params ? params : init.data(), pb, cudaMemcpyHostToDevice) !=
            cudaSuccess ||
        cudaMemset(p->d_m, 0, pb) != cudaSuccess || cudaMemset(p->d_v, 0, pb) != cudaSuccess ||
        cudaMemset(p->d_step, 0, sizeof(int)) != cudaSuccess)
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
                      p->d_frag, p->d_bias, static_cast<uint8_t *>(d_emb), ef,
                      as_stream(stream)));
    return BM3D_B200_OK;
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
