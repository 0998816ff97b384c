/*
 * Test infrastructure only (the oracle): C restatement of the learned block
 * matcher of vapoursynth-bm3dcuda_b200/csrc/bm3d_learned.cu, which has no
 * counterpart in the reference. It follows the project's definition step for
 * step (exact integer distances of the 8-bit embeddings, cells ranked with
 * the reference's insertion rule, exact block distances with the reference's
 * FP32 arithmetic, compute_distance in cpu_source/source.cpp:122-136), so the
 * CUDA matcher's lists must equal these exactly for the same embeddings.
 * Blocks that fall back get this restatement's exhaustive search
 * (block_matching_temporal, cpu_source/source.cpp:220-321).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define REAL float
#define SFX _lf32
#define RFMA(a, b, c) fmaf((a), (b), (c))
#define RABS(a) fabsf(a)
#define RSQRT(a) sqrtf(a)
#define AGG_DIVIDE(a, b) ((a) * (1.0f / (b)))
#include "bm3d_port_impl.h"

static void cell_embedding(uint8_t out[16], const uint8_t *emb, int w2, int gx, int gy) {
    memcpy(out, emb + ((size_t)(gy + 2) * w2 + (gx + 2)) * 16, 16);
}

/* Exact integer squared distance of two 8-bit embeddings, as a float (exact:
 * at most 16 * 255^2 < 2^24). */
static float emb_dist(const uint8_t a[16], const uint8_t b[16]) {
    uint32_t acc = 0;
    for (int c = 0; c < 16; ++c) {
        int d = (int)a[c] - (int)b[c];
        acc += (uint32_t)(d * d);
    }
    return (float)acc;
}

typedef struct {
    int l, r, t, b;
} Box;

/* Window of a stage around centre position (px, py); temporal centres are
 * kept within the stage's reach m = bm_range + t * ps_range of the block. */
static Box stage_box(int st, int x, int y, int m, int range, int px, int py, int width,
                     int height) {
    int cx = x, cy = y;
    if (st > 0) {
        cx = px < x - m + range ? x - m + range : px;
        cx = cx > x + m - range ? x + m - range : cx;
        cy = py < y - m + range ? y - m + range : py;
        cy = cy > y + m - range ? y + m - range : cy;
    }
    Box b;
    b.l = cx - range > 0 ? cx - range : 0;
    b.r = cx + range < width - 8 ? cx + range : width - 8;
    b.t = cy - range > 0 ? cy - range : 0;
    b.b = cy + range < height - 8 ? cy + range : height - 8;
    return b;
}

static int in_cells(Box b, int gx, int gy) {
    return gx >= (b.l >> 1) && gx <= (b.r >> 1) && gy >= (b.t >> 1) && gy <= (b.b >> 1);
}

/* One stage's learned search of frame z into the per-frame list f*. */
static void learned_stage(float fe[8], int fx[8], int fy[8], int fz[8], int st, int z, int x,
                          int y, int m, int range, int nwin, const int *lx, const int *ly,
                          int keep, const uint8_t er[16], const uint8_t *emb, int w2,
                          const float ref[8][8], const float *plane, int stride, int width,
                          int height) {
    float ce[8];
    int cx[8], cy[8], cw[8];
    for (int i = 0; i < 8; ++i) {
        ce[i] = FLT_MAX;
        cx[i] = cy[i] = cw[i] = 0;
    }
    Box boxes[8];
    for (int i = 0; i < nwin; ++i)
        boxes[i] = stage_box(st, x, y, m, range, st > 0 ? lx[i] : 0, st > 0 ? ly[i] : 0, width,
                             height);
    for (int i = 0; i < nwin; ++i) {
        Box bi = boxes[i];
        for (int gy = bi.t >> 1; gy <= (bi.b >> 1); ++gy)
            for (int gx = bi.l >> 1; gx <= (bi.r >> 1); ++gx) {
                int seen = 0;
                for (int j = 0; j < i; ++j) seen |= in_cells(boxes[j], gx, gy);
                if (seen) continue;
                uint8_t ec[16];
                cell_embedding(ec, emb, w2, gx, gy);
                float d = emb_dist(er, ec);
                if (d < ce[keep - 1]) list_insert_lf32(ce, cx, cy, cw, d, gx, gy, i);
            }
    }
    for (int k = 0; k < keep; ++k) {
        if (!(ce[k] < FLT_MAX)) break;
        Box bw = boxes[cw[k]];
        for (int dv = 0; dv < 2; ++dv)
            for (int du = 0; du < 2; ++du) {
                int u = 2 * cx[k] + du, v = 2 * cy[k] + dv;
                if (u < bw.l || u > bw.r || v < bw.t || v > bw.b) continue;
                float e = ssd_lf32(ref, &plane[(size_t)v * stride + u], stride);
                if (e < fe[7]) list_insert_lf32(fe, fx, fy, fz, e, u, v, z);
            }
    }
}

/* frames: 2r+1 planes [height][stride]; embs: their 8-bit embeddings
 * [height/2][width/2][16]. match_out: [nblocks][8][3] (x, y, z);
 * fallback_out (optional): [nblocks] flags. Returns the block count. */
int port_learned_match(const float *const *frames, const uint8_t *const *embs, int width,
                       int height, int stride, int block_step, int bm_range, int radius,
                       int ps_num, int ps_range, int cells_s, int cells_t, float fallback_ssd,
                       int *match_out, int *fallback_out) {
    if (width < 16 || height < 16 || stride < width || block_step < 1 || block_step > 8 ||
        bm_range < 1 || radius < 0 || ps_num < 1 || ps_num > 8 || ps_range < 1 || cells_s < 1 ||
        cells_s > 8 || cells_t < 1 || cells_t > 8)
        return -1;
    const int w2 = width / 2;
    const int center = radius;
    int nb = 0;
    for (int by = 0; by < height - 8 + block_step; by += block_step) {
        for (int bx = 0; bx < width - 8 + block_step; bx += block_step, ++nb) {
            const int x = bx < width - 8 ? bx : width - 8;
            const int y = by < height - 8 ? by : height - 8;
            float ref[8][8];
            for (int r = 0; r < 8; ++r)
                for (int c = 0; c < 8; ++c)
                    ref[r][c] = frames[center][(size_t)(y + r) * stride + x + c];
            uint8_t er[16];
            cell_embedding(er, embs[center], w2, x >> 1, y >> 1);
            float le[8];
            int ix[8], iy[8], iz[8];
            for (int i = 0; i < 8; ++i) {
                le[i] = FLT_MAX;
                ix[i] = x;
                iy[i] = y;
                iz[i] = center;
            }
            /* stage 0 */
            learned_stage(le, ix, iy, iz, 0, center, x, y, bm_range, bm_range, 1, NULL, NULL,
                          cells_s, er, embs[center], w2, ref, frames[center], stride, width,
                          height);
            int sx[8], sy[8];
            for (int i = 0; i < 8; ++i) {
                sx[i] = ix[i];
                sy[i] = iy[i];
            }
            for (int dir = -1; dir <= 1; dir += 2) {
                int lx[8], ly[8];
                memcpy(lx, sx, sizeof lx);
                memcpy(ly, sy, sizeof ly);
                for (int t = 1; t <= radius; ++t) {
                    const int z = center + dir * t;
                    const int m = bm_range + t * ps_range;
                    float fe[8];
                    int fx[8], fy[8], fz[8];
                    for (int i = 0; i < 8; ++i) {
                        fe[i] = FLT_MAX;
                        fx[i] = fy[i] = 0;
                        fz[i] = z;
                    }
                    learned_stage(fe, fx, fy, fz, 1, z, x, y, m, ps_range, ps_num, lx, ly,
                                  cells_t, er, embs[z], w2, ref, frames[z], stride, width,
                                  height);
                    for (int i = 0; i < ps_num; ++i)
                        if (fe[i] < le[7]) list_insert_lf32(le, ix, iy, iz, fe[i], fx[i], fy[i], z);
                    memcpy(lx, fx, sizeof lx);
                    memcpy(ly, fy, sizeof ly);
                }
            }
            int fell = 0;
            if (fallback_ssd > 0.0f) {
                float best = FLT_MAX;
                for (int i = 0; i < 8; ++i)
                    if (!(ix[i] == x && iy[i] == y && iz[i] == center) && le[i] < best)
                        best = le[i];
                fell = !(best <= fallback_ssd);
            }
            if (fell) {
                for (int i = 0; i < 8; ++i) {
                    le[i] = FLT_MAX;
                    ix[i] = x;
                    iy[i] = y;
                    iz[i] = center;
                }
                if (radius == 0)
                    block_matching_lf32(le, ix, iy, iz, 0, ref, frames[0], stride, width, height,
                                        bm_range, x, y, 0);
                else
                    block_matching_temporal_lf32(le, ix, iy, iz, ref, frames, stride, width,
                                                 height, bm_range, x, y, radius, ps_num,
                                                 ps_range, 0);
            }
            insert_center_lf32(ix, iy, iz, x, y, center);
            for (int i = 0; i < 8; ++i) {
                match_out[((size_t)nb * 8 + i) * 3 + 0] = ix[i];
                match_out[((size_t)nb * 8 + i) * 3 + 1] = iy[i];
                match_out[((size_t)nb * 8 + i) * 3 + 2] = iz[i];
            }
            if (fallback_out) fallback_out[nb] = fell;
        }
    }
    return nb;
}

/* Reference values of the proposer's inference arithmetic for one frame:
 * the 2x2 means, BF16-rounded operands, exact (double) sums, BF16-rounded
 * activations after bias + ReLU, and the final embedding before its FP16
 * rounding. params: the 4800 FP32 parameters (see bm3d_b200.h). out:
 * [height/2][width/2][16] floats. */
static float bf16_round(float v) {
    uint32_t b;
    memcpy(&b, &v, 4);
    if ((b & 0x7f800000u) == 0x7f800000u) return v;
    b += 0x7fffu + ((b >> 16) & 1u); /* round to nearest even */
    b &= 0xffff0000u;
    memcpy(&v, &b, 4);
    return v;
}

void port_proposer_embed_bf16(const float *plane, int width, int height, int stride,
                              const float *params, float *out) {
    const int w2 = width / 2, h2 = height / 2;
    const size_t np = (size_t)w2 * h2;
    float *x0 = malloc(np * sizeof(float));
    float *a1 = malloc(np * 16 * sizeof(float));
    float *a2 = malloc(np * 16 * sizeof(float));
    float wq[4800];
    for (int i = 0; i < 4800; ++i) wq[i] = bf16_round(params[i]);
    for (int y = 0; y < h2; ++y)
        for (int x = 0; x < w2; ++x) {
            const float *s = plane + (size_t)(2 * y) * stride + 2 * x;
            x0[(size_t)y * w2 + x] = bf16_round(0.25f * ((s[0] + s[1]) + (s[stride] + s[stride + 1])));
        }
    const int offw[3] = {0, 160, 2480}, offb[3] = {144, 2464, 4784}, cin[3] = {1, 16, 16};
    const float *in = x0;
    float *outs[3] = {a1, a2, out};
    for (int layer = 0; layer < 3; ++layer) {
        float *o = outs[layer];
        for (int y = 0; y < h2; ++y)
            for (int x = 0; x < w2; ++x)
                for (int co = 0; co < 16; ++co) {
                    double acc = 0.0;
                    for (int dy = 0; dy < 3; ++dy)
                        for (int dx = 0; dx < 3; ++dx) {
                            int yy = y + dy - 1, xx = x + dx - 1;
                            if (yy < 0 || yy >= h2 || xx < 0 || xx >= w2) continue;
                            for (int ci = 0; ci < cin[layer]; ++ci)
                                acc += (double)in[((size_t)yy * w2 + xx) * cin[layer] + ci] *
                                       (double)wq[offw[layer] +
                                                  ((dy * 3 + dx) * cin[layer] + ci) * 16 + co];
                        }
                    float v = (float)acc + params[offb[layer] + co];
                    if (layer < 2) v = bf16_round(v > 0.0f ? v : 0.0f);
                    o[((size_t)y * w2 + x) * 16 + co] = v;
                }
        in = o;
    }
    free(x0);
    free(a1);
    free(a2);
}
