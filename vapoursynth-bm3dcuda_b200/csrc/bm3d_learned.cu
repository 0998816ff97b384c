// Learned block matching for BM3D / V-BM3D on sm_100a (no counterpart in the
// reference; the exhaustive search it prunes is source/kernel.cu:432-647).
//
// Same work layout and stages as the exhaustive matcher (bm3d_match.cu): a
// thread per reference block, a warp per 4 x 8 blocks, stage 0 the centre
// frame, stages 1..2r the neighbour frames in the reference's order, each
// stage's pixel region staged in shared memory. What changes is which
// candidates a stage scores exactly:
//
//   * candidate cells: the cells (u/2, v/2) of the stage's search windows -
//     the bm_range window in stage 0, the union of the ps_num predictive
//     windows in a temporal stage (a cell is taken once, under the first
//     window whose cell rectangle holds it);
//   * ranking: squared distance between the 8-bit embeddings of the
//     reference block's own cell (centre frame) and the candidate cell (stage
//     frame), exact in integers (per-byte absolute differences and 4-way dot
//     products); the best cells_s (stage 0) or cells_t (temporal) cells are
//     kept, ties to the earlier cell (window order, then row-major);
//   * exact scoring: the (up to) four block origins of every kept cell, in
//     ranking order and row-major within a cell, that lie in the window the
//     cell was taken under, with the reference's block distance and list
//     insertion (so every distance is bit-identical to the exhaustive one).
//
// The per-frame lists are merged into the block's list exactly as in the
// exhaustive search (first ps_num entries of each frame), and the centre
// block is inserted at the end. A block whose best match other than itself
// is farther than fallback_ssd is appended to a list; the fallback kernel
// re-runs the exhaustive search for exactly those blocks and overwrites
// their lists with the exhaustive result.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "bm3d_device.cuh"
#include "bm3d_internal.h"

namespace bm3d {

namespace {

// Search window i of a stage: the clamped candidate box (image coordinates).
struct Box {
    int l, r, t, b;
};

__device__ __forceinline__ Box stage_box(const MatchParams &p, int st, int x, int y, int m,
                                         int range, int center_pos) {
    int cx = x, cy = y;
    if (st > 0) {
        cx = min(max(pos_x(center_pos), x - m + range), x + m - range);
        cy = min(max(pos_y(center_pos), y - m + range), y + m - range);
    }
    return Box{max(cx - range, 0), min(cx + range, p.width - 8), max(cy - range, 0),
               min(cy + range, p.height - 8)};
}

__device__ __forceinline__ bool in_cells(const Box &bx, int gx, int gy) {
    return gx >= (bx.l >> 1) && gx <= (bx.r >> 1) && gy >= (bx.t >> 1) && gy <= (bx.b >> 1);
}

// Squared distance of two cells' embeddings (16 unsigned 8-bit channels):
// per-byte absolute differences, then four 4-way dot products. Exact.
__device__ __forceinline__ unsigned emb_dist(const uint4 a, const uint4 b) {
    unsigned d = __vabsdiffu4(a.x, b.x);
    unsigned acc = __dp4a(d, d, 0u);
    d = __vabsdiffu4(a.y, b.y);
    acc = __dp4a(d, d, acc);
    d = __vabsdiffu4(a.z, b.z);
    acc = __dp4a(d, d, acc);
    d = __vabsdiffu4(a.w, b.w);
    return __dp4a(d, d, acc);
}

__device__ __forceinline__ const uint4 *cell_ptr(const uint4 *emb, int w2, int gx, int gy) {
    return emb + ((size_t)(gy + 2) * w2 + (gx + 2));
}

// Cell keys: key = embedding distance << 12 | ordinal, the ordinal numbering
// a stage's candidate cells in window order, then row-major within the
// window's cell rectangle (distances are below 2^20: 16 channels of at most
// 255^2; ordinals below 4096, checked on the host). Ascending keys are the
// ranking order - smaller distance first, ties to the earlier cell - so the
// best K cells are kept by a branchless min/max insertion network, the same
// for every lane of a warp.
constexpr int kOrdinalBits = 12;
constexpr unsigned kNoKey = 0xffffffffu;

template <int K>
__device__ __forceinline__ void key_insert(unsigned (&keys)[K], unsigned key) {
#pragma unroll
    for (int i = 0; i < K; ++i) {
        const unsigned lo = min(keys[i], key);
        key = max(keys[i], key);
        keys[i] = lo;
    }
}

// Cell rectangle of a search box.
struct CellRect {
    int gx0, gx1, gy0, gy1;
};

__device__ __forceinline__ CellRect cell_rect(const Box &b) {
    return CellRect{b.l >> 1, b.r >> 1, b.t >> 1, b.b >> 1};
}

// Ranks the cells of search window i of a stage into `keys`, skipping cells
// that an earlier window's cell rectangle already held (b0: window 0's box;
// windows 1 .. i-1 are recomputed from their centres in `last`). ord0: the
// ordinal of the window's first cell. The window's cell rows are walked one
// by one, four cells per iteration with their loads issued first; a skipped
// cell inserts the empty key (a no-op of the min/max network), so the walk
// has no divergent branch.
template <int K>
__device__ __forceinline__ void rank_cells(unsigned (&keys)[K], const uint4 er,
                                           const uint4 *__restrict__ emb, int w2, const Box &bi,
                                           unsigned ord0, int i, const Box &b0,
                                           const MatchParams &p, int st, int x, int y, int m,
                                           int range, const int (&last)[8]) {
    const CellRect cr = cell_rect(bi);
    const CellRect c0 = cell_rect(b0);
    auto seen_earlier = [&](int gx, int gy) {
        if (i == 0) return false;
        bool seen = gx >= c0.gx0 && gx <= c0.gx1 && gy >= c0.gy0 && gy <= c0.gy1;
        for (int j = 1; j < i; ++j)
            seen |= in_cells(stage_box(p, st, x, y, m, range, pick(last, j)), gx, gy);
        return seen;
    };
    const int ncol = cr.gx1 - cr.gx0 + 1;
    unsigned o = ord0;
    for (int gy = cr.gy0; gy <= cr.gy1; ++gy, o += (unsigned)ncol) {
        const uint4 *row = cell_ptr(emb, w2, cr.gx0, gy);
        int k = 0;
        for (; k + 3 < ncol; k += 4) {
            uint4 e[4];
#pragma unroll
            for (int j = 0; j < 4; ++j) e[j] = __ldg(row + k + j);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const unsigned key = (emb_dist(er, e[j]) << kOrdinalBits) | (o + k + j);
                key_insert(keys, seen_earlier(cr.gx0 + k + j, gy) ? kNoKey : key);
            }
        }
        for (; k < ncol; ++k) {
            const unsigned key = (emb_dist(er, __ldg(row + k)) << kOrdinalBits) | (o + k);
            key_insert(keys, seen_earlier(cr.gx0 + k, gy) ? kNoKey : key);
        }
    }
}

template <int K>
__device__ void learned_tile(const MatchParams &p, const LearnedParams &lp, int tile_x,
                             int tile_y, int win, float *tile) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nbx_cta = (blockDim.x >> 5) * 4;
    const int bx = tile_x * nbx_cta + warp * 4 + (lane & 3);
    const int by = tile_y * 8 + (lane >> 2);
    const bool active = bx < p.nbx && by < p.nby;

    const int x = min(bx * p.block_step, p.width - 8);
    const int y = min(by * p.block_step, p.height - 8);

    const int bx_first = tile_x * nbx_cta;
    const int bx_last = min(bx_first + nbx_cta - 1, p.nbx - 1);
    const int by_first = tile_y * 8;
    const int by_last = min(by_first + 7, p.nby - 1);
    const int xa = min(bx_first * p.block_step, p.width - 8);
    const int xb = min(bx_last * p.block_step, p.width - 8);
    const int ya = min(by_first * p.block_step, p.height - 8);
    const int yb = min(by_last * p.block_step, p.height - 8);

    const int r = p.radius;
    const int center = r;
    const int tw = 2 * r + 1;
    const float *const *frames = p.frames + (size_t)win * tw;
    const uint4 *const *embs = reinterpret_cast<const uint4 *const *>(lp.embs) + (size_t)win * tw;

    f32x2 refp[4][8];
    uint4 er = make_uint4(0, 0, 0, 0);
    List8 list;
    list_init(list, FLT_MAX, pack_pos(x, y, center));
    int *center_pos = reinterpret_cast<int *>(tile + (size_t)p.pitch * p.tile_rows) + threadIdx.x;
    int last[8];

    for (int st = 0; st <= 2 * r; ++st) {
        const int t = st <= r ? st : st - r;
        const int z = st == 0 ? center : (st <= r ? center - t : center + t);
        const int m = p.bm_range + t * p.ps_range;
        // one extra column / row on each side: a kept cell may start one
        // pixel before its window and its strip reads one column past it
        const int tx0 = xa - m - 1, ty0 = ya - m - 1;
        const int twid = xb - xa + 2 * m + 10;
        const int thei = yb - ya + 2 * m + 10;
        if (st > 0) __syncthreads();
        load_tile(tile, frames[z], p.width, p.height, p.stride, tx0, ty0, twid, thei, p.pitch);
        __syncthreads();
        if (st == 0) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    refp[q][c] = pack2(tile[skewed(y - ty0 + 2 * q, x - tx0 + c, p.pitch)],
                                       tile[skewed(y - ty0 + 2 * q + 1, x - tx0 + c, p.pitch)]);
            if (active) er = __ldg(cell_ptr(embs[center], lp.w2, x >> 1, y >> 1));
        }
        if (!active) continue;
        if (st == r + 1) {
#pragma unroll
            for (int i = 0; i < 8; ++i) last[i] = center_pos[i * blockDim.x];
        }
        const int range = st == 0 ? p.bm_range : p.ps_range;
        const int nwin = st == 0 ? 1 : p.ps_num;
        const int keep = st == 0 ? lp.cells_s : lp.cells_t;
        const uint4 *emb = embs[z];

        // rank the candidate cells
        unsigned keys[K];
#pragma unroll
        for (int k = 0; k < K; ++k) keys[k] = kNoKey;
        const Box b0 = stage_box(p, st, x, y, m, range, st > 0 ? last[0] : 0);
        {
            unsigned ord0 = 0;
            for (int i = 0; i < nwin; ++i) {
                const Box bi = i == 0 ? b0 : stage_box(p, st, x, y, m, range, pick(last, i));
                rank_cells(keys, er, emb, lp.w2, bi, ord0, i, b0, p, st, x, y, m, range, last);
                const CellRect cr = cell_rect(bi);
                ord0 += (unsigned)((cr.gx1 - cr.gx0 + 1) * (cr.gy1 - cr.gy0 + 1));
            }
        }

        // exact distances of the kept cells' block origins, in ranking order
        List8 fl;
        list_init(fl, FLT_MAX, st == 0 ? pack_pos(x, y, center) : pack_pos(0, 0, z));
        for (int k = 0; k < keep; ++k) {
            const unsigned key = pick(keys, k);
            if (key == kNoKey) break;
            // window and cell of the ordinal
            int ord = (int)(key & ((1u << kOrdinalBits) - 1u));
            int wi = 0;
            Box bw = b0;
            CellRect cr = cell_rect(b0);
            for (;;) {
                const int n = (cr.gx1 - cr.gx0 + 1) * (cr.gy1 - cr.gy0 + 1);
                if (ord < n || wi + 1 >= nwin) break;
                ord -= n;
                ++wi;
                bw = stage_box(p, st, x, y, m, range, pick(last, wi));
                cr = cell_rect(bw);
            }
            const int ncol = cr.gx1 - cr.gx0 + 1;
            const int gy = ord / ncol;
            const int u = 2 * (cr.gx0 + ord - gy * ncol), v = 2 * (cr.gy0 + gy);
#pragma unroll
            for (int dv = 0; dv < 2; ++dv) {
                int roff[8];
#pragma unroll
                for (int rr = 0; rr < 8; ++rr) roff[rr] = skewed(v + dv - ty0 + rr, u - tx0, p.pitch);
                float err[2];
                ssd_strip<2>(refp, tile, roff, err);
#pragma unroll
                for (int du = 0; du < 2; ++du) {
                    const int cu = u + du, cv = v + dv;
                    if (cu >= bw.l && cu <= bw.r && cv >= bw.t && cv <= bw.b &&
                        err[du] < fl.e[7])
                        list_insert(fl, err[du], pack_pos(cu, cv, z));
                }
            }
        }

        if (st == 0) {
            list = fl;
#pragma unroll
            for (int i = 0; i < 8; ++i) center_pos[i * blockDim.x] = last[i] = fl.p[i];
        } else {
            for (int i = 0; i < p.ps_num; ++i) {
                const float e = pick(fl.e, i);
                if (e < list.e[7]) list_insert(list, e, pick(fl.p, i));
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) last[i] = fl.p[i];
        }
    }

    if (!active) return;

    const int cpos = pack_pos(x, y, center);
    const int blk = by * p.nbx + bx;
    if (lp.fallback_ssd > 0.0f) {
        float best = FLT_MAX;
#pragma unroll
        for (int i = 0; i < 8; ++i)
            if (list.p[i] != cpos) best = fminf(best, list.e[i]);
        if (!(best <= lp.fallback_ssd)) {
            const unsigned slot = atomicAdd(lp.fallback_count, 1u);
            if (slot < lp.fallback_capacity)
                lp.fallback[slot] = (unsigned)win * (unsigned)(p.nbx * p.nby) + (unsigned)blk;
        }
    }

    bool found = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) found |= list.p[i] == cpos;
    if (!found) {
#pragma unroll
        for (int i = 7; i > 0; --i) list.p[i] = list.p[i - 1];
        list.p[0] = cpos;
    }
    int4 *out = reinterpret_cast<int4 *>(p.matches + ((size_t)win * p.nbx * p.nby + blk) * 8);
    out[0] = make_int4(list.p[0], list.p[1], list.p[2], list.p[3]);
    out[1] = make_int4(list.p[4], list.p[5], list.p[6], list.p[7]);
}

// CTAs are taken row-band-major across windows: consecutive CTAs cover one
// band of tile rows in every window before the next band, so the CTAs that
// run together read the same rows of the (shared) frames and embeddings and
// those stay in L2 (window-major order re-reads them from DRAM).
template <int K>
__global__ void __launch_bounds__(128, 3) learned_match_kernel(MatchParams p, LearnedParams lp) {
    extern __shared__ float tile[];
    const unsigned id = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const unsigned rest = id / gridDim.x;
    learned_tile<K>(p, lp, (int)(id % gridDim.x), (int)(rest / gridDim.z),
                    p.win0 + (int)(rest % gridDim.z), tile);
}

// ---------------------------------------------------------------------------
// Exhaustive re-search of listed blocks, one warp per block. The lanes
// compute the distances of a stage's candidates (reference scan order,
// windows in order, overlapping windows scanned twice as the reference does)
// into shared memory; lane 0 then feeds them to the lists in that order. The
// distances come from the same strip routine as the exhaustive matcher, so
// the result is the exhaustive matcher's list for that block.
// ---------------------------------------------------------------------------
constexpr int kFallbackWarps = 4;

__global__ void __launch_bounds__(32 * kFallbackWarps)
    fallback_kernel(MatchParams p, const unsigned *__restrict__ entries,
                    const unsigned *__restrict__ count, int buf_floats, int region_floats) {
    extern __shared__ float fbuf[];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    float *errs = fbuf + (size_t)warp * (buf_floats + region_floats);
    float *region = errs + buf_floats;  // the current window's pixels (+7 rows, +7 columns)
    const unsigned n = *count;
    const int nblk = p.nbx * p.nby;
    const int r = p.radius, center = r, tw = 2 * r + 1;
    for (unsigned ei = blockIdx.x * kFallbackWarps + warp; ei < n;
         ei += gridDim.x * kFallbackWarps) {
        const unsigned e = entries[ei];
        const int win = (int)(e / (unsigned)nblk), blk = (int)(e % (unsigned)nblk);
        const int bx = blk % p.nbx, by = blk / p.nbx;
        const int x = min(bx * p.block_step, p.width - 8);
        const int y = min(by * p.block_step, p.height - 8);
        const float *const *frames = p.frames + (size_t)win * tw;
        f32x2 refp[4][8];
        {
            const float *c = frames[center] + (size_t)y * p.stride + x;
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    refp[q][j] = pack2(__ldg(c + (2 * q) * p.stride + j),
                                       __ldg(c + (2 * q + 1) * p.stride + j));
        }
        List8 list;  // meaningful in lane 0
        list_init(list, FLT_MAX, pack_pos(x, y, center));
        int last[8], spos[8];  // window centres (all lanes); spatial list positions
        for (int st = 0; st <= 2 * r; ++st) {
            const int t = st <= r ? st : st - r;
            const int z = st == 0 ? center : (st <= r ? center - t : center + t);
            const int m = p.bm_range + t * p.ps_range;
            const int range = st == 0 ? p.bm_range : p.ps_range;
            const int nwin = st == 0 ? 1 : p.ps_num;
            if (st == r + 1) {
                // the +1 direction starts again from the spatial list
#pragma unroll
                for (int i = 0; i < 8; ++i) last[i] = spos[i];
            }
            const float *plane = frames[z];
            // distances of all candidates of the stage, in scan order
            int base = 0;
            for (int i = 0; i < nwin; ++i) {
                const Box b = stage_box(p, st, x, y, m, range, st > 0 ? pick(last, i) : 0);
                const int cw = b.r - b.l + 1, nc = cw * (b.b - b.t + 1);
                // stage the window's pixel region once (it lies inside the plane:
                // b.r + 7 <= width - 1, b.b + 7 <= height - 1); without room for it
                // (very large ranges) the distances read the plane directly
                const bool staged = region_floats > 0;
                const int rp = staged ? cw + 7 : p.stride;
                const float *src = staged ? region : plane + (size_t)b.t * p.stride + b.l;
                if (staged) {
                    const int rn = rp * (b.b - b.t + 8);
                    __syncwarp();
                    for (int k = lane; k < rn; k += 32)
                        region[k] =
                            __ldg(plane + (size_t)(b.t + k / rp) * p.stride + b.l + k % rp);
                    __syncwarp();
                }
                for (int c = lane; c < nc; c += 32) {
                    const int cu = c % cw, cv = c / cw;
                    int roff[8];
#pragma unroll
                    for (int rr = 0; rr < 8; ++rr) roff[rr] = (cv + rr) * rp + cu;
                    float err[1];
                    ssd_strip<1>(refp, src, roff, err);
                    errs[base + c] = err[0];
                }
                base += nc;
            }
            __syncwarp();
            // The stage's list: inserting every candidate in scan order with a
            // strict < keeps the 8 smallest by (distance, scan index). Each lane
            // keeps that list for its candidates o = lane, lane + 32, ...; eight
            // warp arg-min rounds over the lanes' heads then give the same list.
            List8 ll;
            list_init(ll, FLT_MAX, 0x7fffffff);
            for (int o = lane; o < base; o += 32) {
                const float ev = errs[o];
                if (ev < ll.e[7]) list_insert(ll, ev, o);
            }
            List8 fl;
            list_init(fl, FLT_MAX, st == 0 ? pack_pos(x, y, center) : pack_pos(0, 0, z));
            int head = 0;
#pragma unroll
            for (int k = 0; k < 8; ++k) {
                const bool have = head < 8;
                const int mine = have ? pick(ll.p, head) : 0x7fffffff;
                float e = have ? pick(ll.e, head) : FLT_MAX;
                int o = mine;
#pragma unroll
                for (int off = 16; off > 0; off >>= 1) {
                    const float oe = __shfl_xor_sync(0xffffffffu, e, off);
                    const int oo = __shfl_xor_sync(0xffffffffu, o, off);
                    if (oe < e || (oe == e && oo < o)) {
                        e = oe;
                        o = oo;
                    }
                }
                if (o == 0x7fffffff) break;  // fewer than 8 candidates (same in all lanes)
                if (mine == o) ++head;
                // the position of scan index o
                int rem = o, pos = 0;
                for (int i = 0; i < nwin; ++i) {
                    const Box b = stage_box(p, st, x, y, m, range, st > 0 ? pick(last, i) : 0);
                    const int cw = b.r - b.l + 1, nc = cw * (b.b - b.t + 1);
                    if (rem < nc) {
                        pos = pack_pos(b.l + rem % cw, b.t + rem / cw, z);
                        break;
                    }
                    rem -= nc;
                }
                fl.e[k] = e;
                fl.p[k] = pos;
            }
            if (lane == 0) {
                if (st == 0) {
                    list = fl;
                } else {
                    for (int i = 0; i < p.ps_num; ++i) {
                        const float ev = pick(fl.e, i);
                        if (ev < list.e[7]) list_insert(list, ev, pick(fl.p, i));
                    }
                }
            }
            __syncwarp();
            // the next stage searches around this frame's list
#pragma unroll
            for (int i = 0; i < 8; ++i) last[i] = __shfl_sync(0xffffffffu, fl.p[i], 0);
            if (st == 0) {
#pragma unroll
                for (int i = 0; i < 8; ++i) spos[i] = last[i];
            }
        }
        if (lane == 0) {
            const int cpos = pack_pos(x, y, center);
            bool found = false;
#pragma unroll
            for (int i = 0; i < 8; ++i) found |= list.p[i] == cpos;
            if (!found) {
#pragma unroll
                for (int i = 7; i > 0; --i) list.p[i] = list.p[i - 1];
                list.p[0] = cpos;
            }
            int4 *out =
                reinterpret_cast<int4 *>(p.matches + ((size_t)win * nblk + blk) * 8);
            out[0] = make_int4(list.p[0], list.p[1], list.p[2], list.p[3]);
            out[1] = make_int4(list.p[4], list.p[5], list.p[6], list.p[7]);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Final-stage lists from the basic stage's: every block's 8 positions of the
// basic stage are scored again on the final stage's matching planes (the
// basic estimate) and sorted by that distance, ties keeping the basic order.
// A warp takes 4 blocks at once, 8 lanes per block, lane = column c: each
// lane loads its column of the reference block and of all 8 candidates (72
// independent loads in flight), sums its column's squared differences in the
// reference's two chains (even rows, odd rows, as a packed pair), and the 8
// column sums are added by the xor tree 1, 2, 4 inside the 8 lanes - the
// reference's block distance (source/kernel.cu:455-471), bit for bit.
// ---------------------------------------------------------------------------
constexpr int kRescoreWarps = 8;

__global__ void __launch_bounds__(32 * kRescoreWarps)
    rescore_kernel(MatchParams p, int nwin) {
    const int lane = threadIdx.x & 31;
    const int g = lane >> 3, c = lane & 7;
    const int nblk = p.nbx * p.nby;
    const int tw = 2 * p.radius + 1;
    const long long total = (long long)nwin * nblk;
    const long long item = ((long long)blockIdx.x * kRescoreWarps + (threadIdx.x >> 5)) * 4 + g;
    const bool active = item < total;
    const long long it = active ? item : total - 1;
    const int win = p.win0 + (int)(it / nblk);
    const int blk = (int)(it % nblk);
    const int bx = blk % p.nbx, by = blk / p.nbx;
    const int x = min(bx * p.block_step, p.width - 8);
    const int y = min(by * p.block_step, p.height - 8);
    const float *const *frames = p.frames + (size_t)win * tw;
    int *lst = p.matches + ((size_t)win * nblk + blk) * 8;
    int pos[8];
    {
        const int4 *m = reinterpret_cast<const int4 *>(lst);
        const int4 a0 = __ldg(m), a1 = __ldg(m + 1);
        pos[0] = a0.x; pos[1] = a0.y; pos[2] = a0.z; pos[3] = a0.w;
        pos[4] = a1.x; pos[5] = a1.y; pos[6] = a1.z; pos[7] = a1.w;
    }
    f32x2 ref[4];
    {
        const float *rb = frames[p.radius] + (size_t)y * p.stride + x + c;
#pragma unroll
        for (int q = 0; q < 4; ++q)
            ref[q] = pack2(__ldg(rb + (size_t)(2 * q) * p.stride),
                           __ldg(rb + (size_t)(2 * q + 1) * p.stride));
    }
    float px[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float *cb =
            frames[pos_z(pos[i])] + (size_t)pos_y(pos[i]) * p.stride + pos_x(pos[i]) + c;
#pragma unroll
        for (int r = 0; r < 8; ++r) px[i][r] = __ldg(cb + (size_t)r * p.stride);
    }
    List8 l;
    list_init(l, FLT_MAX, 0);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        f32x2 e = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const f32x2 d = sub2(ref[q], pack2(px[i][2 * q], px[i][2 * q + 1]));
            e = q == 0 ? mul2(d, d) : fma2(d, d, e);
        }
        float e0, e1;
        unpack2(e, e0, e1);
        float sd = __fadd_rn(e0, e1);
        sd = __fadd_rn(sd, __shfl_xor_sync(0xffffffffu, sd, 1));
        sd = __fadd_rn(sd, __shfl_xor_sync(0xffffffffu, sd, 2));
        sd = __fadd_rn(sd, __shfl_xor_sync(0xffffffffu, sd, 4));
        list_insert(l, sd, pos[i]);  // basic order: ties keep the earlier entry
    }
    if (active && c == 0) {
        int4 *out = reinterpret_cast<int4 *>(lst);
        out[0] = make_int4(l.p[0], l.p[1], l.p[2], l.p[3]);
        out[1] = make_int4(l.p[4], l.p[5], l.p[6], l.p[7]);
    }
}

}  // namespace

cudaError_t launch_rescore(const MatchParams &p, int nwin, cudaStream_t stream) {
    const long long total = (long long)nwin * p.nbx * p.nby;
    if (total <= 0) return cudaSuccess;
    const long long per_cta = 4LL * kRescoreWarps;  // 4 blocks per warp
    const long long grid = (total + per_cta - 1) / per_cta;
    if (grid > 0x7fffffffLL) return cudaErrorInvalidValue;
    rescore_kernel<<<(unsigned)grid, 32 * kRescoreWarps, 0, stream>>>(p, nwin);
    return cudaGetLastError();
}

MatchGeometry learned_geometry(int width, int height, int block_step, int bm_range, int radius,
                               int ps_range) {
    MatchGeometry g{};
    g.nbx = (width - 8 + block_step - 1) / block_step + 1;
    g.nby = (height - 8 + block_step - 1) / block_step + 1;
    const int mmax = bm_range + radius * ps_range;
    for (int wx = 4; wx >= 1; wx /= 2) {
        const int tw = (4 * wx - 1) * block_step + 2 * mmax + 10;
        const int th = 7 * block_step + 2 * mmax + 10;
        g.wx = wx;
        g.pitch = tw + 8;
        g.tile_rows = th;
        g.smem = (size_t)g.pitch * th * sizeof(float) + 8 * 32 * wx * sizeof(int);
        if (g.smem <= 72 * 1024) break;
    }
    g.ks = g.kt = 2;
    return g;
}

bool learned_ordinals_fit(int bm_range, int ps_num, int ps_range) {
    // a window of half-range R spans at most R + 1 cells per axis
    const long long sp = (long long)(bm_range + 2) * (bm_range + 2);
    const long long tp = (long long)ps_num * (ps_range + 2) * (ps_range + 2);
    return sp <= (1 << kOrdinalBits) && tp <= (1 << kOrdinalBits);
}

template <int K>
cudaError_t launch_learned_k(const MatchParams &p, const LearnedParams &lp, const MatchGeometry &g,
                             int nwin, cudaStream_t stream) {
    static int configured[64] = {0};
    cudaError_t e = raise_smem_limit(configured, (const void *)learned_match_kernel<K>, g.smem);
    if (e != cudaSuccess) return e;
    dim3 block(32 * g.wx);
    dim3 grid((p.nbx + 4 * g.wx - 1) / (4 * g.wx), (p.nby + 7) / 8, nwin);
    learned_match_kernel<K><<<grid, block, g.smem, stream>>>(p, lp);
    return cudaGetLastError();
}

cudaError_t launch_learned_match(const MatchParams &p, const LearnedParams &lp,
                                 const MatchGeometry &g, int nwin, cudaStream_t stream) {
    if (g.smem > 220 * 1024 || lp.cells_s < 1 || lp.cells_s > 8 || lp.cells_t < 1 ||
        lp.cells_t > 8 || !learned_ordinals_fit(p.bm_range, p.ps_num, p.ps_range))
        return cudaErrorInvalidValue;
    if (std::max(lp.cells_s, lp.cells_t) <= 2) return launch_learned_k<2>(p, lp, g, nwin, stream);
    return std::max(lp.cells_s, lp.cells_t) <= 4 ? launch_learned_k<4>(p, lp, g, nwin, stream)
                                                 : launch_learned_k<8>(p, lp, g, nwin, stream);
}

cudaError_t launch_match_fallback(const MatchParams &p, const unsigned *list,
                                  const unsigned *count, cudaStream_t stream) {
    const int ws = 2 * p.bm_range + 1, wt = 2 * p.ps_range + 1;
    const int buf = std::max(ws * ws, p.radius > 0 ? p.ps_num * wt * wt : 0);
    int region = std::max((ws + 7) * (ws + 7), p.radius > 0 ? (wt + 7) * (wt + 7) : 0);
    if ((size_t)(buf + region) * kFallbackWarps * sizeof(float) > 200 * 1024) region = 0;
    const size_t smem = (size_t)(buf + region) * kFallbackWarps * sizeof(float);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    static int configured[64] = {0};
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = raise_smem_limit(configured, (const void *)fallback_kernel, smem)) != cudaSuccess)
        return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    fallback_kernel<<<2 * sms, 32 * kFallbackWarps, smem, stream>>>(p, list, count, buf, region);
    return cudaGetLastError();
}

}  // namespace bm3d
