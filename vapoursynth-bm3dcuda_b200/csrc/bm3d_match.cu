// Block matching for BM3D / V-BM3D on sm_100a.
//
// Computes, for every reference block of every temporal window in a batch,
// the reference's 8-entry match list: exhaustive SSD search over the
// (2*bm_range+1)^2 window in the centre frame, then (radius > 0) the
// predictive search over ps_num windows of (2*ps_range+1)^2 per neighbour
// frame, then the centre-block insertion (source/kernel.cu:389-647,
// cpu_source/source.cpp:143-391, 787-844).
//
// Work layout
//   * one thread owns one reference block and scans all of its candidates in
//     the reference's scan order, so the strict-< list insertion gives
//     exactly the reference's list (ties keep the earlier candidate);
//   * a warp owns 4 x 8 reference blocks, a CTA WX such warps side by side;
//   * the search runs as 1 + 2r stages (centre frame, then frames c-1 .. c-r,
//     then c+1 .. c+r). Each stage stages the CTA's pixel region of its frame
//     into shared memory, then every thread scans its windows of that stage
//     with one strip routine (ssd_strip: one pixel load feeds up to 8
//     candidates). A single scan site and a single strip width keep the
//     unrolled code small enough for the instruction cache;
//   * shared-memory rows are skewed by (row / 8) mod 8 words, which makes the
//     32 threads of a warp hit 32 distinct banks when block_step is 8.
#include <cuda_runtime.h>

#include "bm3d_device.cuh"
#include "bm3d_internal.h"

namespace bm3d {

namespace {

// Scan one search window of a reference block in scan order (rows, then
// columns), feeding every in-range candidate to `list`.
//   wx: unclamped window origin column (centre - range), image coordinates
//   [left, right] x [top, bottom]: the clamped candidate range
//   (tx0, ty0): image coordinates of the tile's (0, 0)
template <int K, int M>
__device__ __forceinline__ void scan_window(List8 &list, const f32x2 (&refp)[4][8],
                                            const RefStats &rs, const float *tile, int pitch,
                                            int tx0, int ty0, int wx, int left, int right,
                                            int top, int bottom, int nsub, int z) {
    for (int row = top; row <= bottom; ++row) {
        int roff[8];
        const int ty = row - ty0;
#pragma unroll
        for (int r = 0; r < 8; ++r) roff[r] = skewed(ty + r, wx - tx0, pitch);
        for (int s = 0; s < nsub; ++s) {
            float err[K];
            if (M == 0) {
                ssd_strip<K>(refp, tile, roff, err);
            } else {
#pragma unroll
                for (int k = 0; k < K; ++k) err[k] = metric_dist<M>(refp, rs, tile, roff, k);
            }
            const int cx0 = wx + s * K;
            // cheap reject: once the list is full most strips improve nothing
            float best = err[0];
#pragma unroll
            for (int k = 1; k < K; ++k) best = fminf(best, err[k]);
            if (!(best < list.e[7])) {
#pragma unroll
                for (int r = 0; r < 8; ++r) roff[r] += K;
                continue;
            }
            unsigned mask = 0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int cx = cx0 + k;
                const bool ok = cx >= left && cx <= right && err[k] < list.e[7];
                mask |= (ok ? 1u : 0u) << k;
            }
            while (mask) {  // ascending k = the reference's scan order
                const int k = __ffs(mask) - 1;
                mask &= mask - 1;
                list_insert(list, pick(err, k), pack_pos(cx0 + k, row, z));
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) roff[r] += K;
        }
    }
}

// One CTA tile of reference blocks: tile (tile_x, tile_y) of window `win`.
// Every thread of the CTA must call it (it synchronises the CTA).
template <int K, int M = 0>
__device__ __forceinline__ void match_tile(const MatchParams &p, int tile_x, int tile_y, int win,
                                           float *tile) {
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nbx_cta = (blockDim.x >> 5) * 4;
    const int bx = tile_x * nbx_cta + warp * 4 + (lane & 3);
    const int by = tile_y * 8 + (lane >> 2);
    const bool active = bx < p.nbx && by < p.nby;

    const int x = min(bx * p.block_step, p.width - 8);
    const int y = min(by * p.block_step, p.height - 8);

    // CTA extent in reference-block origins
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
    const float *const *frames = p.frames + (size_t)win * (2 * r + 1);

    f32x2 refp[4][8];
    RefStats rs{0.0f, 0.0f};
    List8 list;
    list_init(list, FLT_MAX, pack_pos(x, y, center));
    // the spatial list's positions seed the +1 direction; parked in shared
    // memory after the tile (one column per thread) to free registers
    int *center_pos = reinterpret_cast<int *>(tile + (size_t)p.pitch * p.tile_rows) + threadIdx.x;
    int last[8];

    // stage 0: centre frame, exhaustive; stages 1..r: frames c-1..c-r;
    // stages r+1..2r: frames c+1..c+r (source/kernel.cu:503-613)
    for (int st = 0; st <= 2 * r; ++st) {
        const int t = st <= r ? st : st - r;
        const int z = st == 0 ? center : (st <= r ? center - t : center + t);
        const int m = p.bm_range + t * p.ps_range;  // reach of this stage's candidates
        const int tx0 = xa - m, ty0 = ya - m;
        const int twid = xb - xa + 2 * m + 8 + p.extra_cols;
        const int thei = yb - ya + 2 * m + 8;
        if (st > 0) __syncthreads();
        load_tile(tile, frames[z], p.width, p.height, p.stride, tx0, ty0, twid, thei, p.pitch);
        __syncthreads();
        if (st == 0) {
            // reference block as packed row pairs (rows 2q, 2q+1 of column c)
#pragma unroll
            for (int q = 0; q < 4; ++q)
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    refp[q][c] = pack2(tile[skewed(y - ty0 + 2 * q, x - tx0 + c, p.pitch)],
                                       tile[skewed(y - ty0 + 2 * q + 1, x - tx0 + c, p.pitch)]);
            if (M != 0) rs = ref_stats<M>(refp);
        }
        if (!active) continue;
        if (st == r + 1) {
#pragma unroll
            for (int i = 0; i < 8; ++i) last[i] = center_pos[i * blockDim.x];
        }
        List8 fl;
        list_init(fl, FLT_MAX, st == 0 ? pack_pos(x, y, center) : pack_pos(0, 0, z));
        const int range = st == 0 ? p.bm_range : p.ps_range;
        const int nwin = st == 0 ? 1 : p.ps_num;
        const int nsub = st == 0 ? p.nsub_s : p.nsub_t;
        for (int i = 0; i < nwin; ++i) {
            int cx = x, cy = y;
            if (st > 0) {
                const int li = pick(last, i);
                // Window centres are earlier matches and lie within
                // bm_range + (t-1)*ps_range of the block; the clamp only bites
                // for lists polluted by non-finite distances.
                cx = min(max(pos_x(li), x - m + range), x + m - range);
                cy = min(max(pos_y(li), y - m + range), y + m - range);
            }
            const int left = max(cx - range, 0), right = min(cx + range, p.width - 8);
            const int top = max(cy - range, 0), bottom = min(cy + range, p.height - 8);
            scan_window<K, M>(fl, refp, rs, tile, p.pitch, tx0, ty0, cx - range, left, right, top,
                              bottom, nsub, z);
        }
        if (st == 0) {
            list = fl;
#pragma unroll
            for (int i = 0; i < 8; ++i) center_pos[i * blockDim.x] = last[i] = fl.p[i];
        } else {
            // merge the frame's first ps_num entries (source/kernel.cu:589-608)
            for (int i = 0; i < p.ps_num; ++i) {
                const float e = pick(fl.e, i);
                if (e < list.e[7]) list_insert(list, e, pick(fl.p, i));
            }
#pragma unroll
            for (int i = 0; i < 8; ++i) last[i] = fl.p[i];
        }
    }

    if (!active) return;

    // ---- centre insertion (source/kernel.cu:616-647) ----------------------
    const int cpos = pack_pos(x, y, center);
    bool found = false;
#pragma unroll
    for (int i = 0; i < 8; ++i) found |= list.p[i] == cpos;
    if (!found) {
#pragma unroll
        for (int i = 7; i > 0; --i) list.p[i] = list.p[i - 1];
        list.p[0] = cpos;
    }

    int4 *out = reinterpret_cast<int4 *>(p.matches + ((size_t)win * p.nbx * p.nby +
                                                      (size_t)by * p.nbx + bx) * 8);
    out[0] = make_int4(list.p[0], list.p[1], list.p[2], list.p[3]);
    out[1] = make_int4(list.p[4], list.p[5], list.p[6], list.p[7]);
}

template <int K, int M = 0>
__global__ void __launch_bounds__(128, 3) match_kernel(MatchParams p) {
    extern __shared__ float tile[];
    match_tile<K, M>(p, blockIdx.x, blockIdx.y, p.win0 + blockIdx.z, tile);
}

// Persistent form for a batch of clips with their own geometry and
// parameters: resident CTAs take CTA tiles from a shared counter, clip-major
// in the order the clips were added; per-clip parameters are staged in
// shared memory for the tile.
template <int K>
__global__ void __launch_bounds__(128, 3) match_batch_kernel(MatchBatch b) {
    extern __shared__ float tile[];
    __shared__ MatchParams ps;
    __shared__ long long item_s;
    const long long total = b.item_off[b.nclips];
    const int nbx_cta = (blockDim.x >> 5) * 4;
    for (;;) {
        if (threadIdx.x == 0) {
            item_s = (long long)atomicAdd(b.counter, 1ULL);
            if (item_s == 0) *b.start_ns = globaltimer_ns();
        }
        __syncthreads();
        const long long item = item_s;
        if (item >= total) break;
        int lo = 0, hi = b.nclips;  // item_off[lo] <= item < item_off[hi]
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (b.item_off[mid] <= item) lo = mid; else hi = mid;
        }
        if (threadIdx.x == 0) ps = b.clips[lo];
        __syncthreads();
        const long long j = item - b.item_off[lo];
        const int ntx = (ps.nbx + nbx_cta - 1) / nbx_cta, nty = (ps.nby + 7) / 8;
        const int tx = (int)(j % ntx), ty = (int)((j / ntx) % nty), win = (int)(j / ((long long)ntx * nty));
        match_tile<K>(ps, tx, ty, win, tile);
        __syncthreads();
    }
}

template <int K, int M = 0>
cudaError_t launch_match_t(const MatchParams &p, dim3 grid, dim3 block, size_t smem,
                           cudaStream_t stream) {
    auto fn = match_kernel<K, M>;
    // The dynamic shared-memory opt-in is per device; raise it only when a
    // launch needs more than this device was configured for, so that launches
    // recorded into CUDA graphs do not repeat the attribute call.
    static int configured[64] = {0};
    cudaError_t e = raise_smem_limit(configured, (const void *)fn, smem);
    if (e != cudaSuccess) return e;
    fn<<<grid, block, smem, stream>>>(p);
    return cudaGetLastError();
}

// Strip width K (candidates per strip) for a spatial window of ws columns and
// temporal windows of wt columns: the K in [8, 12] with the fewest evaluated
// distances, counting both the strip overrun and the (K + 7) / K pixel loads.
int choose_strip_width(int ws, int wt, int radius, int ps_num) {
    const double spatial = (double)ws * ws;
    const double temporal = radius > 0 ? 2.0 * radius * ps_num * wt * wt : 0.0;
    int best = 8;
    double best_cost = 1e300;
    for (int K = 8; K <= 12; ++K) {
        const double over_s = (double)((ws + K - 1) / K * K) / ws;
        const double over_t = radius > 0 ? (double)((wt + K - 1) / K * K) / wt : 1.0;
        // ~143 FP32 operations per distance plus 8 (K + 7) / K shared-memory loads
        const double per = 143.0 + 8.0 * (K + 7) / K;
        const double cost = (spatial * over_s + temporal * over_t) * per;
        if (cost < best_cost) {
            best_cost = cost;
            best = K;
        }
    }
    return best;
}

}  // namespace

MatchGeometry match_geometry_with(int width, int height, int block_step, int bm_range, int radius,
                                  int ps_range, int wx, int K) {
    MatchGeometry g{};
    g.nbx = (width - 8 + block_step - 1) / block_step + 1;
    g.nby = (height - 8 + block_step - 1) / block_step + 1;
    const int ws = 2 * bm_range + 1, wt = 2 * ps_range + 1;
    g.ks = g.kt = K;
    g.nsub_s = (ws + g.ks - 1) / g.ks;
    g.nsub_t = (wt + g.kt - 1) / g.kt;
    g.extra_cols = std::max(g.nsub_s * g.ks - ws, radius > 0 ? g.nsub_t * g.kt - wt : 0);
    const int mmax = bm_range + radius * ps_range;
    const int tw = (4 * wx - 1) * block_step + 2 * mmax + 8 + g.extra_cols;
    const int th = 7 * block_step + 2 * mmax + 8;
    g.wx = wx;
    g.pitch = tw + 8;
    g.tile_rows = th;
    g.smem = (size_t)g.pitch * th * sizeof(float) + 8 * 32 * wx * sizeof(int);
    return g;
}

MatchGeometry match_geometry(int width, int height, int block_step, int bm_range, int radius,
                             int ps_range) {
    const int K = choose_strip_width(2 * bm_range + 1, 2 * ps_range + 1, radius, 2);
    // the widest CTA (in warps) whose tile fits comfortably
    MatchGeometry g{};
    for (int wx = 4; wx >= 1; wx /= 2) {
        g = match_geometry_with(width, height, block_step, bm_range, radius, ps_range, wx, K);
        if (g.smem <= 72 * 1024) break;
    }
    return g;
}

long long match_tiles(const MatchGeometry &g, int nwin) {
    return (long long)((g.nbx + 4 * g.wx - 1) / (4 * g.wx)) * ((g.nby + 7) / 8) * nwin;
}

template <int K>
cudaError_t launch_match_batch_t(const MatchBatch &b, int wx, size_t smem, cudaStream_t stream) {
    auto fn = match_batch_kernel<K>;
    static int configured[64] = {0};
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if ((e = raise_smem_limit(configured, (const void *)fn, smem)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, 32 * wx, smem)) !=
        cudaSuccess)
        return e;
    fn<<<sms * std::max(1, per_sm), 32 * wx, smem, stream>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_match_batch(const MatchBatch &b, int K, int wx, size_t smem,
                               cudaStream_t stream) {
    if (smem > 220 * 1024) return cudaErrorInvalidValue;
    switch (K) {
        case 9: return launch_match_batch_t<9>(b, wx, smem, stream);
        case 10: return launch_match_batch_t<10>(b, wx, smem, stream);
        case 11: return launch_match_batch_t<11>(b, wx, smem, stream);
        case 12: return launch_match_batch_t<12>(b, wx, smem, stream);
        default: return launch_match_batch_t<8>(b, wx, smem, stream);
    }
}

cudaError_t launch_match(const MatchParams &p, const MatchGeometry &g, int nwin,
                         cudaStream_t stream) {
    if (g.smem > 220 * 1024) return cudaErrorInvalidValue;
    dim3 block(32 * g.wx);
    dim3 grid((p.nbx + 4 * g.wx - 1) / (4 * g.wx), (p.nby + 7) / 8, nwin);
    if (p.metric != 0) {
        // one candidate per strip: the tile (sized for the SSD strips) covers it
        MatchParams q = p;
        q.nsub_s = 2 * p.bm_range + 1;
        q.nsub_t = 2 * p.ps_range + 1;
        switch (p.metric) {
            case 1: return launch_match_t<1, 1>(q, grid, block, g.smem, stream);
            case 2: return launch_match_t<1, 2>(q, grid, block, g.smem, stream);
            case 3: return launch_match_t<1, 3>(q, grid, block, g.smem, stream);
            case 4: return launch_match_t<1, 4>(q, grid, block, g.smem, stream);
            default: return cudaErrorInvalidValue;
        }
    }
    switch (g.ks) {
        case 9: return launch_match_t<9>(p, grid, block, g.smem, stream);
        case 10: return launch_match_t<10>(p, grid, block, g.smem, stream);
        case 11: return launch_match_t<11>(p, grid, block, g.smem, stream);
        case 12: return launch_match_t<12>(p, grid, block, g.smem, stream);
        default: return launch_match_t<8>(p, grid, block, g.smem, stream);
    }
}

}  // namespace bm3d
