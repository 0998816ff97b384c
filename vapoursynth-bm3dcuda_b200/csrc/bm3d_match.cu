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
//   * each search stage (centre frame, then frame c-1, c-2, ..., c+1, c+2,
//     ...) first stages the CTA's pixel region of that frame into shared
//     memory, then every thread runs its strips over it (ssd_strip: one pixel
//     load feeds up to 8 candidates);
//   * shared-memory rows are skewed by (row / 8) mod 8 words, which makes the
//     32 threads of a warp hit 32 distinct banks when block_step is 8.
#include <cuda_runtime.h>

#include "bm3d_device.cuh"
#include "bm3d_internal.h"

namespace bm3d {

namespace {

__device__ __forceinline__ int skewed(int ty, int tx, int pitch) {
    return ty * pitch + ((ty >> 3) & 7) + tx;
}

// Stage the pixel rectangle [y0, y0+th) x [x0, x0+tw) of `plane` into the
// tile; pixels outside the image read as 0 (they are never ranked).
__device__ void load_tile(float *tile, const float *__restrict__ plane, int width, int height,
                          int stride, int x0, int y0, int tw, int th, int pitch) {
    const int nthreads = blockDim.x;
    for (int ty = threadIdx.x / 32; ty < th; ty += nthreads / 32) {
        const int gy = y0 + ty;
        const bool row_ok = gy >= 0 && gy < height;
        const float *src = plane + (size_t)(row_ok ? gy : 0) * stride;
        float *dst = tile + ty * pitch + ((ty >> 3) & 7);
        for (int tx = threadIdx.x % 32; tx < tw; tx += 32) {
            const int gx = x0 + tx;
            float v = 0.0f;
            if (row_ok && gx >= 0 && gx < width) v = __ldg(src + gx);
            dst[tx] = v;
        }
    }
}

// Scan one search window of a reference block in scan order (rows, then
// columns), feeding every in-range candidate to `list`.
//   (wx, wy): unclamped window origin (centre - range), in image coordinates
//   [left, right] x [top, bottom]: the clamped candidate range
//   (tx0, ty0): image coordinates of the tile's (0, 0)
template <int K>
__device__ __forceinline__ void scan_window(List8 &list, const float (&ref)[8][8],
                                            const float *tile, int pitch, int tx0, int ty0,
                                            int wx, int left, int right, int top, int bottom,
                                            int nsub, int z) {
    for (int row = top; row <= bottom; ++row) {
        int roff[8];
        const int ty = row - ty0;
#pragma unroll
        for (int r = 0; r < 8; ++r) roff[r] = skewed(ty + r, wx - tx0, pitch);
        for (int s = 0; s < nsub; ++s) {
            float err[K];
            ssd_strip<K>(ref, tile, roff, err);
            const int cx0 = wx + s * K;
            // filter against the current worst entry before the (rare) inserts
            unsigned mask = 0;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const int cx = cx0 + k;
                const bool ok = cx >= left && cx <= right && err[k] < list.e[7];
                mask |= (ok ? 1u : 0u) << k;
            }
            if (mask) {
#pragma unroll
                for (int k = 0; k < K; ++k) {
                    if (mask & (1u << k)) list_insert(list, err[k], pack_pos(cx0 + k, row, z));
                }
            }
#pragma unroll
            for (int r = 0; r < 8; ++r) roff[r] += K;
        }
    }
}

template <int KS, int KT>
__global__ void __launch_bounds__(128, 3) match_kernel(MatchParams p) {
    extern __shared__ float tile[];

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int nbx_cta = (blockDim.x >> 5) * 4;
    const int bx = blockIdx.x * nbx_cta + warp * 4 + (lane & 3);
    const int by = blockIdx.y * 8 + (lane >> 2);
    const int win = blockIdx.z;
    const bool active = bx < p.nbx && by < p.nby;

    const int x = min(bx * p.block_step, p.width - 8);
    const int y = min(by * p.block_step, p.height - 8);

    // CTA extent in reference-block origins
    const int bx_first = blockIdx.x * nbx_cta;
    const int bx_last = min(bx_first + nbx_cta - 1, p.nbx - 1);
    const int by_first = blockIdx.y * 8;
    const int by_last = min(by_first + 7, p.nby - 1);
    const int xa = min(bx_first * p.block_step, p.width - 8);
    const int xb = min(bx_last * p.block_step, p.width - 8);
    const int ya = min(by_first * p.block_step, p.height - 8);
    const int yb = min(by_last * p.block_step, p.height - 8);

    const int tw = 2 * p.radius + 1;
    const int center = p.radius;
    const float *const *frames = p.frames + (size_t)win * tw;

    float ref[8][8];
    List8 list;
    list_init(list, FLT_MAX, pack_pos(x, y, center));

    // ---- stage 0: exhaustive search in the centre frame -------------------
    {
        const int m = p.bm_range;
        const int tx0 = xa - m, ty0 = ya - m;
        const int twid = xb - xa + 2 * m + 8 + p.extra_cols;
        const int thei = yb - ya + 2 * m + 8;
        load_tile(tile, frames[center], p.width, p.height, p.stride, tx0, ty0, twid, thei,
                  p.pitch);
        __syncthreads();
        // reference block from the staged centre frame
#pragma unroll
        for (int r = 0; r < 8; ++r) {
#pragma unroll
            for (int c = 0; c < 8; ++c) ref[r][c] = tile[skewed(y - ty0 + r, x - tx0 + c, p.pitch)];
        }
        if (active) {
            const int left = max(x - m, 0), right = min(x + m, p.width - 8);
            const int top = max(y - m, 0), bottom = min(y + m, p.height - 8);
            scan_window<KS>(list, ref, tile, p.pitch, tx0, ty0, x - m, left, right, top, bottom,
                            p.nsub_s, center);
        }
    }

    // ---- temporal predictive search (source/kernel.cu:495-614) ------------
    if (p.radius > 0) {
        int center_pos[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) center_pos[i] = list.p[i];
        for (int dir = -1; dir <= 1; dir += 2) {
            int last[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) last[i] = center_pos[i];
            for (int t = 1; t <= p.radius; ++t) {
                const int z = center + dir * t;
                const int m = p.bm_range + t * p.ps_range;
                const int tx0 = xa - m, ty0 = ya - m;
                const int twid = xb - xa + 2 * m + 8 + p.extra_cols;
                const int thei = yb - ya + 2 * m + 8;
                __syncthreads();
                load_tile(tile, frames[z], p.width, p.height, p.stride, tx0, ty0, twid, thei,
                          p.pitch);
                __syncthreads();
                if (active) {
                    List8 fl;
                    list_init(fl, FLT_MAX, pack_pos(0, 0, z));
                    const int pr = p.ps_range;
                    for (int i = 0; i < p.ps_num; ++i) {
                        int li = last[0];
#pragma unroll
                        for (int k = 1; k < 8; ++k) li = (i == k) ? last[k] : li;
                        int xx = pos_x(li), yy = pos_y(li);
                        // Window centres are earlier matches and lie within
                        // bm_range + (t-1)*ps_range of the block; the clamp only
                        // bites for lists polluted by non-finite distances.
                        xx = min(max(xx, x - m + pr), x + m - pr);
                        yy = min(max(yy, y - m + pr), y + m - pr);
                        const int left = max(xx - pr, 0), right = min(xx + pr, p.width - 8);
                        const int top = max(yy - pr, 0), bottom = min(yy + pr, p.height - 8);
                        scan_window<KT>(fl, ref, tile, p.pitch, tx0, ty0, xx - pr, left, right,
                                        top, bottom, p.nsub_t, z);
                    }
                    // merge the frame's first ps_num entries (source/kernel.cu:589-608)
                    for (int i = 0; i < p.ps_num; ++i) {
                        float e = fl.e[0];
                        int q = fl.p[0];
#pragma unroll
                        for (int k = 1; k < 8; ++k) {
                            e = (i == k) ? fl.e[k] : e;
                            q = (i == k) ? fl.p[k] : q;
                        }
                        if (e < list.e[7]) list_insert(list, e, q);
                    }
#pragma unroll
                    for (int i = 0; i < 8; ++i) last[i] = fl.p[i];
                }
            }
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

template <int KS, int KT>
cudaError_t launch_match_t(const MatchParams &p, dim3 grid, dim3 block, size_t smem,
                           cudaStream_t stream) {
    auto fn = match_kernel<KS, KT>;
    // The dynamic shared-memory opt-in is per device; raise it only when a
    // launch needs more than this device was configured for, so that launches
    // recorded into CUDA graphs do not repeat the attribute call.
    static int configured[64] = {0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 64 || configured[dev] < (int)smem) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        if (dev >= 0 && dev < 64) configured[dev] = (int)smem;
    }
    fn<<<grid, block, smem, stream>>>(p);
    return cudaGetLastError();
}

int strip_width(int window) {
    // Preferred strip widths: 19 candidates -> 2 x 10, 33 -> 3 x 11, 9 -> 9.
    if (window == 19 || window == 20) return 10;
    if (window == 33) return 11;
    if (window == 9) return 9;
    return 8;
}

}  // namespace

int match_nsub(int window, int K) { return (window + K - 1) / K; }

MatchGeometry match_geometry(int width, int height, int block_step, int bm_range, int radius,
                             int ps_range) {
    MatchGeometry g{};
    g.nbx = (width - 8 + block_step - 1) / block_step + 1;
    g.nby = (height - 8 + block_step - 1) / block_step + 1;
    g.ks = strip_width(2 * bm_range + 1);
    g.kt = strip_width(2 * ps_range + 1);
    g.nsub_s = match_nsub(2 * bm_range + 1, g.ks);
    g.nsub_t = match_nsub(2 * ps_range + 1, g.kt);
    g.extra_cols = std::max(g.nsub_s * g.ks - (2 * bm_range + 1),
                            radius > 0 ? g.nsub_t * g.kt - (2 * ps_range + 1) : 0);
    const int mmax = bm_range + radius * ps_range;
    // pick the widest CTA (in warps) whose tile fits comfortably
    for (int wx = 4; wx >= 1; wx /= 2) {
        const int tw = (4 * wx - 1) * block_step + 2 * mmax + 8 + g.extra_cols;
        const int th = 7 * block_step + 2 * mmax + 8;
        const int pitch = tw + 8;
        const size_t smem = (size_t)pitch * th * sizeof(float);
        g.wx = wx;
        g.pitch = pitch;
        g.smem = smem;
        if (smem <= 72 * 1024) break;
    }
    return g;
}

cudaError_t launch_match(const MatchParams &p, const MatchGeometry &g, int nwin,
                         cudaStream_t stream) {
    if (g.smem > 220 * 1024) return cudaErrorInvalidValue;
    dim3 block(32 * g.wx);
    dim3 grid((p.nbx + 4 * g.wx - 1) / (4 * g.wx), (p.nby + 7) / 8, nwin);
    if (g.ks == 10 && g.kt == 9) return launch_match_t<10, 9>(p, grid, block, g.smem, stream);
    if (g.ks == 11 && g.kt == 9) return launch_match_t<11, 9>(p, grid, block, g.smem, stream);
    if (g.ks == 10 && g.kt == 8) return launch_match_t<10, 8>(p, grid, block, g.smem, stream);
    if (g.ks == 11 && g.kt == 8) return launch_match_t<11, 8>(p, grid, block, g.smem, stream);
    if (g.ks == 8 && g.kt == 9) return launch_match_t<8, 9>(p, grid, block, g.smem, stream);
    if (g.ks == 9 && g.kt == 9) return launch_match_t<9, 9>(p, grid, block, g.smem, stream);
    if (g.ks == 9 && g.kt == 8) return launch_match_t<9, 8>(p, grid, block, g.smem, stream);
    return launch_match_t<8, 8>(p, grid, block, g.smem, stream);
}

}  // namespace bm3d
