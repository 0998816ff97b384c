// Batched two-stage V-BM3D for many single-plane clips of uneven size and
// parameters (include/bm3d_b200.h, section 4).
//
// Every stage of the pipeline runs as one persistent launch over all clips:
// resident CTAs take work items (match tiles, filter group ranges,
// aggregation tiles) from a shared counter, clip-major. The six launches and
// the zeroing between them are recorded once into a CUDA graph; a run is one
// graph launch. A project-written autotuner picks the match kernel's CTA
// width and strip width for the batch by timing the candidates on it. The
// final aggregation stamps each clip's completion time on the device clock,
// so per-clip latencies come from the GPU, not the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <limits>
#include <new>
#include <string>
#include <vector>

#include "bm3d_b200.h"
#include "bm3d_device.cuh"
#include "bm3d_internal.h"

using namespace bm3d;

// defined with the rest of the C ABI (bm3d_capi.cu)
namespace bm3d {
int abi_fail(int code, const char *msg);
}

namespace {

int bfail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    return bm3d::abi_fail(code, buf);
}

#define BTRY(expr)                                                                       \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return bfail(BM3D_B200_ERR_CUDA, "BM3D batch: '%s' failed: %s", #expr,      \
                         cudaGetErrorString(e_));                                        \
    } while (0)

struct BatchClip {
    int w = 0, h = 0, n = 0, stride = 0;
    bm3d_b200_params prm{};
    const float *d_src = nullptr;
    float *d_dst = nullptr;
    // owned scratch
    float *d_basic = nullptr;
    float *d_acc = nullptr;
    int *d_matches = nullptr;
    void **d_tab = nullptr;   // [basic: match src ref acc][final: match src ref acc]
    float *d_mult = nullptr;  // [basic][final]
};

constexpr int kCounters = 8;  // 6 stage counters, start stamp, spare stamp

}  // namespace

struct bm3d_b200_batch {
    int device = 0;
    std::vector<BatchClip> clips;
    int wx = 4, K = 10;
    // resident CTAs per SM of the persistent filter (basic, final) and
    // aggregation launches (0: as many as fit)
    int filter_per_sm[2] = {0, 0}, agg_per_sm = 0;
    bool tuned = false, prepared = false;
    // device descriptor arrays
    MatchParams *d_mp = nullptr;       // [2][nclips]
    FilterParams *d_fp = nullptr;      // [2][nclips]
    AggregateParams *d_ap = nullptr;   // [2][nclips]
    long long *d_off = nullptr;        // [6][nclips + 1]
    unsigned long long *d_ctr = nullptr;  // [kCounters]
    unsigned *d_remaining = nullptr;   // [nclips]
    unsigned *d_remaining_init = nullptr;  // [nclips] tiles per clip of the final aggregation
    unsigned long long *d_end = nullptr;  // [nclips]
    std::vector<unsigned> remaining_init;
    size_t match_smem = 0;
    cudaStream_t cap = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace {

void release_clip_scratch(BatchClip &c) {
    cudaFree(c.d_basic);
    cudaFree(c.d_acc);
    cudaFree(c.d_matches);
    cudaFree(c.d_tab);
    cudaFree(c.d_mult);
    c.d_basic = c.d_acc = nullptr;
    c.d_matches = nullptr;
    c.d_tab = nullptr;
    c.d_mult = nullptr;
}

void release_device(bm3d_b200_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
    cudaFree(b->d_mp);
    cudaFree(b->d_fp);
    cudaFree(b->d_ap);
    cudaFree(b->d_off);
    cudaFree(b->d_ctr);
    cudaFree(b->d_remaining);
    cudaFree(b->d_remaining_init);
    cudaFree(b->d_end);
    b->d_remaining_init = nullptr;
    b->d_mp = nullptr;
    b->d_fp = nullptr;
    b->d_ap = nullptr;
    b->d_off = nullptr;
    b->d_ctr = nullptr;
    b->d_remaining = nullptr;
    b->d_end = nullptr;
    b->prepared = false;
}

MatchGeometry clip_geometry(const bm3d_b200_batch *b, const BatchClip &c, int wx, int K) {
    return match_geometry_with(c.w, c.h, c.prm.block_step[0], c.prm.bm_range[0], c.prm.radius,
                               c.prm.ps_range[0], wx, K);
}

// Stage tables of one clip (fused VAggregate mapping, source/source.cpp:830-844).
void build_tables(const BatchClip &c, bool final_, std::vector<void *> &tab,
                  std::vector<float> &mult) {
    const int N = c.n, r = c.prm.radius, tw = 2 * r + 1;
    const size_t ntab = (size_t)N * tw, plane = (size_t)c.h * c.stride, ff = plane;
    tab.assign(4 * ntab, nullptr);
    mult.assign(ntab, r > 0 ? 0.0f : 1.0f);
    auto clampf = [&](int f) { return std::min(std::max(f, 0), N - 1); };
    const float *mclip = final_ ? c.d_basic : c.d_src;
    for (int n = 0; n < N; ++n)
        for (int z = 0; z < tw; ++z) {
            const size_t k = (size_t)n * tw + z;
            const size_t f = (size_t)clampf(n - r + z);
            tab[k] = (void *)(mclip + f * ff);
            tab[ntab + k] = (void *)(c.d_src + f * ff);
            tab[2 * ntab + k] = final_ ? (void *)(c.d_basic + f * ff) : nullptr;
            tab[3 * ntab + k] = r > 0 ? nullptr : (void *)(c.d_acc + (size_t)n * 2 * plane);
        }
    if (r > 0)
        for (int m = 0; m < N; ++m)
            for (int i = 0; i < tw; ++i) {
                const int f = clampf(m - r + i);
                const int s = std::min(std::max(2 * r - i, m - N + 1 + r), m + r);
                const size_t k = (size_t)f * tw + s;
                tab[3 * ntab + k] = (void *)(c.d_acc + (size_t)m * 2 * plane);
                mult[k] += 1.0f;
            }
}

// Descriptors and offsets for the current (wx, K); allocates scratch once.
int prepare(bm3d_b200_batch *b) {
    const int nc = (int)b->clips.size();
    if (nc == 0) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: no clips");
    BTRY(cudaSetDevice(b->device));
    release_device(b);
    std::vector<MatchParams> mp(2 * nc);
    std::vector<FilterParams> fp(2 * nc);
    std::vector<AggregateParams> ap(2 * nc);
    std::vector<long long> off(6 * (nc + 1), 0);
    b->remaining_init.assign(nc, 0);
    b->match_smem = 0;
    for (int i = 0; i < nc; ++i) {
        BatchClip &c = b->clips[i];
        const int N = c.n, tw = 2 * c.prm.radius + 1;
        const size_t ntab = (size_t)N * tw, plane = (size_t)c.h * c.stride;
        const MatchGeometry g = clip_geometry(b, c, b->wx, b->K);
        if (g.smem > 220 * 1024)
            return bfail(BM3D_B200_ERR_UNSUPPORTED, "BM3D batch: clip %d needs %zu B of shared memory",
                         i, g.smem);
        b->match_smem = std::max(b->match_smem, g.smem);
        if (!c.d_basic) {
            BTRY(cudaMalloc(&c.d_basic, (size_t)N * plane * sizeof(float)));
            BTRY(cudaMalloc(&c.d_acc, (size_t)N * 2 * plane * sizeof(float)));
            BTRY(cudaMalloc(&c.d_matches, (size_t)N * g.nbx * g.nby * 8 * sizeof(int)));
            BTRY(cudaMalloc(&c.d_tab, 8 * ntab * sizeof(void *)));
            BTRY(cudaMalloc(&c.d_mult, 2 * ntab * sizeof(float)));
            for (int st = 0; st < 2; ++st) {
                std::vector<void *> tab;
                std::vector<float> mult;
                build_tables(c, st == 1, tab, mult);
                BTRY(cudaMemcpy(c.d_tab + st * 4 * ntab, tab.data(), tab.size() * sizeof(void *),
                                cudaMemcpyHostToDevice));
                BTRY(cudaMemcpy(c.d_mult + st * ntab, mult.data(), ntab * sizeof(float),
                                cudaMemcpyHostToDevice));
            }
        }
        const float sig[2] = {bm3d_b200_scale_sigma(c.prm.sigma[0], 0),
                              bm3d_b200_scale_sigma(c.prm.sigma[0], 1)};
        for (int st = 0; st < 2; ++st) {
            void **tab = c.d_tab + st * 4 * ntab;
            MatchParams &m = mp[st * nc + i];
            m = MatchParams{};
            m.frames = reinterpret_cast<const float *const *>(tab);
            m.matches = c.d_matches;
            m.width = c.w;
            m.height = c.h;
            m.stride = c.stride;
            m.block_step = c.prm.block_step[0];
            m.bm_range = c.prm.bm_range[0];
            m.radius = c.prm.radius;
            m.ps_num = c.prm.ps_num[0];
            m.ps_range = c.prm.ps_range[0];
            m.nbx = g.nbx;
            m.nby = g.nby;
            m.pitch = g.pitch;
            m.tile_rows = g.tile_rows;
            m.extra_cols = g.extra_cols;
            m.nsub_s = g.nsub_s;
            m.nsub_t = g.nsub_t;
            FilterParams &f = fp[st * nc + i];
            f = FilterParams{};
            f.src = reinterpret_cast<const float *const *>(tab + ntab);
            f.ref = st ? reinterpret_cast<const float *const *>(tab + 2 * ntab) : nullptr;
            f.acc = reinterpret_cast<float *const *>(tab + 3 * ntab);
            f.mult = c.prm.radius > 0 ? c.d_mult + st * ntab : nullptr;
            f.matches = c.d_matches;
            f.weight_offset = (long long)plane;
            f.acc_stride = c.stride;
            f.stride = c.stride;
            f.radius = c.prm.radius;
            f.nblk = g.nbx * g.nby;
            f.nbx = g.nbx;
            f.nwin = N;
            f.corner_weight = 1;
            f.sigma = sig[st];
            f.extractor = c.prm.extractor_exp ? std::ldexp(1.0f, c.prm.extractor_exp) : 0.0f;
            AggregateParams &a = ap[st * nc + i];
            a = AggregateParams{};
            a.dst = st ? c.d_dst : c.d_basic;
            a.wdst = c.d_acc;
            a.dst_plane_stride = (long long)plane;
            a.acc_plane_stride = (long long)2 * plane;
            a.weight_offset = (long long)plane;
            a.dst_stride = c.stride;
            a.acc_stride = c.stride;
            a.width = c.w;
            a.height = c.h;
            a.nplanes = N;
            a.corner_weight = 1;
            a.vec = aggregate_vec(a);
            // item counts: [match b, filter b, agg b, match f, filter f, agg f]
            const long long items[3] = {match_tiles(g, N), filter_ctas(f), aggregate_tiles(a)};
            for (int k = 0; k < 3; ++k)
                off[(st * 3 + k) * (nc + 1) + i + 1] = items[k];
            if (st == 1) b->remaining_init[i] = (unsigned)items[2];
        }
    }
    for (int s = 0; s < 6; ++s)
        for (int i = 0; i < nc; ++i) off[s * (nc + 1) + i + 1] += off[s * (nc + 1) + i];
    BTRY(cudaMalloc(&b->d_mp, mp.size() * sizeof(MatchParams)));
    BTRY(cudaMalloc(&b->d_fp, fp.size() * sizeof(FilterParams)));
    BTRY(cudaMalloc(&b->d_ap, ap.size() * sizeof(AggregateParams)));
    BTRY(cudaMalloc(&b->d_off, off.size() * sizeof(long long)));
    BTRY(cudaMalloc(&b->d_ctr, kCounters * sizeof(unsigned long long)));
    BTRY(cudaMalloc(&b->d_remaining, nc * sizeof(unsigned)));
    BTRY(cudaMalloc(&b->d_remaining_init, nc * sizeof(unsigned)));
    BTRY(cudaMalloc(&b->d_end, nc * sizeof(unsigned long long)));
    BTRY(cudaMemcpy(b->d_remaining_init, b->remaining_init.data(), nc * sizeof(unsigned),
                    cudaMemcpyHostToDevice));
    BTRY(cudaMemcpy(b->d_mp, mp.data(), mp.size() * sizeof(MatchParams), cudaMemcpyHostToDevice));
    BTRY(cudaMemcpy(b->d_fp, fp.data(), fp.size() * sizeof(FilterParams), cudaMemcpyHostToDevice));
    BTRY(cudaMemcpy(b->d_ap, ap.data(), ap.size() * sizeof(AggregateParams), cudaMemcpyHostToDevice));
    BTRY(cudaMemcpy(b->d_off, off.data(), off.size() * sizeof(long long), cudaMemcpyHostToDevice));
    b->prepared = true;
    return BM3D_B200_OK;
}

// The basic-stage match launch alone (autotuner probe).
int enqueue_match(bm3d_b200_batch *b, int st, unsigned long long *counter,
                  unsigned long long *stamp, cudaStream_t s) {
    const int nc = (int)b->clips.size();
    MatchBatch mb{b->d_mp + st * nc, b->d_off + (st * 3 + 0) * (nc + 1), nc, counter, stamp};
    BTRY(launch_match_batch(mb, b->K, b->wx, b->match_smem, s));
    return BM3D_B200_OK;
}

// Whole two-stage pipeline for every clip.
int enqueue_all(bm3d_b200_batch *b, cudaStream_t s) {
    const int nc = (int)b->clips.size();
    BTRY(cudaMemsetAsync(b->d_ctr, 0, kCounters * sizeof(unsigned long long), s));
    BTRY(cudaMemcpyAsync(b->d_remaining, b->d_remaining_init, nc * sizeof(unsigned),
                         cudaMemcpyDeviceToDevice, s));
    for (int st = 0; st < 2; ++st) {
        for (const BatchClip &c : b->clips)
            BTRY(cudaMemsetAsync(c.d_acc, 0, (size_t)c.n * 2 * c.h * c.stride * sizeof(float), s));
        // the batch start is stamped by the first basic tile; the final
        // stage's first tile writes the spare slot
        if (int rc = enqueue_match(b, st, b->d_ctr + st * 3 + 0, b->d_ctr + 6 + st, s)) return rc;
        FilterBatch fb{b->d_fp + st * nc, b->d_off + (st * 3 + 1) * (nc + 1), nc,
                       b->d_ctr + st * 3 + 1};
        BTRY(launch_filter_batch(fb, st == 1, s, b->filter_per_sm[st]));
        AggregateBatch ab{b->d_ap + st * nc, b->d_off + (st * 3 + 2) * (nc + 1), nc,
                          b->d_ctr + st * 3 + 2, st == 1 ? b->d_remaining : nullptr,
                          st == 1 ? b->d_end : nullptr};
        BTRY(launch_aggregate_batch(ab, s, b->agg_per_sm));
    }
    return BM3D_B200_OK;
}

int capture(bm3d_b200_batch *b) {
    if (!b->cap) BTRY(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    // first run outside capture (kernel attributes), then record
    if (int rc = enqueue_all(b, b->cap)) return rc;
    BTRY(cudaStreamSynchronize(b->cap));
    BTRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_all(b, b->cap);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(b->cap, &graph);
    if (rc) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess)
        return bfail(BM3D_B200_ERR_CUDA, "BM3D batch: capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess)
        return bfail(BM3D_B200_ERR_CUDA, "BM3D batch: instantiation failed: %s",
                     cudaGetErrorString(e));
    return BM3D_B200_OK;
}

}  // namespace

extern "C" int bm3d_b200_batch_create(bm3d_b200_batch **out, int device_id) {
    if (!out) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: null handle");
    *out = nullptr;
    int count = 0;
    BTRY(cudaGetDeviceCount(&count));
    if (device_id < 0 || device_id >= count)
        return bfail(BM3D_B200_ERR_INVALID, "BM3D: invalid device ID (%d)", device_id);
    auto *b = new (std::nothrow) bm3d_b200_batch;
    if (!b) return bfail(BM3D_B200_ERR_NOMEM, "BM3D batch: out of host memory");
    b->device = device_id;
    *out = b;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_batch_add(bm3d_b200_batch *b, int width, int height, int num_frames,
                                   const bm3d_b200_params *params, const float *d_src,
                                   float *d_dst, int *clip_index) {
    if (!b || !params || !d_src || !d_dst)
        return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: null argument");
    if (num_frames <= 0) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: clip has no frames");
    const bm3d_b200_params &p = *params;
    if (!(p.sigma[0] >= std::numeric_limits<float>::epsilon()))
        return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: sigma must be positive");
    if (width < 8 || height < 8 || width > BM3D_B200_MAX_DIM || height > BM3D_B200_MAX_DIM)
        return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: unsupported plane size %dx%d", width,
                     height);
    if (p.block_step[0] < 1 || p.block_step[0] > 8 || p.bm_range[0] < 1 || p.radius < 0 ||
        p.radius > BM3D_B200_MAX_RADIUS || p.ps_num[0] < 1 || p.ps_num[0] > 8 ||
        p.ps_range[0] < 1)
        return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: search parameters out of range");
    BatchClip c;
    c.w = width;
    c.h = height;
    c.n = num_frames;
    c.stride = (width + 31) / 32 * 32;
    c.prm = p;
    c.d_src = d_src;
    c.d_dst = d_dst;
    b->clips.push_back(c);
    b->prepared = false;
    if (clip_index) *clip_index = (int)b->clips.size() - 1;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_batch_autotune(bm3d_b200_batch *b, void *stream) {
    if (!b) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: null handle");
    BTRY(cudaSetDevice(b->device));
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // the events are released on every return path
    struct Events {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ~Events() {
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
        }
    } ev;
    BTRY(cudaEventCreate(&ev.e0));
    BTRY(cudaEventCreate(&ev.e1));
    cudaEvent_t e0 = ev.e0, e1 = ev.e1;
    float best = FLT_MAX;
    int best_wx = b->wx, best_k = b->K;
    for (int wx : {1, 2, 4}) {
        for (int K = 8; K <= 12; ++K) {
            b->wx = wx;
            b->K = K;
            if (prepare(b) != BM3D_B200_OK) continue;  // e.g. tile too large
            float t = FLT_MAX;
            for (int rep = 0; rep < 2; ++rep) {
                BTRY(cudaMemsetAsync(b->d_ctr, 0, kCounters * sizeof(unsigned long long), s));
                BTRY(cudaEventRecord(e0, s));
                if (int rc = enqueue_match(b, 0, b->d_ctr, b->d_ctr + 7, s)) return rc;
                BTRY(cudaEventRecord(e1, s));
                BTRY(cudaEventSynchronize(e1));
                float ms = 0;
                BTRY(cudaEventElapsedTime(&ms, e0, e1));
                t = std::min(t, ms);
            }
            if (t < best) {
                best = t;
                best_wx = wx;
                best_k = K;
            }
        }
    }
    b->wx = best_wx;
    b->K = best_k;
    if (int rc = prepare(b)) return rc;
    // Persistent filter and aggregation grids: one whole pipeline run fills
    // the match lists and accumulators, then each stage's launch alone is
    // timed with 1 .. 4 (filter) or 1, 2, 4, 8 (aggregation) resident CTAs
    // per SM, capped at the occupancy limit. The repeated launches only add
    // to the accumulators, which every real run clears first.
    const int nc = (int)b->clips.size();
    if (int rc = enqueue_all(b, s)) return rc;
    auto time_launch = [&](auto &&launch, float *ms_out) -> int {
        float t = FLT_MAX;
        for (int rep = 0; rep < 2; ++rep) {
            BTRY(cudaMemsetAsync(b->d_ctr, 0, kCounters * sizeof(unsigned long long), s));
            BTRY(cudaEventRecord(e0, s));
            BTRY(launch());
            BTRY(cudaEventRecord(e1, s));
            BTRY(cudaEventSynchronize(e1));
            float ms = 0;
            BTRY(cudaEventElapsedTime(&ms, e0, e1));
            t = std::min(t, ms);
        }
        *ms_out = t;
        return BM3D_B200_OK;
    };
    for (int st = 0; st < 2; ++st) {
        float best_t = FLT_MAX;
        int best_n = 0;
        for (int per_sm = 1; per_sm <= 4; ++per_sm) {
            FilterBatch fb{b->d_fp + st * nc, b->d_off + (st * 3 + 1) * (nc + 1), nc, b->d_ctr};
            float t = 0;
            if (int rc = time_launch(
                    [&] { return launch_filter_batch(fb, st == 1, s, per_sm); }, &t))
                return rc;
            if (t < best_t) {
                best_t = t;
                best_n = per_sm;
            }
        }
        b->filter_per_sm[st] = best_n;
    }
    {
        float best_t = FLT_MAX;
        int best_n = 0;
        for (int per_sm = 1; per_sm <= 8; per_sm *= 2) {
            AggregateBatch ab{b->d_ap, b->d_off + 2 * (nc + 1), nc, b->d_ctr, nullptr, nullptr};
            float t = 0;
            if (int rc = time_launch([&] { return launch_aggregate_batch(ab, s, per_sm); }, &t))
                return rc;
            if (t < best_t) {
                best_t = t;
                best_n = per_sm;
            }
        }
        b->agg_per_sm = best_n;
    }
    BTRY(cudaStreamSynchronize(s));
    if (b->exec) {  // recorded with the previous grids
        cudaGraphExecDestroy(b->exec);
        b->exec = nullptr;
    }
    b->tuned = true;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_batch_config(const bm3d_b200_batch *b, int *cta_warps, int *strip) {
    if (!b) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: null handle");
    if (cta_warps) *cta_warps = b->wx;
    if (strip) *strip = b->K;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_batch_grids(const bm3d_b200_batch *b, int *filter_basic_per_sm,
                                     int *filter_final_per_sm, int *aggregate_per_sm) {
    if (!b) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: null handle");
    if (filter_basic_per_sm) *filter_basic_per_sm = b->filter_per_sm[0];
    if (filter_final_per_sm) *filter_final_per_sm = b->filter_per_sm[1];
    if (aggregate_per_sm) *aggregate_per_sm = b->agg_per_sm;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_batch_run(bm3d_b200_batch *b, void *stream) {
    if (!b) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: null handle");
    BTRY(cudaSetDevice(b->device));
    if (!b->prepared) {
        if (int rc = prepare(b)) return rc;
    }
    if (!b->exec) {
        if (int rc = capture(b)) return rc;
    }
    BTRY(cudaGraphLaunch(b->exec, reinterpret_cast<cudaStream_t>(stream)));
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_batch_basic(bm3d_b200_batch *b, int clip_index, float *d_basic,
                                     void *stream) {
    if (!b || !d_basic) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: null argument");
    if (clip_index < 0 || clip_index >= (int)b->clips.size())
        return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: no clip %d", clip_index);
    const BatchClip &c = b->clips[clip_index];
    if (!b->prepared || !c.d_basic)
        return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: not run yet");
    BTRY(cudaSetDevice(b->device));
    BTRY(cudaMemcpyAsync(d_basic, c.d_basic, (size_t)c.n * c.h * c.stride * sizeof(float),
                         cudaMemcpyDeviceToDevice, reinterpret_cast<cudaStream_t>(stream)));
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_batch_latencies(bm3d_b200_batch *b, double *ms, int capacity) {
    if (!b || !ms) return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: null argument");
    const int nc = (int)b->clips.size();
    if (capacity < nc || !b->prepared)
        return bfail(BM3D_B200_ERR_INVALID, "BM3D batch: not run yet or buffer too small");
    BTRY(cudaSetDevice(b->device));
    BTRY(cudaDeviceSynchronize());
    std::vector<unsigned long long> end(nc), ctr(kCounters);
    BTRY(cudaMemcpy(end.data(), b->d_end, nc * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    BTRY(cudaMemcpy(ctr.data(), b->d_ctr, kCounters * sizeof(unsigned long long),
                    cudaMemcpyDeviceToHost));
    for (int i = 0; i < nc; ++i) ms[i] = (double)(long long)(end[i] - ctr[6]) * 1e-6;
    return BM3D_B200_OK;
}

extern "C" void bm3d_b200_batch_destroy(bm3d_b200_batch *b) {
    if (!b) return;
    cudaSetDevice(b->device);
    cudaDeviceSynchronize();
    release_device(b);
    for (auto &c : b->clips) release_clip_scratch(c);
    if (b->cap) cudaStreamDestroy(b->cap);
    delete b;
}
