// Host runtime of the bm3d_b200 C ABI (include/bm3d_b200.h).
//
// Owns argument validation (the reference's create-time checks,
// source/source.cpp:476-634), scratch allocation, pointer tables that map
// every (window, temporal slot) to its planes, CUDA graphs for the
// per-window pipeline, and the device-resident clip pipeline.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cfloat>
#include <condition_variable>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <functional>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "bm3d_b200.h"
#include "bm3d_device.cuh"
#include "bm3d_internal.h"

using namespace bm3d;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define CUDA_TRY(expr)                                                                      \
    do {                                                                                    \
        cudaError_t e_ = (expr);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail(BM3D_B200_ERR_CUDA, "BM3D: '%s' failed: %s", #expr,               \
                        cudaGetErrorString(e_));                                            \
    } while (0)

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

int check_search(int width, int height, int stride, int block_step, int bm_range, int radius,
                 int ps_num, int ps_range) {
    if (width < 8 || height < 8)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: plane must be at least 8x8 (got %dx%d)", width,
                    height);
    if (width > BM3D_B200_MAX_DIM || height > BM3D_B200_MAX_DIM)
        return fail(BM3D_B200_ERR_UNSUPPORTED, "BM3D: plane sides above %d are not supported",
                    BM3D_B200_MAX_DIM);
    if (stride < width) return fail(BM3D_B200_ERR_INVALID, "BM3D: stride smaller than width");
    if (block_step <= 0 || block_step > 8)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: \"block_step\" must be in range [1, 8]");
    if (bm_range <= 0) return fail(BM3D_B200_ERR_INVALID, "BM3D: \"bm_range\" must be positive");
    if (radius < 0) return fail(BM3D_B200_ERR_INVALID, "BM3D: \"radius\" must be non-negative");
    if (radius > BM3D_B200_MAX_RADIUS)
        return fail(BM3D_B200_ERR_UNSUPPORTED, "BM3D: \"radius\" above %d is not supported",
                    BM3D_B200_MAX_RADIUS);
    if (ps_num <= 0 || ps_num > 8)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: \"ps_num\" must be in range [1, 8]");
    if (ps_range <= 0) return fail(BM3D_B200_ERR_INVALID, "BM3D: \"ps_range\" must be positive");
    MatchGeometry g = match_geometry(width, height, block_step, bm_range, radius, ps_range);
    if (g.smem > 220 * 1024)
        return fail(BM3D_B200_ERR_UNSUPPORTED,
                    "BM3D: search range too large for the on-chip tile (bm_range + radius * "
                    "ps_range = %d)",
                    bm_range + radius * ps_range);
    return BM3D_B200_OK;
}

MatchParams make_match_params(const MatchGeometry &g, const float *const *d_frames, int *d_matches,
                              int width, int height, int stride, int block_step, int bm_range,
                              int radius, int ps_num, int ps_range) {
    MatchParams p{};
    p.frames = d_frames;
    p.matches = d_matches;
    p.width = width;
    p.height = height;
    p.stride = stride;
    p.block_step = block_step;
    p.bm_range = bm_range;
    p.radius = radius;
    p.ps_num = ps_num;
    p.ps_range = ps_range;
    p.nbx = g.nbx;
    p.nby = g.nby;
    p.pitch = g.pitch;
    p.tile_rows = g.tile_rows;
    p.extra_cols = g.extra_cols;
    p.nsub_s = g.nsub_s;
    p.nsub_t = g.nsub_t;
    return p;
}

int unpack_matches(const std::vector<int> &packed, int *h_xyz, int nblk) {
    for (int b = 0; b < nblk; ++b)
        for (int k = 0; k < 8; ++k) {
            const int q = packed[(size_t)b * 8 + k];
            h_xyz[((size_t)b * 8 + k) * 3 + 0] = pos_x(q);
            h_xyz[((size_t)b * 8 + k) * 3 + 1] = pos_y(q);
            h_xyz[((size_t)b * 8 + k) * 3 + 2] = pos_z(q);
        }
    return BM3D_B200_OK;
}

}  // namespace

// ===========================================================================
// common
// ===========================================================================
extern "C" const char *bm3d_b200_last_error(void) { return g_last_error.c_str(); }

namespace bm3d {
// Error reporting for the other translation units of the ABI.
int abi_fail(int code, const char *msg) {
    g_last_error = msg;
    return code;
}
}  // namespace bm3d

extern "C" int bm3d_b200_abi_version(void) { return 1; }

extern "C" float bm3d_b200_scale_sigma(float sigma, int final_) {
    sigma *= (3.0f / 4.0f) / 255.0f * 64.0f * (final_ ? 1.0f : 2.7f);
    return sigma;
}

// ===========================================================================
// 1. reference graph replacement
// ===========================================================================
struct bm3d_b200_graph {
    int device = 0;
    float *d_res = nullptr, *d_src = nullptr, *h_res = nullptr;
    int width = 0, height = 0, stride = 0;
    float sigma[3] = {0, 0, 0};
    int block_step = 8, bm_range = 9, radius = 0, ps_num = 2, ps_range = 4;
    bool chroma = false, final_ = false;
    float extractor = 0.0f;
    int nplanes = 1;
    int metric = 0, tx2 = 0, tx1 = 0;  // run-time-compiled plugin variants
    MatchGeometry geo{};
    int *d_matches = nullptr;
    void **d_tab = nullptr;  // [mframes tw][src np*tw][ref np*tw][acc np*tw]
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t exec_full = nullptr, exec_dev = nullptr;
};

namespace {

int graph_enqueue(bm3d_b200_graph *g, cudaStream_t s, bool copies) {
    const int tw = 2 * g->radius + 1;
    const size_t plane = (size_t)g->height * g->stride;
    const size_t pitch = (size_t)g->stride * sizeof(float);
    if (copies) {
        const size_t rows = (size_t)(g->final_ ? 2 : 1) * g->nplanes * tw * g->height;
        CUDA_TRY(cudaMemcpy2DAsync(g->d_src, pitch, g->h_res, pitch, g->width * sizeof(float), rows,
                                   cudaMemcpyHostToDevice, s));
    }
    CUDA_TRY(cudaMemsetAsync(g->d_res, 0, (size_t)g->nplanes * tw * 2 * plane * sizeof(float), s));
    const float *const *tab = reinterpret_cast<const float *const *>(g->d_tab);
    MatchParams mp = make_match_params(g->geo, tab, g->d_matches, g->width, g->height, g->stride,
                                       g->block_step, g->bm_range, g->radius, g->ps_num,
                                       g->ps_range);
    mp.metric = g->metric;
    CUDA_TRY(launch_match(mp, g->geo, 1, s));
    for (int q = 0; q < g->nplanes; ++q) {
        if (g->chroma && g->sigma[q] < FLT_EPSILON) continue;
        FilterParams fp{};
        fp.src = tab + tw + (size_t)q * tw;
        fp.ref = g->final_ ? tab + tw + (size_t)g->nplanes * tw + (size_t)q * tw : nullptr;
        fp.acc = reinterpret_cast<float *const *>(g->d_tab + tw + (size_t)2 * g->nplanes * tw +
                                                  (size_t)q * tw);
        fp.mult = nullptr;
        fp.matches = g->d_matches;
        fp.weight_offset = (long long)plane;
        fp.acc_stride = g->stride;
        fp.stride = g->stride;
        fp.radius = g->radius;
        fp.nblk = g->geo.nbx * g->geo.nby;
        fp.nbx = g->geo.nbx;
        fp.corner_weight = 0;
        fp.nwin = 1;
        fp.sigma = g->sigma[q];
        fp.extractor = g->extractor;
        fp.t2d = g->tx2;
        fp.t1d = g->tx1;
        CUDA_TRY(launch_filter(fp, g->final_, s));
    }
    if (copies) {
        const size_t rows = (size_t)g->nplanes * tw * 2 * g->height;
        CUDA_TRY(cudaMemcpy2DAsync(g->h_res, pitch, g->d_res, pitch, g->width * sizeof(float), rows,
                                   cudaMemcpyDeviceToHost, s));
    }
    return BM3D_B200_OK;
}

int graph_capture(bm3d_b200_graph *g, bool copies, cudaGraphExec_t *exec) {
    CUDA_TRY(cudaStreamBeginCapture(g->cap_stream, cudaStreamCaptureModeThreadLocal));
    int rc = graph_enqueue(g, g->cap_stream, copies);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(g->cap_stream, &graph);
    if (rc != BM3D_B200_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (e != cudaSuccess)
        return fail(BM3D_B200_ERR_CUDA, "BM3D: graph capture failed: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess)
        return fail(BM3D_B200_ERR_CUDA, "BM3D: graph instantiation failed: %s",
                    cudaGetErrorString(e));
    return BM3D_B200_OK;
}

}  // namespace

static int graph_create_impl(bm3d_b200_graph **out, float *d_res, float *d_src, float *h_res,
                             int width, int height, int stride, float sigma, int block_step,
                             int bm_range, int radius, int ps_num, int ps_range, int chroma,
                             float sigma_u, float sigma_v, int final_, float extractor,
                             int bm_error, int transform_2d, int transform_1d) {
    if (!out) return fail(BM3D_B200_ERR_INVALID, "BM3D: null output handle");
    *out = nullptr;
    if (!d_res || !d_src) return fail(BM3D_B200_ERR_INVALID, "BM3D: null device buffer");
    if (int rc = check_search(width, height, stride, block_step, bm_range, radius, ps_num,
                              ps_range))
        return rc;
    if (!(sigma >= 0.0f) || !(sigma_u >= 0.0f) || !(sigma_v >= 0.0f))
        return fail(BM3D_B200_ERR_INVALID, "BM3D: \"sigma\" must be non-negative");
    auto *g = new (std::nothrow) bm3d_b200_graph;
    if (!g) return fail(BM3D_B200_ERR_NOMEM, "BM3D: out of host memory");
    cudaGetDevice(&g->device);
    g->d_res = d_res;
    g->d_src = d_src;
    g->h_res = h_res;
    g->width = width;
    g->height = height;
    g->stride = stride;
    g->sigma[0] = sigma;
    g->sigma[1] = sigma_u;
    g->sigma[2] = sigma_v;
    g->block_step = block_step;
    g->bm_range = bm_range;
    g->radius = radius;
    g->ps_num = ps_num;
    g->ps_range = ps_range;
    g->chroma = chroma != 0;
    g->final_ = final_ != 0;
    g->extractor = extractor;
    g->nplanes = chroma ? 3 : 1;
    g->metric = bm_error;
    g->tx2 = transform_2d;
    g->tx1 = transform_1d;
    g->geo = match_geometry(width, height, block_step, bm_range, radius, ps_range);

    auto cleanup = [&](int rc) {
        bm3d_b200_graph_destroy(g);
        return rc;
    };
    const int tw = 2 * radius + 1;
    const size_t nblk = (size_t)g->geo.nbx * g->geo.nby;
    cudaError_t e = cudaMalloc(&g->d_matches, nblk * 8 * sizeof(int));
    if (e != cudaSuccess)
        return cleanup(fail(BM3D_B200_ERR_CUDA, "BM3D: cudaMalloc failed: %s", cudaGetErrorString(e)));
    const size_t ntab = (size_t)tw * (1 + 3 * g->nplanes);
    e = cudaMalloc(&g->d_tab, ntab * sizeof(void *));
    if (e != cudaSuccess)
        return cleanup(fail(BM3D_B200_ERR_CUDA, "BM3D: cudaMalloc failed: %s", cudaGetErrorString(e)));
    // pointer tables into the reference layouts of d_src / d_res
    std::vector<void *> tab(ntab, nullptr);
    const size_t plane = (size_t)height * stride;
    const int np = g->nplanes;
    auto src_plane = [&](int half, int q, int z) {
        return (void *)(d_src + (((size_t)half * np + q) * tw + z) * plane);
    };
    for (int z = 0; z < tw; ++z) tab[z] = src_plane(0, 0, z);  // ref clip (final) or src (basic)
    for (int q = 0; q < np; ++q)
        for (int z = 0; z < tw; ++z) {
            tab[tw + (size_t)q * tw + z] = src_plane(g->final_ ? 1 : 0, q, z);
            tab[tw + (size_t)np * tw + (size_t)q * tw + z] = g->final_ ? src_plane(0, q, z) : nullptr;
            tab[tw + (size_t)2 * np * tw + (size_t)q * tw + z] =
                (void *)(d_res + (((size_t)q * tw + z) * 2) * plane);
        }
    e = cudaMemcpy(g->d_tab, tab.data(), ntab * sizeof(void *), cudaMemcpyHostToDevice);
    if (e != cudaSuccess)
        return cleanup(fail(BM3D_B200_ERR_CUDA, "BM3D: cudaMemcpy failed: %s", cudaGetErrorString(e)));
    e = cudaStreamCreateWithFlags(&g->cap_stream, cudaStreamNonBlocking);
    if (e != cudaSuccess)
        return cleanup(fail(BM3D_B200_ERR_CUDA, "BM3D: cudaStreamCreate failed: %s",
                            cudaGetErrorString(e)));
    // set kernel attributes outside of capture, then build both graphs
    if (int rc = graph_enqueue(g, g->cap_stream, false)) return cleanup(rc);
    e = cudaStreamSynchronize(g->cap_stream);
    if (e != cudaSuccess)
        return cleanup(fail(BM3D_B200_ERR_CUDA, "BM3D: warm-up failed: %s", cudaGetErrorString(e)));
    if (h_res) {
        if (int rc = graph_capture(g, true, &g->exec_full)) return cleanup(rc);
    }
    if (int rc = graph_capture(g, false, &g->exec_dev)) return cleanup(rc);
    *out = g;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_graph_create(bm3d_b200_graph **out, float *d_res, float *d_src,
                                      float *h_res, int width, int height, int stride, float sigma,
                                      int block_step, int bm_range, int radius, int ps_num,
                                      int ps_range, int chroma, float sigma_u, float sigma_v,
                                      int final_, float extractor) {
    return graph_create_impl(out, d_res, d_src, h_res, width, height, stride, sigma, block_step,
                             bm_range, radius, ps_num, ps_range, chroma, sigma_u, sigma_v, final_,
                             extractor, BM3D_B200_BM_SSD, BM3D_B200_TX_DCT, BM3D_B200_TX_DCT);
}

extern "C" int bm3d_b200_graph_create_rtc(bm3d_b200_graph **out, float *d_res, float *d_src,
                                          float *h_res, int width, int height, int stride,
                                          float sigma, int block_step, int bm_range, int radius,
                                          int ps_num, int ps_range, int chroma, float sigma_u,
                                          float sigma_v, int final_, float extractor,
                                          int bm_error, int transform_2d, int transform_1d) {
    if (out) *out = nullptr;
    if (bm_error < BM3D_B200_BM_SSD || bm_error > BM3D_B200_BM_SSD_NORM)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'bm_error_s': %d", bm_error);
    if (transform_2d < BM3D_B200_TX_DCT || transform_2d > BM3D_B200_TX_BIOR1_5)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'transform_2d_s': %d", transform_2d);
    if (transform_1d < BM3D_B200_TX_DCT || transform_1d > BM3D_B200_TX_BIOR1_5)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'transform_1d_s': %d", transform_1d);
    return graph_create_impl(out, d_res, d_src, h_res, width, height, stride, sigma, block_step,
                             bm_range, radius, ps_num, ps_range, chroma, sigma_u, sigma_v, final_,
                             extractor, bm_error, transform_2d, transform_1d);
}

extern "C" int bm3d_b200_graph_launch(bm3d_b200_graph *g, void *stream) {
    if (!g) return fail(BM3D_B200_ERR_INVALID, "BM3D: null graph");
    if (!g->exec_full) return fail(BM3D_B200_ERR_INVALID, "BM3D: graph created without h_res");
    CUDA_TRY(cudaGraphLaunch(g->exec_full, as_stream(stream)));
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_graph_launch_device(bm3d_b200_graph *g, void *stream) {
    if (!g) return fail(BM3D_B200_ERR_INVALID, "BM3D: null graph");
    CUDA_TRY(cudaGraphLaunch(g->exec_dev, as_stream(stream)));
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_graph_matches(bm3d_b200_graph *g, int *h_xyz, int capacity_blocks,
                                       int *nblocks) {
    if (!g || !h_xyz) return fail(BM3D_B200_ERR_INVALID, "BM3D: null argument");
    const int nblk = g->geo.nbx * g->geo.nby;
    if (nblocks) *nblocks = nblk;
    if (capacity_blocks < nblk) return fail(BM3D_B200_ERR_INVALID, "BM3D: match buffer too small");
    std::vector<int> packed((size_t)nblk * 8);
    CUDA_TRY(cudaDeviceSynchronize());
    CUDA_TRY(cudaMemcpy(packed.data(), g->d_matches, packed.size() * sizeof(int),
                        cudaMemcpyDeviceToHost));
    return unpack_matches(packed, h_xyz, nblk);
}

extern "C" void bm3d_b200_graph_destroy(bm3d_b200_graph *g) {
    if (!g) return;
    if (g->exec_full) cudaGraphExecDestroy(g->exec_full);
    if (g->exec_dev) cudaGraphExecDestroy(g->exec_dev);
    if (g->cap_stream) cudaStreamDestroy(g->cap_stream);
    if (g->d_matches) cudaFree(g->d_matches);
    if (g->d_tab) cudaFree(g->d_tab);
    delete g;
}

// ===========================================================================
// 2. aggregation
// ===========================================================================
extern "C" int bm3d_b200_aggregate(float *d_dst, int dst_stride, const float *d_res,
                                   int res_stride, int width, int height, void *stream) {
    if (!d_dst || !d_res || width <= 0 || height <= 0 || dst_stride < width || res_stride < width)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid aggregation arguments");
    AggregateParams p{};
    p.dst = d_dst;
    p.wdst = d_res;
    p.weight_offset = (long long)height * res_stride;
    p.dst_stride = dst_stride;
    p.acc_stride = res_stride;
    p.width = width;
    p.height = height;
    p.nplanes = 1;
    CUDA_TRY(launch_aggregate(p, as_stream(stream)));
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_vaggregate(float *d_dst, int dst_stride, const float *const *vframes,
                                    int raw_stride, int width, int height, int radius, int n,
                                    int num_frames, void *stream) {
    if (!d_dst || !vframes || width <= 0 || height <= 0 || dst_stride < width ||
        raw_stride < width || radius < 0 || num_frames <= 0 || n < 0 || n >= num_frames)
        return fail(BM3D_B200_ERR_INVALID, "VAggregate: invalid arguments");
    if (radius > BM3D_B200_MAX_RADIUS)
        return fail(BM3D_B200_ERR_UNSUPPORTED, "VAggregate: radius above %d", BM3D_B200_MAX_RADIUS);
    VAggregateParams p{};
    p.dst = d_dst;
    for (int i = 0; i < 2 * radius + 1; ++i) {
        if (!vframes[i]) return fail(BM3D_B200_ERR_INVALID, "VAggregate: null frame pointer");
        p.vf[i] = vframes[i];
    }
    p.dst_stride = dst_stride;
    p.raw_stride = raw_stride;
    p.width = width;
    p.height = height;
    p.radius = radius;
    p.n0 = n;
    p.num_frames = num_frames;
    p.nout = 1;
    CUDA_TRY(launch_vaggregate(p, as_stream(stream)));
    return BM3D_B200_OK;
}

// ===========================================================================
// 3. device-resident clip pipeline
// ===========================================================================
struct bm3d_b200_clip {
    int device = 0;
    int width = 0, height = 0, nplanes = 1, ssw = 0, ssh = 0, nframes = 0;
    bm3d_b200_params prm{};
    int stride = 0;
    int pw[3] = {0, 0, 0}, ph[3] = {0, 0, 0};
    long long poff[3] = {0, 0, 0};     // plane offsets within a source frame
    long long rawoff[3] = {0, 0, 0};   // plane offsets within a raw output frame
    long long frame_floats = 0, raw_frame_floats = 0;
    bool process[3] = {false, false, false};
    float sigma_basic[3] = {0, 0, 0}, sigma_final[3] = {0, 0, 0};
    MatchGeometry geo[3]{};
    int *d_matches = nullptr;
    float *d_acc = nullptr;   // [N][2][H][stride] accumulators of one plane
    float *d_mult = nullptr;  // [N][2r+1]
    void **d_tab = nullptr;   // 5 tables of N*(2r+1) pointers
    float *d_basic = nullptr, *d_io_src = nullptr, *d_io_ref = nullptr, *d_io_dst = nullptr;
    size_t io_dst_floats = 0;
    cudaStream_t stream = nullptr;
    // pipelined host two-stage path (allocated on first use)
    float *d_acc2 = nullptr;   // final-stage accumulators
    void **d_ptab = nullptr;   // 8 tables of N*(2r+1) pointers (basic, final)
    float *d_pmult = nullptr;  // 2 tables of N*(2r+1) multiplicities
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaStream_t s_fin = nullptr;  // final stage, overlapping the basic stage of later chunks
    cudaEvent_t ev_in = nullptr, ev_out = nullptr, ev_bas = nullptr, ev_fin = nullptr;
    // the last call's completion on its stream: every call waits for it first,
    // since the clip's buffers and tables are shared by its calls
    cudaEvent_t ev_done = nullptr;
    // per-stage CUDA-event timers (bm3d_b200_clip_set_profiling)
    bool profiling = false;
    struct Mark {
        int stage;
        cudaEvent_t a, b;
        int kernels;  // kernel launches between a and b
    };
    std::vector<Mark> marks;
    double stage_ms[BM3D_B200_NUM_STAGES] = {};
    long long stage_launches[BM3D_B200_NUM_STAGES] = {};
    // learned matching (bm3d_b200_clip_set_proposer)
    bm3d_b200_proposer *prop = nullptr;
    int cells_s = 4, cells_t = 4;
    float fb_tau = 0.0f;
    MatchGeometry lgeo{};
    uint8_t *d_emb = nullptr;     // [2][N][h/2][w/2][16] bytes: basic-stage src, final-stage ref
    void **d_etab = nullptr;      // [2][N*(2r+1)] embedding pointer per window slot
    unsigned *d_fb = nullptr;     // [2][N * nblk] blocks listed for the exhaustive re-search
    unsigned *d_fbcount = nullptr;  // [2] (basic, final: the two stages may run concurrently)
    size_t fb_stride = 0;
    unsigned long long *d_fbtotal = nullptr;
    long long stat_blocks = 0;
    // final stage of a two-stage run with a proposer: 0 learned search on the
    // basic estimate, 1 the basic stage's lists re-scored on it
    int final_matching = 0;
    int precision = 0;  // filter transform: 0 FP32 (reference factorisation), 1 split-BF16,
                        // 2 FP16 Kronecker form on tcgen05
    unsigned *h_tcerr = nullptr, *d_tcerr = nullptr;  // precision 2 error word (mapped host)
    // run-time-compiled plugin variants per plane (bm3d_b200_clip_set_variant)
    int metric[3] = {0, 0, 0}, tx2[3] = {0, 0, 0}, tx1[3] = {0, 0, 0};
};

namespace {

int clip_check(const bm3d_b200_clip *c);

// Orders a call's work on `s` after the clip's previous call, whatever stream
// that used (not while `s` is being captured into a graph).
int clip_begin(bm3d_b200_clip *c, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(s, &cs));
    if (cs != cudaStreamCaptureStatusNone) return BM3D_B200_OK;
    if (!c->ev_done) CUDA_TRY(cudaEventCreateWithFlags(&c->ev_done, cudaEventDisableTiming));
    CUDA_TRY(cudaStreamWaitEvent(s, c->ev_done, 0));
    return BM3D_B200_OK;
}
int clip_end(bm3d_b200_clip *c, cudaStream_t s) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CUDA_TRY(cudaStreamIsCapturing(s, &cs));
    if (cs == cudaStreamCaptureStatusNone && c->ev_done) CUDA_TRY(cudaEventRecord(c->ev_done, s));
    return BM3D_B200_OK;
}

// Records `launch` (`kernels` kernel launches) between two events on `s`
// when profiling is on.
template <typename F>
int timed(bm3d_b200_clip *c, int stage, cudaStream_t s, F &&launch, int kernels = 1) {
    if (!c->profiling) {
        CUDA_TRY(launch());
        return BM3D_B200_OK;
    }
    bm3d_b200_clip::Mark m{stage, nullptr, nullptr, kernels};
    CUDA_TRY(cudaEventCreate(&m.a));
    CUDA_TRY(cudaEventCreate(&m.b));
    c->marks.push_back(m);
    CUDA_TRY(cudaEventRecord(m.a, s));
    CUDA_TRY(launch());
    CUDA_TRY(cudaEventRecord(m.b, s));
    return BM3D_B200_OK;
}

}  // namespace

extern "C" void bm3d_b200_params_default(bm3d_b200_params *p) {
    if (!p) return;
    for (int i = 0; i < 3; ++i) {
        p->sigma[i] = 3.0f;
        p->block_step[i] = 8;
        p->bm_range[i] = 9;
        p->ps_num[i] = 2;
        p->ps_range[i] = 4;
    }
    p->radius = 0;
    p->chroma = 0;
    p->extractor_exp = 0;
    p->zero_init = 1;
}

namespace {

float extractor_of(int e) { return e ? std::ldexp(1.0f, e) : 0.0f; }

// Which plane's search parameters drive a plane job (chroma: plane 0).
int job_params_plane(const bm3d_b200_clip *c, int q) { return c->prm.chroma ? 0 : q; }

__global__ void add_count_kernel(const unsigned *count, unsigned long long *total) {
    atomicAdd(total, (unsigned long long)*count);
}

// FP16 proposer embeddings of frames [f0, f1) of plane 0 of `clip` into
// embedding set `which` (0: basic-stage source, 1: final-stage reference).
int embed_frames(bm3d_b200_clip *c, int which, const float *clip, int f0, int f1,
                 cudaStream_t s) {
    if (f1 <= f0) return BM3D_B200_OK;
    const long long ef = (long long)(c->pw[0] / 2) * (c->ph[0] / 2) * 16;
    uint8_t *dst = c->d_emb + ((size_t)which * c->nframes + f0) * ef;
    return timed(c, BM3D_B200_STAGE_PROPOSE, s, [&] {
        return launch_embed(clip + (size_t)f0 * c->frame_floats + c->poff[0], c->frame_floats,
                            f1 - f0, c->pw[0], c->ph[0], c->stride, proposer_frag(c->prop),
                            proposer_bias(c->prop), dst, ef, proposer_err(c->prop), s);
    });
}

// Learned block matching of windows [mp.win0, mp.win0 + nwin) of plane 0
// with embedding set `which`, then the exhaustive re-search of the blocks it
// lists. mp carries the exhaustive geometry; the learned tile replaces it.
int learned_windows(bm3d_b200_clip *c, MatchParams mp, int which, int nwin, cudaStream_t s) {
    const size_t ntab = (size_t)c->nframes * (2 * c->prm.radius + 1);
    const int nblk = mp.nbx * mp.nby;
    LearnedParams lp{};
    lp.embs = reinterpret_cast<const void *const *>(c->d_etab + which * ntab);
    lp.w2 = c->pw[0] / 2;
    lp.cells_s = c->cells_s;
    lp.cells_t = c->cells_t;
    const float sg = c->prm.sigma[0] / 255.0f;
    lp.fallback_ssd = c->fb_tau > 0.0f ? c->fb_tau * 128.0f * sg * sg : 0.0f;
    unsigned *fb = c->d_fb + (size_t)which * c->fb_stride;
    unsigned *fbcount = c->d_fbcount + which;
    lp.fallback = fb;
    lp.fallback_count = fbcount;
    lp.fallback_capacity = (unsigned)((size_t)c->nframes * nblk);
    MatchParams lm = mp;
    lm.pitch = c->lgeo.pitch;
    lm.tile_rows = c->lgeo.tile_rows;
    CUDA_TRY(cudaMemsetAsync(fbcount, 0, sizeof(unsigned), s));
    if (int rc = timed(c, which ? BM3D_B200_STAGE_MATCH_FINAL : BM3D_B200_STAGE_MATCH, s,
                       [&] { return launch_learned_match(lm, lp, c->lgeo, nwin, s); }))
        return rc;
    c->stat_blocks += (long long)nwin * nblk;
    if (!(lp.fallback_ssd > 0.0f)) return BM3D_B200_OK;
    return timed(c, BM3D_B200_STAGE_FALLBACK, s, [&]() -> cudaError_t {
        cudaError_t e = launch_match_fallback(mp, fb, fbcount, s);
        if (e != cudaSuccess) return e;
        add_count_kernel<<<1, 1, 0, s>>>(fbcount, c->d_fbtotal);
        return cudaGetLastError();
    }, 2);
}

// The final stage's lists from the basic stage's (windows [mp.win0, mp.win0 +
// nwin)), re-scored on the final stage's matching planes.
int rescore_windows(bm3d_b200_clip *c, const MatchParams &mp, int nwin, cudaStream_t s) {
    const int nblk = mp.nbx * mp.nby;
    return timed(c, BM3D_B200_STAGE_MATCH_FINAL, s, [&]() -> cudaError_t {
        c->stat_blocks += (long long)nwin * nblk;
        return launch_rescore(mp, nwin, s);
    });
}

// basic_lists: d_matches holds this clip's basic-stage lists of every window
// (the final half of a two-stage run), which the final stage may re-score.
int clip_run_impl(bm3d_b200_clip *c, const float *d_src, const float *d_ref, float *d_dst,
                  int dst_mode, cudaStream_t s, bool basic_lists = false) {
    const int N = c->nframes;
    const int r = c->prm.radius;
    const int tw = 2 * r + 1;
    const bool final_ = d_ref != nullptr;
    const bool raw = dst_mode == BM3D_B200_DST_RAW && r > 0;
    const size_t ntab = (size_t)N * tw;
    std::vector<void *> tab(5 * ntab, nullptr);
    std::vector<float> mult(ntab, 1.0f);
    auto clampf = [&](int f) { return std::min(std::max(f, 0), N - 1); };

    // zero-init / pass-through of unprocessed planes
    if (raw) {
        for (int q = 0; q < c->nplanes; ++q) {
            if (c->process[q] || !c->prm.zero_init) continue;
            const size_t rows = (size_t)tw * 2 * c->ph[q];
            CUDA_TRY(cudaMemset2DAsync(d_dst + c->rawoff[q], c->raw_frame_floats * sizeof(float), 0,
                                       rows * c->stride * sizeof(float), N, s));
        }
    } else {
        for (int q = 0; q < c->nplanes; ++q) {
            if (c->process[q]) continue;
            CUDA_TRY(cudaMemcpy2DAsync(d_dst + c->poff[q], c->frame_floats * sizeof(float),
                                       d_src + c->poff[q], c->frame_floats * sizeof(float),
                                       (size_t)c->ph[q] * c->stride * sizeof(float), N,
                                       cudaMemcpyDeviceToDevice, s));
        }
    }

    // plane jobs: chroma -> one job over 3 planes matching on plane 0
    const int njobs = c->prm.chroma ? 1 : c->nplanes;
    for (int job = 0; job < njobs; ++job) {
        const int mq = c->prm.chroma ? 0 : job;  // matching plane
        if (!c->prm.chroma && !c->process[mq]) continue;
        if (c->prm.chroma && !(c->process[0] || c->process[1] || c->process[2])) continue;
        const int pq = job_params_plane(c, mq);
        const MatchGeometry &g = c->geo[mq];
        const int W = c->pw[mq], H = c->ph[mq];
        const float *mclip = final_ ? d_ref : d_src;
        for (int n = 0; n < N; ++n)
            for (int z = 0; z < tw; ++z)
                tab[(size_t)n * tw + z] =
                    (void *)(mclip + (size_t)clampf(n - r + z) * c->frame_floats + c->poff[mq]);
        // planes filtered by this job
        const int q_first = c->prm.chroma ? 0 : mq;
        const int q_last = c->prm.chroma ? 2 : mq;
        // upload the matching table first (filter tables are rebuilt per plane)
        const float *const *d_mtab = reinterpret_cast<const float *const *>(c->d_tab);
        CUDA_TRY(cudaMemcpyAsync(c->d_tab, tab.data(), ntab * sizeof(void *),
                                 cudaMemcpyHostToDevice, s));
        MatchParams mp = make_match_params(g, d_mtab, c->d_matches, W, H, c->stride,
                                           c->prm.block_step[pq], c->prm.bm_range[pq], r,
                                           c->prm.ps_num[pq], c->prm.ps_range[pq]);
        mp.metric = c->metric[pq];
        if (c->prop && mq == 0 && final_ && basic_lists && c->final_matching != 0 &&
            !c->prm.chroma) {
            if (c->final_matching == BM3D_B200_FINAL_MATCH_BASIC_LISTS)
                if (int rc = rescore_windows(c, mp, N, s)) return rc;
        } else if (c->prop && mq == 0) {
            if (int rc = embed_frames(c, final_ ? 1 : 0, mclip, 0, N, s)) return rc;
            if (int rc = learned_windows(c, mp, final_ ? 1 : 0, N, s)) return rc;
        } else if (int rc = timed(c, final_ ? BM3D_B200_STAGE_MATCH_FINAL : BM3D_B200_STAGE_MATCH,
                                  s, [&] { return launch_match(mp, g, N, s); })) {
            return rc;
        }
        for (int q = q_first; q <= q_last; ++q) {
            const float sigma = final_ ? c->sigma_final[q] : c->sigma_basic[q];
            if (c->prm.chroma && sigma < FLT_EPSILON) continue;
            if (!c->process[q]) continue;
            const int Hq = c->ph[q];
            const size_t plane = (size_t)Hq * c->stride;
            void **src_t = tab.data() + ntab, **ref_t = tab.data() + 2 * ntab,
                 **acc_t = tab.data() + 3 * ntab;
            for (int n = 0; n < N; ++n)
                for (int z = 0; z < tw; ++z) {
                    const size_t k = (size_t)n * tw + z;
                    const size_t f = (size_t)clampf(n - r + z);
                    src_t[k] = (void *)(d_src + f * c->frame_floats + c->poff[q]);
                    ref_t[k] = final_ ? (void *)(d_ref + f * c->frame_floats + c->poff[q]) : nullptr;
                    mult[k] = 1.0f;
                    if (raw) {
                        acc_t[k] = (void *)(d_dst + (size_t)n * c->raw_frame_floats + c->rawoff[q] +
                                            (size_t)z * 2 * plane);
                    } else if (r == 0) {
                        acc_t[k] = (void *)(c->d_acc + (size_t)n * 2 * plane);
                    } else {
                        acc_t[k] = nullptr;
                        mult[k] = 0.0f;
                    }
                }
            if (!raw && r > 0) {
                // VAggregate of frame m sums slab s_i of frame f_i for i = 0..2r
                // (source/source.cpp:830-844); route each slab straight into
                // frame m's accumulator, counting repeats.
                for (int m = 0; m < N; ++m)
                    for (int i = 0; i < tw; ++i) {
                        const int f = clampf(m - r + i);
                        const int sidx = std::min(std::max(2 * r - i, m - N + 1 + r), m + r);
                        const size_t k = (size_t)f * tw + sidx;
                        acc_t[k] = (void *)(c->d_acc + (size_t)m * 2 * plane);
                        mult[k] += 1.0f;
                    }
            }
            CUDA_TRY(cudaMemcpyAsync(c->d_tab + ntab, tab.data() + ntab, 3 * ntab * sizeof(void *),
                                     cudaMemcpyHostToDevice, s));
            CUDA_TRY(cudaMemcpyAsync(c->d_mult, mult.data(), ntab * sizeof(float),
                                     cudaMemcpyHostToDevice, s));
            if (raw) {
                CUDA_TRY(cudaMemset2DAsync(d_dst + c->rawoff[q], c->raw_frame_floats * sizeof(float),
                                           0, (size_t)tw * 2 * plane * sizeof(float), N, s));
            } else {
                CUDA_TRY(cudaMemsetAsync(c->d_acc, 0, (size_t)N * 2 * plane * sizeof(float), s));
            }
            FilterParams fp{};
            fp.src = reinterpret_cast<const float *const *>(c->d_tab + ntab);
            fp.ref = final_ ? reinterpret_cast<const float *const *>(c->d_tab + 2 * ntab) : nullptr;
            fp.acc = reinterpret_cast<float *const *>(c->d_tab + 3 * ntab);
            fp.mult = (!raw && r > 0) ? c->d_mult : nullptr;
            fp.matches = c->d_matches;
            fp.weight_offset = (long long)plane;
            fp.acc_stride = c->stride;
            fp.stride = c->stride;
            fp.radius = r;
            fp.nblk = g.nbx * g.nby;
            fp.nbx = g.nbx;
            fp.corner_weight = raw ? 0 : 1;
            fp.nwin = N;
            fp.sigma = sigma;
            fp.extractor = extractor_of(c->prm.extractor_exp);
            fp.precision = c->precision;
            fp.err = c->d_tcerr;
            fp.t2d = c->tx2[c->prm.chroma ? 0 : q];
            fp.t1d = c->tx1[c->prm.chroma ? 0 : q];
            if (int rc = timed(c, final_ ? BM3D_B200_STAGE_FILTER_FINAL : BM3D_B200_STAGE_FILTER,
                               s, [&] { return launch_filter(fp, final_, s); }))
                return rc;
            if (!raw) {
                AggregateParams ap{};
                ap.dst = d_dst + c->poff[q];
                ap.wdst = c->d_acc;
                ap.dst_plane_stride = c->frame_floats;
                ap.acc_plane_stride = (long long)2 * plane;
                ap.weight_offset = (long long)plane;
                ap.dst_stride = c->stride;
                ap.acc_stride = c->stride;
                ap.width = c->pw[q];
                ap.height = Hq;
                ap.nplanes = N;
                ap.corner_weight = 1;
                if (int rc = timed(c, BM3D_B200_STAGE_AGGREGATE, s,
                                   [&] { return launch_aggregate(ap, s); }))
                    return rc;
            }
        }
    }
    return BM3D_B200_OK;
}

}  // namespace

extern "C" int bm3d_b200_clip_create(bm3d_b200_clip **out, int width, int height, int num_planes,
                                     int subsampling_w, int subsampling_h, int num_frames,
                                     const bm3d_b200_params *params, int device_id) {
    if (!out) return fail(BM3D_B200_ERR_INVALID, "BM3D: null output handle");
    *out = nullptr;
    if (!params) return fail(BM3D_B200_ERR_INVALID, "BM3D: null params");
    if (num_planes != 1 && num_planes != 3)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: clips have 1 or 3 planes");
    if (num_frames <= 0) return fail(BM3D_B200_ERR_INVALID, "BM3D: clip has no frames");
    if (subsampling_w < 0 || subsampling_h < 0 || subsampling_w > 2 || subsampling_h > 2)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid subsampling");
    const bm3d_b200_params &p = *params;
    if (p.chroma && (num_planes != 3 || subsampling_w || subsampling_h))
        return fail(BM3D_B200_ERR_INVALID, "BM3D: clip format must be YUV444 when \"chroma\" is true");
    for (int i = 0; i < 3; ++i)
        if (!(p.sigma[i] >= 0.0f)) return fail(BM3D_B200_ERR_INVALID, "BM3D: \"sigma\" must be non-negative");
    // search parameters of every matched plane, before touching the device
    for (int q = 0; q < num_planes; ++q) {
        const int pq = p.chroma ? 0 : q;
        const bool matched = p.chroma ? q == 0 : !(p.sigma[q] < FLT_EPSILON);
        if (!matched) continue;
        const int w = q == 0 ? width : width >> subsampling_w;
        const int h = q == 0 ? height : height >> subsampling_h;
        if (int rc = check_search(w, h, (width + 31) / 32 * 32, p.block_step[pq], p.bm_range[pq],
                                  p.radius, p.ps_num[pq], p.ps_range[pq]))
            return rc;
    }
    int count = 0;
    CUDA_TRY(cudaGetDeviceCount(&count));
    if (device_id < 0 || device_id >= count)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid device ID (%d)", device_id);
    CUDA_TRY(cudaSetDevice(device_id));

    auto *c = new (std::nothrow) bm3d_b200_clip;
    if (!c) return fail(BM3D_B200_ERR_NOMEM, "BM3D: out of host memory");
    auto cleanup = [&](int rc) {
        bm3d_b200_clip_destroy(c);
        return rc;
    };
    c->device = device_id;
    c->width = width;
    c->height = height;
    c->nplanes = num_planes;
    c->ssw = subsampling_w;
    c->ssh = subsampling_h;
    c->nframes = num_frames;
    c->prm = p;
    c->stride = (width + 31) / 32 * 32;
    long long off = 0, roff = 0;
    const int tw = 2 * p.radius + 1;
    for (int q = 0; q < num_planes; ++q) {
        c->pw[q] = q == 0 ? width : width >> subsampling_w;
        c->ph[q] = q == 0 ? height : height >> subsampling_h;
        c->poff[q] = off;
        c->rawoff[q] = roff;
        off += (long long)c->ph[q] * c->stride;
        roff += (long long)c->ph[q] * c->stride * 2 * tw;
        c->process[q] = !(p.sigma[q] < FLT_EPSILON);
        c->sigma_basic[q] = bm3d_b200_scale_sigma(p.sigma[q], 0);
        c->sigma_final[q] = bm3d_b200_scale_sigma(p.sigma[q], 1);
    }
    c->frame_floats = off;
    c->raw_frame_floats = roff;
    size_t max_blk = 0;
    size_t max_plane = 0;
    for (int q = 0; q < num_planes; ++q) {
        const int pq = p.chroma ? 0 : q;
        const bool matched = p.chroma ? q == 0 : c->process[q];
        max_plane = std::max(max_plane, (size_t)c->ph[q] * c->stride);
        if (!matched) continue;
        if (int rc = check_search(c->pw[q], c->ph[q], c->stride, p.block_step[pq], p.bm_range[pq],
                                  p.radius, p.ps_num[pq], p.ps_range[pq]))
            return cleanup(rc);
        c->geo[q] = match_geometry(c->pw[q], c->ph[q], p.block_step[pq], p.bm_range[pq], p.radius,
                                   p.ps_range[pq]);
        max_blk = std::max(max_blk, (size_t)c->geo[q].nbx * c->geo[q].nby);
    }
    if (p.chroma) {
        c->geo[1] = c->geo[2] = c->geo[0];
    }
    const size_t ntab = (size_t)num_frames * tw;
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&c->d_matches, std::max<size_t>(1, max_blk * num_frames) * 8 * sizeof(int));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_acc, (size_t)num_frames * 2 * max_plane * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_mult, ntab * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&c->d_tab, 5 * ntab * sizeof(void *));
    if (e != cudaSuccess)
        return cleanup(fail(BM3D_B200_ERR_CUDA, "BM3D: allocation failed: %s", cudaGetErrorString(e)));
    *out = c;
    return BM3D_B200_OK;
}

extern "C" long long bm3d_b200_clip_frame_floats(const bm3d_b200_clip *c) {
    return c ? c->frame_floats : 0;
}
extern "C" long long bm3d_b200_clip_raw_frame_floats(const bm3d_b200_clip *c) {
    return c ? c->raw_frame_floats : 0;
}
extern "C" int bm3d_b200_clip_stride(const bm3d_b200_clip *c) { return c ? c->stride : 0; }

extern "C" int bm3d_b200_clip_run(bm3d_b200_clip *c, const float *d_src, const float *d_ref,
                                  float *d_dst, int dst_mode, void *stream) {
    if (!c || !d_src || !d_dst) return fail(BM3D_B200_ERR_INVALID, "BM3D: null argument");
    if (dst_mode != BM3D_B200_DST_AGGREGATED && dst_mode != BM3D_B200_DST_RAW)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: unknown dst_mode %d", dst_mode);
    CUDA_TRY(cudaSetDevice(c->device));
    const cudaStream_t s = as_stream(stream);
    if (int rc = clip_begin(c, s)) return rc;
    if (int rc = clip_run_impl(c, d_src, d_ref, d_dst, dst_mode, s)) return rc;
    return clip_end(c, s);
}

namespace {

int ensure_io(bm3d_b200_clip *c, size_t dst_floats, bool need_ref) {
    const size_t src_floats = (size_t)c->nframes * c->frame_floats;
    if (!c->d_io_src) CUDA_TRY(cudaMalloc(&c->d_io_src, src_floats * sizeof(float)));
    if (need_ref && !c->d_io_ref) CUDA_TRY(cudaMalloc(&c->d_io_ref, src_floats * sizeof(float)));
    if (c->io_dst_floats < dst_floats) {
        if (c->d_io_dst) cudaFree(c->d_io_dst);
        c->d_io_dst = nullptr;
        CUDA_TRY(cudaMalloc(&c->d_io_dst, dst_floats * sizeof(float)));
        c->io_dst_floats = dst_floats;
    }
    return BM3D_B200_OK;
}

}  // namespace

extern "C" int bm3d_b200_clip_run_host(bm3d_b200_clip *c, const float *h_src, const float *h_ref,
                                       float *h_dst, int dst_mode, void *stream) {
    if (!c || !h_src || !h_dst) return fail(BM3D_B200_ERR_INVALID, "BM3D: null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t s = stream ? as_stream(stream) : c->stream;
    const bool raw = dst_mode == BM3D_B200_DST_RAW && c->prm.radius > 0;
    const size_t src_floats = (size_t)c->nframes * c->frame_floats;
    const size_t dst_floats = (size_t)c->nframes * (raw ? c->raw_frame_floats : c->frame_floats);
    if (int rc = ensure_io(c, dst_floats, h_ref != nullptr)) return rc;
    if (int rc = clip_begin(c, s)) return rc;
    CUDA_TRY(cudaMemcpyAsync(c->d_io_src, h_src, src_floats * sizeof(float), cudaMemcpyHostToDevice,
                             s));
    if (h_ref)
        CUDA_TRY(cudaMemcpyAsync(c->d_io_ref, h_ref, src_floats * sizeof(float),
                                 cudaMemcpyHostToDevice, s));
    if (int rc = clip_run_impl(c, c->d_io_src, h_ref ? c->d_io_ref : nullptr, c->d_io_dst, dst_mode,
                               s))
        return rc;
    CUDA_TRY(cudaMemcpyAsync(h_dst, c->d_io_dst, dst_floats * sizeof(float), cudaMemcpyDeviceToHost,
                             s));
    if (int rc = clip_end(c, s)) return rc;
    CUDA_TRY(cudaStreamSynchronize(s));
    return clip_check(c);
}

extern "C" int bm3d_b200_clip_twostage(bm3d_b200_clip *c, const float *d_src, float *d_basic,
                                       float *d_dst, void *stream) {
    if (!c || !d_src || !d_basic || !d_dst) return fail(BM3D_B200_ERR_INVALID, "BM3D: null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t s = as_stream(stream);
    if (int rc = clip_begin(c, s)) return rc;
    if (int rc = clip_run_impl(c, d_src, nullptr, d_basic, BM3D_B200_DST_AGGREGATED, s)) return rc;
    if (int rc = clip_run_impl(c, d_src, d_basic, d_dst, BM3D_B200_DST_AGGREGATED, s, true))
        return rc;
    return clip_end(c, s);
}

namespace {

// Device tables of one fused stage of a single-plane clip for all N windows:
// [match frames][src][ref][acc targets] (N*(2r+1) pointers each) and the
// multiplicities; acc targets follow the VAggregate mapping
// (source/source.cpp:830-844) into frame accumulators [N][2][H][stride].
int upload_stage_tables(bm3d_b200_clip *c, void **d_tab, float *d_mult, const float *d_src,
                        const float *d_ref, float *d_acc, cudaStream_t s) {
    const int N = c->nframes, r = c->prm.radius, tw = 2 * r + 1;
    const size_t ntab = (size_t)N * tw;
    const size_t plane = (size_t)c->ph[0] * c->stride;
    std::vector<void *> tab(4 * ntab, nullptr);
    std::vector<float> mult(ntab, r > 0 ? 0.0f : 1.0f);
    auto clampf = [&](int f) { return std::min(std::max(f, 0), N - 1); };
    const float *mclip = d_ref ? d_ref : d_src;
    for (int n = 0; n < N; ++n)
        for (int z = 0; z < tw; ++z) {
            const size_t k = (size_t)n * tw + z;
            const size_t f = (size_t)clampf(n - r + z);
            tab[k] = (void *)(mclip + f * c->frame_floats);
            tab[ntab + k] = (void *)(d_src + f * c->frame_floats);
            tab[2 * ntab + k] = d_ref ? (void *)(d_ref + f * c->frame_floats) : nullptr;
            tab[3 * ntab + k] = r > 0 ? nullptr : (void *)(d_acc + (size_t)n * 2 * plane);
        }
    if (r > 0) {
        for (int m = 0; m < N; ++m)
            for (int i = 0; i < tw; ++i) {
                const int f = clampf(m - r + i);
                const int sidx = std::min(std::max(2 * r - i, m - N + 1 + r), m + r);
                const size_t k = (size_t)f * tw + sidx;
                tab[3 * ntab + k] = (void *)(d_acc + (size_t)m * 2 * plane);
                mult[k] += 1.0f;
            }
    }
    CUDA_TRY(cudaMemcpyAsync(d_tab, tab.data(), tab.size() * sizeof(void *),
                             cudaMemcpyHostToDevice, s));
    CUDA_TRY(cudaMemcpyAsync(d_mult, mult.data(), ntab * sizeof(float), cudaMemcpyHostToDevice, s));
    return BM3D_B200_OK;
}

// Block matching + filtering of windows [w0, w1) of one fused stage.
int run_stage_windows(bm3d_b200_clip *c, void **d_tab, float *d_mult, bool final_, int w0, int w1,
                      cudaStream_t s) {
    if (w1 <= w0) return BM3D_B200_OK;
    const int N = c->nframes, r = c->prm.radius, tw = 2 * r + 1;
    const size_t ntab = (size_t)N * tw;
    const MatchGeometry &g = c->geo[0];
    MatchParams mp = make_match_params(g, reinterpret_cast<const float *const *>(d_tab),
                                       c->d_matches, c->pw[0], c->ph[0], c->stride,
                                       c->prm.block_step[0], c->prm.bm_range[0], r,
                                       c->prm.ps_num[0], c->prm.ps_range[0]);
    mp.win0 = w0;
    mp.metric = c->metric[0];
    if (c->prop && final_ && c->final_matching != 0) {
        if (c->final_matching == BM3D_B200_FINAL_MATCH_BASIC_LISTS)
            if (int rc = rescore_windows(c, mp, w1 - w0, s)) return rc;
    } else if (c->prop) {
        if (int rc = learned_windows(c, mp, final_ ? 1 : 0, w1 - w0, s)) return rc;
    } else if (int rc = timed(c, final_ ? BM3D_B200_STAGE_MATCH_FINAL : BM3D_B200_STAGE_MATCH,
                              s, [&] { return launch_match(mp, g, w1 - w0, s); })) {
        return rc;
    }
    FilterParams fp{};
    fp.src = reinterpret_cast<const float *const *>(d_tab + ntab);
    fp.ref = final_ ? reinterpret_cast<const float *const *>(d_tab + 2 * ntab) : nullptr;
    fp.acc = reinterpret_cast<float *const *>(d_tab + 3 * ntab);
    fp.mult = r > 0 ? d_mult : nullptr;
    fp.matches = c->d_matches;
    fp.weight_offset = (long long)c->ph[0] * c->stride;
    fp.acc_stride = c->stride;
    fp.stride = c->stride;
    fp.radius = r;
    fp.nblk = g.nbx * g.nby;
    fp.nbx = g.nbx;
    fp.win0 = w0;
    fp.nwin = w1 - w0;
    fp.corner_weight = 1;
    fp.sigma = final_ ? c->sigma_final[0] : c->sigma_basic[0];
    fp.extractor = extractor_of(c->prm.extractor_exp);
    fp.precision = c->precision;
    fp.err = c->d_tcerr;
    fp.t2d = c->tx2[0];
    fp.t1d = c->tx1[0];
    return timed(c, final_ ? BM3D_B200_STAGE_FILTER_FINAL : BM3D_B200_STAGE_FILTER, s,
                 [&] { return launch_filter(fp, final_, s); });
}

// dst frames [a0, a1) = accumulators [a0, a1) divided.
int aggregate_frames(bm3d_b200_clip *c, const float *d_acc, float *d_dst, int a0, int a1,
                     cudaStream_t s) {
    if (a1 <= a0) return BM3D_B200_OK;
    const size_t plane = (size_t)c->ph[0] * c->stride;
    AggregateParams ap{};
    ap.dst = d_dst + (size_t)a0 * c->frame_floats;
    ap.wdst = d_acc + (size_t)a0 * 2 * plane;
    ap.dst_plane_stride = c->frame_floats;
    ap.acc_plane_stride = (long long)2 * plane;
    ap.weight_offset = (long long)plane;
    ap.dst_stride = c->stride;
    ap.acc_stride = c->stride;
    ap.width = c->pw[0];
    ap.height = c->ph[0];
    ap.nplanes = a1 - a0;
    ap.corner_weight = 1;
    return timed(c, BM3D_B200_STAGE_AGGREGATE, s, [&] { return launch_aggregate(ap, s); });
}

// Two-stage V-BM3D of a single-plane clip from host to host, software
// pipelined in chunks of windows so that the upload of later frames and the
// download of finished ones overlap the kernels: basic frame m is final once
// windows up to m + r are filtered, final window n can start once basic
// frames up to n + r are final, so each stage trails the previous by r frames.
int twostage_pipelined(bm3d_b200_clip *c, const float *h_src, float *h_dst, cudaStream_t s,
                       bool throughput) {
    const int N = c->nframes, r = c->prm.radius, tw = 2 * r + 1;
    const size_t ntab = (size_t)N * tw;
    const size_t ff = c->frame_floats;
    const size_t plane = (size_t)c->ph[0] * c->stride;
    if (!c->d_acc2) CUDA_TRY(cudaMalloc(&c->d_acc2, (size_t)N * 2 * plane * sizeof(float)));
    if (!c->d_ptab) CUDA_TRY(cudaMalloc(&c->d_ptab, 8 * ntab * sizeof(void *)));
    if (!c->d_pmult) CUDA_TRY(cudaMalloc(&c->d_pmult, 2 * ntab * sizeof(float)));
    if (!c->s_in) CUDA_TRY(cudaStreamCreateWithFlags(&c->s_in, cudaStreamNonBlocking));
    if (!c->s_out) CUDA_TRY(cudaStreamCreateWithFlags(&c->s_out, cudaStreamNonBlocking));
    if (!c->ev_in) CUDA_TRY(cudaEventCreateWithFlags(&c->ev_in, cudaEventDisableTiming));
    if (!c->ev_out) CUDA_TRY(cudaEventCreateWithFlags(&c->ev_out, cudaEventDisableTiming));
    if (!c->s_fin) CUDA_TRY(cudaStreamCreateWithFlags(&c->s_fin, cudaStreamNonBlocking));
    if (!c->ev_bas) CUDA_TRY(cudaEventCreateWithFlags(&c->ev_bas, cudaEventDisableTiming));
    if (!c->ev_fin) CUDA_TRY(cudaEventCreateWithFlags(&c->ev_fin, cudaEventDisableTiming));
    cudaStream_t sf = c->s_fin;
    float *d_src = c->d_io_src, *d_basic = c->d_basic, *d_dst = c->d_io_dst;
    void **tb = c->d_ptab, **tf = c->d_ptab + 4 * ntab;
    float *mb = c->d_pmult, *mf = c->d_pmult + ntab;
    if (int rc = upload_stage_tables(c, tb, mb, d_src, nullptr, c->d_acc, s)) return rc;
    if (int rc = upload_stage_tables(c, tf, mf, d_src, d_basic, c->d_acc2, s)) return rc;
    // the copy streams start after everything already queued on s; the first
    // upload overlaps the clearing of the accumulators, each stage's on the
    // stream that accumulates into it
    CUDA_TRY(cudaEventRecord(c->ev_in, s));
    CUDA_TRY(cudaStreamWaitEvent(c->s_in, c->ev_in, 0));
    CUDA_TRY(cudaStreamWaitEvent(c->s_out, c->ev_in, 0));
    CUDA_TRY(cudaStreamWaitEvent(sf, c->ev_in, 0));
    CUDA_TRY(cudaMemsetAsync(c->d_acc, 0, (size_t)N * 2 * plane * sizeof(float), s));
    CUDA_TRY(cudaMemsetAsync(c->d_acc2, 0, (size_t)N * 2 * plane * sizeof(float), sf));

    // Basic-stage windows advance chunk by chunk; each step uploads what the
    // chunk needs, then runs every later stage as far as its inputs allow and
    // downloads the finished frames. Chunks start at one window, so compute
    // starts after r + 1 frames have arrived, and grow by 2, 4, 5, 6, 6, ...
    // windows; the last two chunks end 2 windows before the clip's end and
    // at it, and the last step splits its final stage, so only the frames of
    // the last windows download after the compute ends (1, 3, 7, 12, 18, 24,
    // 28, 30 for 30 frames: the fastest of the schedules measured for one
    // call at a time). `throughput` (another clip's call in flight, which
    // covers this one's copies): three equal chunks, the least compute
    // (10, 20, 30: 8.05 ms per clip against 8.35 with the latency schedule).
    std::vector<int> ends;
    if (throughput) {
        for (int k = 1; k <= 3; ++k) {
            const int e = (k * N + 2) / 3;
            if (ends.empty() || e > ends.back()) ends.push_back(e);
        }
    } else {
        ends.push_back(std::min(1, N));
        for (int k = 0, w = 1;; ++k) {
            const int next = w + (k == 0 ? 2 : k == 1 ? 4 : k == 2 ? 5 : 6);
            if (next >= N - 2) break;
            ends.push_back(next);
            w = next;
        }
        if (N - 2 > ends.back()) ends.push_back(N - 2);
        if (N > ends.back()) ends.push_back(N);
    }
    int uploaded = 0, basic_done = 0, basic_agg = 0, final_done = 0, final_agg = 0, downloaded = 0;
    // The final stage runs on its own stream: the final windows of one chunk
    // overlap the basic windows of the next, which fills each launch's tail.
    auto advance_final = [&](int fcap) -> int {
        const int f1 = std::min(fcap, basic_agg == N ? N : std::max(0, basic_agg - r));
        if (f1 <= final_done) return BM3D_B200_OK;
        if (int rc = run_stage_windows(c, tf, mf, true, final_done, f1, sf)) return rc;
        final_done = std::max(final_done, f1);
        const int g1 = final_done == N ? N : std::max(0, final_done - r);
        if (int rc = aggregate_frames(c, c->d_acc2, d_dst, final_agg, g1, sf)) return rc;
        final_agg = std::max(final_agg, g1);
        if (final_agg > downloaded) {
            CUDA_TRY(cudaEventRecord(c->ev_fin, sf));
            CUDA_TRY(cudaStreamWaitEvent(c->s_out, c->ev_fin, 0));
            CUDA_TRY(cudaMemcpyAsync(h_dst + (size_t)downloaded * ff, d_dst + (size_t)downloaded * ff,
                                     (size_t)(final_agg - downloaded) * ff * sizeof(float),
                                     cudaMemcpyDeviceToHost, c->s_out));
            downloaded = final_agg;
        }
        return BM3D_B200_OK;
    };
    for (const int w1 : ends) {
        const int need = w1 == N ? N : std::min(N, w1 + r);
        if (need > uploaded) {
            CUDA_TRY(cudaMemcpyAsync(d_src + (size_t)uploaded * ff, h_src + (size_t)uploaded * ff,
                                     (size_t)(need - uploaded) * ff * sizeof(float),
                                     cudaMemcpyHostToDevice, c->s_in));
            CUDA_TRY(cudaEventRecord(c->ev_in, c->s_in));
            CUDA_TRY(cudaStreamWaitEvent(s, c->ev_in, 0));
            if (c->prop)
                if (int rc = embed_frames(c, 0, d_src, uploaded, need, s)) return rc;
            uploaded = need;
        }
        if (int rc = run_stage_windows(c, tb, mb, false, basic_done, w1, s)) return rc;
        basic_done = w1;
        const int a1 = basic_done == N ? N : std::max(0, basic_done - r);
        if (int rc = aggregate_frames(c, c->d_acc, d_basic, basic_agg, a1, s)) return rc;
        // the final stage, its embeddings of the basic estimate included,
        // continues on its own stream from here
        CUDA_TRY(cudaEventRecord(c->ev_bas, s));
        CUDA_TRY(cudaStreamWaitEvent(sf, c->ev_bas, 0));
        if (c->prop && c->final_matching == 0)
            if (int rc = embed_frames(c, 1, d_basic, basic_agg, a1, sf)) return rc;
        basic_agg = std::max(basic_agg, a1);
        // the last step runs its final stage in pieces (to N-4, N-3, N-2,
        // then N), so the finished frames download while the rest computes
        if (w1 == N)
            for (int k = 4; k >= 2; --k)
                if (N - k > final_done + 2)
                    if (int rc = advance_final(N - k)) return rc;
        if (int rc = advance_final(N)) return rc;
    }
    // the caller's stream owns completion: join the final-stage and download
    // streams into it
    CUDA_TRY(cudaEventRecord(c->ev_fin, sf));
    CUDA_TRY(cudaStreamWaitEvent(s, c->ev_fin, 0));
    CUDA_TRY(cudaEventRecord(c->ev_out, c->s_out));
    CUDA_TRY(cudaStreamWaitEvent(s, c->ev_out, 0));
    return BM3D_B200_OK;
}

int twostage_host(bm3d_b200_clip *c, const float *h_src, float *h_dst, void *stream, bool wait) {
    if (!c || !h_src || !h_dst) return fail(BM3D_B200_ERR_INVALID, "BM3D: null argument");
    CUDA_TRY(cudaSetDevice(c->device));
    cudaStream_t s = stream ? as_stream(stream) : c->stream;
    const size_t src_floats = (size_t)c->nframes * c->frame_floats;
    if (int rc = ensure_io(c, src_floats, false)) return rc;
    if (!c->d_basic) CUDA_TRY(cudaMalloc(&c->d_basic, src_floats * sizeof(float)));
    if (int rc = clip_begin(c, s)) return rc;
    if (c->nplanes == 1 && c->process[0]) {
        if (int rc = twostage_pipelined(c, h_src, h_dst, s, !wait)) return rc;
        if (int rc = clip_end(c, s)) return rc;
        if (!wait) return BM3D_B200_OK;
        CUDA_TRY(cudaStreamSynchronize(s));
        return clip_check(c);
    }
    CUDA_TRY(cudaMemcpyAsync(c->d_io_src, h_src, src_floats * sizeof(float), cudaMemcpyHostToDevice,
                             s));
    if (int rc = bm3d_b200_clip_twostage(c, c->d_io_src, c->d_basic, c->d_io_dst, s)) return rc;
    CUDA_TRY(cudaMemcpyAsync(h_dst, c->d_io_dst, src_floats * sizeof(float), cudaMemcpyDeviceToHost,
                             s));
    if (int rc = clip_end(c, s)) return rc;
    if (!wait) return BM3D_B200_OK;
    CUDA_TRY(cudaStreamSynchronize(s));
    return clip_check(c);
}

}  // namespace

extern "C" int bm3d_b200_clip_twostage_host(bm3d_b200_clip *c, const float *h_src, float *h_dst,
                                            void *stream) {
    return twostage_host(c, h_src, h_dst, stream, true);
}

extern "C" int bm3d_b200_clip_twostage_host_async(bm3d_b200_clip *c, const float *h_src,
                                                  float *h_dst, void *stream) {
    return twostage_host(c, h_src, h_dst, stream, false);
}

extern "C" int bm3d_b200_clip_set_profiling(bm3d_b200_clip *c, int enable) {
    if (!c) return fail(BM3D_B200_ERR_INVALID, "BM3D: null clip");
    c->profiling = enable != 0;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_clip_stage_times(bm3d_b200_clip *c, double *ms, long long *launches,
                                          int reset) {
    if (!c) return fail(BM3D_B200_ERR_INVALID, "BM3D: null clip");
    CUDA_TRY(cudaSetDevice(c->device));
    for (auto &m : c->marks) {
        CUDA_TRY(cudaEventSynchronize(m.b));
        float t = 0.0f;
        CUDA_TRY(cudaEventElapsedTime(&t, m.a, m.b));
        c->stage_ms[m.stage] += t;
        c->stage_launches[m.stage] += m.kernels;
        cudaEventDestroy(m.a);
        cudaEventDestroy(m.b);
    }
    c->marks.clear();
    for (int i = 0; i < BM3D_B200_NUM_STAGES; ++i) {
        if (ms) ms[i] = c->stage_ms[i];
        if (launches) launches[i] = c->stage_launches[i];
        if (reset) {
            c->stage_ms[i] = 0.0;
            c->stage_launches[i] = 0;
        }
    }
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_clip_set_proposer(bm3d_b200_clip *c, bm3d_b200_proposer *p,
                                           int cells_spatial, int cells_temporal,
                                           float fallback_tau) {
    if (!c) return fail(BM3D_B200_ERR_INVALID, "BM3D: null clip");
    if (!p) {
        c->prop = nullptr;
        return BM3D_B200_OK;
    }
    if (cells_spatial < 1 || cells_spatial > 8 || cells_temporal < 1 || cells_temporal > 8)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: proposal cell counts must be in range [1, 8]");
    if (!(fallback_tau >= 0.0f)) return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid fallback_tau");
    for (int q = 0; q < 3; ++q)
        if (c->metric[q] || c->tx2[q] || c->tx1[q])
            return fail(BM3D_B200_ERR_UNSUPPORTED,
                        "BM3D: learned matching runs with the SSD and DCT defaults only");
    if (c->nplanes != 1 && !c->prm.chroma)
        return fail(BM3D_B200_ERR_UNSUPPORTED,
                    "BM3D: learned matching needs a single-plane clip or chroma matching");
    if (proposer_device(p) != c->device)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: proposer and clip are on different devices");
    if (c->pw[0] < 16 || c->ph[0] < 16)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: learned matching needs planes of 16x16 or more");
    CUDA_TRY(cudaSetDevice(c->device));
    const int N = c->nframes, r = c->prm.radius, tw = 2 * r + 1;
    const size_t ntab = (size_t)N * tw;
    const MatchGeometry lg = learned_geometry(c->pw[0], c->ph[0], c->prm.block_step[0],
                                              c->prm.bm_range[0], r, c->prm.ps_range[0]);
    if (lg.smem > 220 * 1024 ||
        !learned_ordinals_fit(c->prm.bm_range[0], c->prm.ps_num[0], c->prm.ps_range[0]))
        return fail(BM3D_B200_ERR_UNSUPPORTED, "BM3D: search range too large for learned matching");
    const size_t ef = (size_t)(c->pw[0] / 2) * (c->ph[0] / 2) * 16;
    if (!c->d_emb) {
        CUDA_TRY(cudaMalloc(&c->d_emb, 2 * (size_t)N * ef));
        CUDA_TRY(cudaMalloc(&c->d_etab, 2 * ntab * sizeof(void *)));
        c->fb_stride = std::max<size_t>(1, (size_t)N * lg.nbx * lg.nby);
        CUDA_TRY(cudaMalloc(&c->d_fb, 2 * c->fb_stride * sizeof(unsigned)));
        CUDA_TRY(cudaMalloc(&c->d_fbcount, 2 * sizeof(unsigned)));
        CUDA_TRY(cudaMalloc(&c->d_fbtotal, sizeof(unsigned long long)));
        CUDA_TRY(cudaMemset(c->d_fbtotal, 0, sizeof(unsigned long long)));
        std::vector<void *> tab(2 * ntab);
        for (int which = 0; which < 2; ++which)
            for (int n = 0; n < N; ++n)
                for (int z = 0; z < tw; ++z) {
                    const int f = std::min(std::max(n - r + z, 0), N - 1);
                    tab[which * ntab + (size_t)n * tw + z] =
                        c->d_emb + ((size_t)which * N + f) * ef;
                }
        CUDA_TRY(cudaMemcpy(c->d_etab, tab.data(), tab.size() * sizeof(void *),
                            cudaMemcpyHostToDevice));
    }
    c->lgeo = lg;
    c->prop = p;
    c->cells_s = cells_spatial;
    c->cells_t = cells_temporal;
    c->fb_tau = fallback_tau;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_clip_set_variant(bm3d_b200_clip *c, const int *bm_error,
                                          const int *transform_2d, const int *transform_1d) {
    if (!c) return fail(BM3D_B200_ERR_INVALID, "BM3D: null clip");
    int m[3], t2[3], t1[3];
    for (int q = 0; q < 3; ++q) {
        m[q] = bm_error ? bm_error[q] : BM3D_B200_BM_SSD;
        t2[q] = transform_2d ? transform_2d[q] : BM3D_B200_TX_DCT;
        t1[q] = transform_1d ? transform_1d[q] : BM3D_B200_TX_DCT;
        if (m[q] < BM3D_B200_BM_SSD || m[q] > BM3D_B200_BM_SSD_NORM)
            return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'bm_error_s': %d", m[q]);
        if (t2[q] < BM3D_B200_TX_DCT || t2[q] > BM3D_B200_TX_BIOR1_5)
            return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'transform_2d_s': %d", t2[q]);
        if (t1[q] < BM3D_B200_TX_DCT || t1[q] > BM3D_B200_TX_BIOR1_5)
            return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'transform_1d_s': %d", t1[q]);
    }
    const bool variant = m[0] || m[1] || m[2] || t2[0] || t2[1] || t2[2] || t1[0] || t1[1] || t1[2];
    if (variant && c->prop)
        return fail(BM3D_B200_ERR_UNSUPPORTED,
                    "BM3D: learned matching runs with the SSD and DCT defaults only");
    if (variant && c->precision != BM3D_B200_PRECISION_FP32)
        return fail(BM3D_B200_ERR_UNSUPPORTED, "BM3D: transform variants run in FP32 only");
    for (int q = 0; q < 3; ++q) {
        c->metric[q] = m[q];
        c->tx2[q] = t2[q];
        c->tx1[q] = t1[q];
    }
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_clip_set_precision(bm3d_b200_clip *c, int precision) {
    if (!c) return fail(BM3D_B200_ERR_INVALID, "BM3D: null clip");
    if (precision != BM3D_B200_PRECISION_FP32 && precision != BM3D_B200_PRECISION_SPLIT_BF16 &&
        precision != BM3D_B200_PRECISION_TC_F16)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: unknown precision %d", precision);
    if (precision != BM3D_B200_PRECISION_FP32)
        for (int q = 0; q < 3; ++q)
            if (c->tx2[q] || c->tx1[q])
                return fail(BM3D_B200_ERR_UNSUPPORTED, "BM3D: transform variants run in FP32 only");
    if (precision == BM3D_B200_PRECISION_TC_F16 && !c->h_tcerr) {
        CUDA_TRY(cudaSetDevice(c->device));
        CUDA_TRY(cudaHostAlloc(&c->h_tcerr, sizeof(unsigned), cudaHostAllocMapped));
        *c->h_tcerr = 0;
        CUDA_TRY(cudaHostGetDevicePointer(reinterpret_cast<void **>(&c->d_tcerr), c->h_tcerr, 0));
    }
    c->precision = precision;
    return BM3D_B200_OK;
}

namespace {
// Host view of the clip's device-side failures: a tensor-core filter CTA or a
// proposer tile that gave up waiting for its MMAs.
int clip_check(const bm3d_b200_clip *c) {
    if (c->h_tcerr && *(volatile unsigned *)c->h_tcerr != 0)
        return fail(BM3D_B200_ERR_CUDA,
                    "BM3D: a tensor-core filter block timed out waiting for its MMAs");
    return proposer_check(c->prop);
}
}  // namespace

extern "C" int bm3d_b200_clip_status(bm3d_b200_clip *c) {
    if (!c) return fail(BM3D_B200_ERR_INVALID, "BM3D: null clip");
    return clip_check(c);
}

extern "C" int bm3d_b200_clip_matches(bm3d_b200_clip *c, int n, int *h_xyz, int capacity_blocks,
                                      int *nblocks) {
    if (!c || !nblocks) return fail(BM3D_B200_ERR_INVALID, "BM3D: null argument");
    const int q = 0;
    const int nblk = c->geo[q].nbx * c->geo[q].nby;
    *nblocks = nblk;
    if (!h_xyz || capacity_blocks < nblk) return BM3D_B200_OK;  // count only
    if (n < 0 || n >= c->nframes)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: frame %d outside the clip", n);
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaDeviceSynchronize());
    std::vector<int> packed((size_t)nblk * 8);
    CUDA_TRY(cudaMemcpy(packed.data(), c->d_matches + (size_t)n * nblk * 8,
                        packed.size() * sizeof(int), cudaMemcpyDeviceToHost));
    return unpack_matches(packed, h_xyz, nblk);
}

extern "C" int bm3d_b200_clip_set_final_matching(bm3d_b200_clip *c, int mode) {
    if (!c) return fail(BM3D_B200_ERR_INVALID, "BM3D: null clip");
    if (mode != BM3D_B200_FINAL_MATCH_SEARCH && mode != BM3D_B200_FINAL_MATCH_BASIC_LISTS &&
        mode != BM3D_B200_FINAL_MATCH_BASIC_ORDER)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: unknown final matching mode %d", mode);
    c->final_matching = mode;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_clip_learned_stats(bm3d_b200_clip *c, long long *blocks,
                                            long long *fallbacks, int reset) {
    if (!c) return fail(BM3D_B200_ERR_INVALID, "BM3D: null clip");
    CUDA_TRY(cudaSetDevice(c->device));
    CUDA_TRY(cudaDeviceSynchronize());
    unsigned long long fb = 0;
    if (c->d_fbtotal)
        CUDA_TRY(cudaMemcpy(&fb, c->d_fbtotal, sizeof(fb), cudaMemcpyDeviceToHost));
    if (blocks) *blocks = c->stat_blocks;
    if (fallbacks) *fallbacks = (long long)fb;
    if (reset) {
        c->stat_blocks = 0;
        if (c->d_fbtotal) CUDA_TRY(cudaMemset(c->d_fbtotal, 0, sizeof(unsigned long long)));
    }
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_learned_match(const float *const *d_frames, const void *const *d_embs,
                                       int width, int height, int stride, int block_step,
                                       int bm_range, int radius, int ps_num, int ps_range,
                                       int cells_spatial, int cells_temporal, float fallback_ssd,
                                       int *h_xyz, int *h_fallback, int capacity_blocks,
                                       int *nblocks) {
    if (!d_frames || !d_embs || !h_xyz || !nblocks)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: null argument");
    if (int rc = check_search(width, height, stride, block_step, bm_range, radius, ps_num,
                              ps_range))
        return rc;
    if (width < 16 || height < 16)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: learned matching needs planes of 16x16 or more");
    if (cells_spatial < 1 || cells_spatial > 8 || cells_temporal < 1 || cells_temporal > 8)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: proposal cell counts must be in range [1, 8]");
    const int tw = 2 * radius + 1;
    const MatchGeometry g = match_geometry(width, height, block_step, bm_range, radius, ps_range);
    const MatchGeometry lg = learned_geometry(width, height, block_step, bm_range, radius,
                                              ps_range);
    if (lg.smem > 220 * 1024 || !learned_ordinals_fit(bm_range, ps_num, ps_range))
        return fail(BM3D_B200_ERR_UNSUPPORTED, "BM3D: search range too large for learned matching");
    const int nblk = g.nbx * g.nby;
    *nblocks = nblk;
    if (capacity_blocks < nblk)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: match buffer holds %d blocks, %d needed",
                    capacity_blocks, nblk);
    void **d_tab = nullptr;
    int *d_m = nullptr;
    unsigned *d_fb = nullptr;
    auto release = [&](int rc) {
        cudaFree(d_tab);
        cudaFree(d_m);
        cudaFree(d_fb);
        return rc;
    };
    if (cudaMalloc(&d_tab, 2 * tw * sizeof(void *)) != cudaSuccess ||
        cudaMalloc(&d_m, (size_t)nblk * 8 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&d_fb, ((size_t)nblk + 1) * sizeof(unsigned)) != cudaSuccess)
        return release(fail(BM3D_B200_ERR_NOMEM, "BM3D: allocation failed"));
    std::vector<const void *> tab(2 * tw);
    for (int z = 0; z < tw; ++z) {
        tab[z] = d_frames[z];
        tab[tw + z] = d_embs[z];
    }
    cudaError_t e = cudaMemcpy(d_tab, tab.data(), tab.size() * sizeof(void *),
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(d_fb + nblk, 0, sizeof(unsigned));
    MatchParams mp = make_match_params(g, reinterpret_cast<const float *const *>(d_tab), d_m,
                                       width, height, stride, block_step, bm_range, radius,
                                       ps_num, ps_range);
    MatchParams lm = mp;
    lm.pitch = lg.pitch;
    lm.tile_rows = lg.tile_rows;
    LearnedParams lp{};
    lp.embs = reinterpret_cast<const void *const *>(d_tab + tw);
    lp.w2 = width / 2;
    lp.cells_s = cells_spatial;
    lp.cells_t = cells_temporal;
    lp.fallback_ssd = fallback_ssd > 0.0f ? fallback_ssd : 0.0f;
    lp.fallback = d_fb;
    lp.fallback_count = d_fb + nblk;
    lp.fallback_capacity = (unsigned)nblk;
    if (e == cudaSuccess) e = launch_learned_match(lm, lp, lg, 1, nullptr);
    if (e == cudaSuccess && lp.fallback_ssd > 0.0f)
        e = launch_match_fallback(mp, d_fb, d_fb + nblk, nullptr);
    std::vector<int> packed((size_t)nblk * 8);
    std::vector<unsigned> fbl((size_t)nblk + 1, 0u);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess)
        e = cudaMemcpy(packed.data(), d_m, packed.size() * sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess)
        e = cudaMemcpy(fbl.data(), d_fb, fbl.size() * sizeof(unsigned), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess)
        return release(fail(BM3D_B200_ERR_CUDA, "BM3D: learned matching failed: %s",
                            cudaGetErrorString(e)));
    unpack_matches(packed, h_xyz, nblk);
    if (h_fallback) {
        std::fill(h_fallback, h_fallback + nblk, 0);
        const unsigned n = std::min<unsigned>(fbl[nblk], (unsigned)nblk);
        for (unsigned i = 0; i < n; ++i) h_fallback[fbl[i] % (unsigned)nblk] = 1;
    }
    return release(BM3D_B200_OK);
}

extern "C" void bm3d_b200_clip_destroy(bm3d_b200_clip *c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (auto &m : c->marks) {
        cudaEventDestroy(m.a);
        cudaEventDestroy(m.b);
    }
    cudaFreeHost(c->h_tcerr);
    cudaFree(c->d_matches);
    cudaFree(c->d_acc);
    cudaFree(c->d_mult);
    cudaFree(c->d_tab);
    cudaFree(c->d_basic);
    cudaFree(c->d_io_src);
    cudaFree(c->d_io_ref);
    cudaFree(c->d_io_dst);
    cudaFree(c->d_acc2);
    cudaFree(c->d_ptab);
    cudaFree(c->d_pmult);
    cudaFree(c->d_emb);
    cudaFree(c->d_etab);
    cudaFree(c->d_fb);
    cudaFree(c->d_fbcount);
    cudaFree(c->d_fbtotal);
    if (c->s_in) cudaStreamDestroy(c->s_in);
    if (c->s_out) cudaStreamDestroy(c->s_out);
    if (c->s_fin) cudaStreamDestroy(c->s_fin);
    if (c->ev_in) cudaEventDestroy(c->ev_in);
    if (c->ev_out) cudaEventDestroy(c->ev_out);
    if (c->ev_bas) cudaEventDestroy(c->ev_bas);
    if (c->ev_fin) cudaEventDestroy(c->ev_fin);
    if (c->ev_done) cudaEventDestroy(c->ev_done);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

// ===========================================================================
// 4. allocation-free per-window pipeline
// ===========================================================================
// Some callers cannot let a library allocate device memory while frames are
// being processed: a host application that owns the whole device-memory
// budget through its own pool, or a real-time pipeline that cannot afford the
// device-wide synchronisation cudaMalloc / cudaFree may cause. For them,
// bm3d_b200_window_noalloc does the device work of bm3d_b200_graph_launch_device
// (zero d_res, block matching, filtering and scatter of one window) with its
// scratch - the plane-pointer tables and the block-matching lists - in the
// file-scope array below instead of cudaMalloc'd memory. The caller still
// provides d_src and d_res.
//
// The array is 8 MiB on every device that loads this library, held until the
// process exits. Every call on a device shares it and leaves its last
// contents behind; nothing in it needs to start at zero, because each call
// writes every table entry and every match list before reading them. Calls
// whose work overlaps on the GPU (different streams, or different host
// threads, on the same device) race on the array: issue them in order on one
// stream.
namespace {

constexpr size_t kNoallocScratchBytes = size_t(8) << 20;
constexpr size_t kNoallocTableBytes = 4096;  // plane-pointer tables (<= 512 entries)
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// The name g_noalloc_scratch in host code is only a stand-in for the symbol;
// its device address is resolved per device with cudaGetSymbolAddress.
std::atomic<void *> g_noalloc_addr[64] = {};

// Resolves the array's address on `device` (the current device) the first
// time a call runs there.
int noalloc_scratch(int device, unsigned char **out) {
    if (device < 0 || device >= 64)
        return fail(BM3D_B200_ERR_UNSUPPORTED, "BM3D: device index %d out of range", device);
    void *ptr = g_noalloc_addr[device].load(std::memory_order_acquire);
    if (!ptr) {
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || !ptr)
            return fail(BM3D_B200_ERR_CUDA, "BM3D: cudaGetSymbolAddress failed: %s",
                        cudaGetErrorString(e));
        g_noalloc_addr[device].store(ptr, std::memory_order_release);
    }
    *out = static_cast<unsigned char *>(ptr);
    return BM3D_B200_OK;
}

struct NoallocTables {
    const float *src;
    float *res;
    long long plane;  // floats per plane
    int tw, np, final_;
};

// Writes the [mframes tw][src np*tw][ref np*tw][acc np*tw] pointer tables of
// one window into the scratch array (same layout as bm3d_b200_graph).
__global__ void noalloc_fill_tables(void **tab, NoallocTables t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int ntw = t.np * t.tw;
    if (i >= t.tw * (1 + 3 * t.np)) return;
    void *v;
    if (i < t.tw) {
        v = (void *)(t.src + (long long)i * t.plane);
    } else {
        const int k = i - t.tw;
        const int part = k / ntw, qz = k % ntw;  // qz = q * tw + z
        if (part == 0)
            v = (void *)(t.src + ((long long)(t.final_ ? ntw : 0) + qz) * t.plane);
        else if (part == 1)
            v = t.final_ ? (void *)(t.src + (long long)qz * t.plane) : nullptr;
        else
            v = (void *)(t.res + (long long)qz * 2 * t.plane);
    }
    tab[i] = v;
}

}  // namespace

extern "C" int bm3d_b200_window_noalloc(float *d_res, const float *d_src, int width, int height,
                                        int stride, float sigma, int block_step, int bm_range,
                                        int radius, int ps_num, int ps_range, int chroma,
                                        float sigma_u, float sigma_v, int final_, float extractor,
                                        void *stream) {
    if (!d_res || !d_src) return fail(BM3D_B200_ERR_INVALID, "BM3D: null device buffer");
    if (int rc = check_search(width, height, stride, block_step, bm_range, radius, ps_num,
                              ps_range))
        return rc;
    if (!(sigma >= 0.0f) || !(sigma_u >= 0.0f) || !(sigma_v >= 0.0f))
        return fail(BM3D_B200_ERR_INVALID, "BM3D: \"sigma\" must be non-negative");
    const MatchGeometry geo = match_geometry(width, height, block_step, bm_range, radius, ps_range);
    const size_t nblk = (size_t)geo.nbx * geo.nby;
    const size_t need = kNoallocTableBytes + nblk * 8 * sizeof(int);
    if (need > kNoallocScratchBytes)
        return fail(BM3D_B200_ERR_UNSUPPORTED,
                    "BM3D: %zu reference blocks exceed the allocation-free path's limit of %zu "
                    "(8 MiB of scratch); use a larger block_step or bm3d_b200_graph_*",
                    nblk, (kNoallocScratchBytes - kNoallocTableBytes) / (8 * sizeof(int)));
    int device = 0;
    CUDA_TRY(cudaGetDevice(&device));
    unsigned char *scratch = nullptr;
    if (int rc = noalloc_scratch(device, &scratch)) return rc;

    cudaStream_t s = as_stream(stream);
    const int tw = 2 * radius + 1;
    const int np = chroma ? 3 : 1;
    const size_t plane = (size_t)height * stride;
    void **tab = reinterpret_cast<void **>(scratch);
    int *matches = reinterpret_cast<int *>(scratch + kNoallocTableBytes);

    NoallocTables t{d_src, d_res, (long long)plane, tw, np, final_ ? 1 : 0};
    const int ntab = tw * (1 + 3 * np);
    noalloc_fill_tables<<<(ntab + 127) / 128, 128, 0, s>>>(tab, t);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemsetAsync(d_res, 0, (size_t)np * tw * 2 * plane * sizeof(float), s));

    const float *const *ctab = reinterpret_cast<const float *const *>(tab);
    MatchParams mp = make_match_params(geo, ctab, matches, width, height, stride, block_step,
                                       bm_range, radius, ps_num, ps_range);
    CUDA_TRY(launch_match(mp, geo, 1, s));
    const float sig[3] = {sigma, sigma_u, sigma_v};
    for (int q = 0; q < np; ++q) {
        if (chroma && sig[q] < FLT_EPSILON) continue;
        FilterParams fp{};
        fp.src = ctab + tw + (size_t)q * tw;
        fp.ref = final_ ? ctab + tw + (size_t)np * tw + (size_t)q * tw : nullptr;
        fp.acc = reinterpret_cast<float *const *>(tab + tw + (size_t)2 * np * tw + (size_t)q * tw);
        fp.mult = nullptr;
        fp.matches = matches;
        fp.weight_offset = (long long)plane;
        fp.acc_stride = stride;
        fp.stride = stride;
        fp.radius = radius;
        fp.nblk = (int)nblk;
        fp.nbx = geo.nbx;
        fp.corner_weight = 0;
        fp.nwin = 1;
        fp.sigma = sig[q];
        fp.extractor = extractor;
        CUDA_TRY(launch_filter(fp, final_ != 0, s));
    }
    return BM3D_B200_OK;
}

// ===========================================================================
// 5. Streaming BM3Dv2 for frame-by-frame hosts
// ===========================================================================
// Source (and reference) frames live in a ring keyed by frame index and are
// uploaded once; every window's raw V-BM3D stack ([planes][2r+1][2][H][stride])
// is computed once into a ring of window slots; output frame n is the
// VAggregate of windows clamp(n-r .. n+r) on the device.
//
// Requests run concurrently (a host such as VapourSynth calls getFrame from
// several worker threads): each takes one of kStreamRequests request contexts
// (its own CUDA stream, tables, match lists and output plane) and holds the
// lock only to claim slots. A slot is produced by the request that claimed it
// first (an upload, or a window's filtering issued on that request's stream
// and marked by the slot's event); other requests that need it wait until the
// event is recorded and then order their stream after it. Slots in use are
// pinned and never evicted; the rings hold every request's frames and
// windows at once, so a claim always finds a slot. The windows a request
// produces run as one batched launch per kernel. Work that waits only on
// uploads never blocks an upload, and window waits come after a request's
// own windows are issued, so requests cannot wait on each other in a cycle.
constexpr int kStreamRequests = 4;  // concurrent requests (the reference's fast=True: 4)

// Host threads that share the memory copies of a stream's requests: run(n, fn)
// calls fn(0) .. fn(n - 1) spread over the pool and the calling thread (which
// also helps with parts queued by other requests) and returns when its n
// parts are done. A part references the caller's fn only until it counts
// down, so nothing outlives the call.
class CopyPool {
  public:
    explicit CopyPool(int nthreads) {
        try {
            for (int i = 0; i < nthreads; ++i) th_.emplace_back([this] { loop(); });
        } catch (...) {
            shutdown();
            throw;
        }
    }
    ~CopyPool() { shutdown(); }
    int threads() const { return (int)th_.size(); }
    void run(int n, const std::function<void(int)> &fn) {
        if (n <= 1 || th_.empty()) {
            for (int i = 0; i < n; ++i) fn(i);
            return;
        }
        auto left = std::make_shared<Latch>(n);
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (int i = 1; i < n; ++i)
                q_.emplace_back([left, &fn, i] {
                    fn(i);
                    left->count_down();
                });
        }
        cv_.notify_all();
        fn(0);
        left->count_down();
        while (!left->done()) {
            std::function<void()> task;
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (!q_.empty()) {
                    task = std::move(q_.front());
                    q_.pop_front();
                }
            }
            if (task) task();
            else left->wait();
        }
    }

  private:
    void shutdown() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_) t.join();
        th_.clear();
    }
    struct Latch {
        explicit Latch(int n) : n(n) {}
        void count_down() {
            std::lock_guard<std::mutex> lk(m);
            if (--n == 0) cv.notify_all();
        }
        bool done() {
            std::lock_guard<std::mutex> lk(m);
            return n == 0;
        }
        void wait() {
            std::unique_lock<std::mutex> lk(m);
            cv.wait(lk, [&] { return n == 0; });
        }
        int n;
        std::mutex m;
        std::condition_variable cv;
    };
    void loop() {
        for (;;) {
            std::function<void()> task;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return stop_ || !q_.empty(); });
                if (q_.empty()) return;  // stopping
                task = std::move(q_.front());
                q_.pop_front();
            }
            task();
        }
    }
    std::vector<std::thread> th_;
    std::deque<std::function<void()>> q_;
    std::mutex mu_;
    std::condition_variable cv_;
    bool stop_ = false;
};

// Copy threads of a stream: up to 8, one fewer than the host's hardware threads.
int copy_pool_threads() {
    const int hw = (int)std::thread::hardware_concurrency();
    return std::max(0, std::min(8, hw - 1));
}

struct bm3d_b200_stream {
    int device = 0;
    int width = 0, height = 0, nplanes = 1, ssw = 0, ssh = 0, nframes = 0;
    bm3d_b200_params prm{};
    bool final_ = false;
    int stride = 0, r = 0, tw = 1;
    int pw[3] = {0, 0, 0}, ph[3] = {0, 0, 0};
    long long poff[3] = {0, 0, 0}, rawoff[3] = {0, 0, 0};
    long long frame_floats = 0, raw_floats = 0;
    bool process[3] = {false, false, false};
    float sigma[3] = {0, 0, 0};
    MatchGeometry geo[3]{};
    size_t max_blk = 1, max_plane = 0;
    int metric[3] = {0, 0, 0}, tx2[3] = {0, 0, 0}, tx1[3] = {0, 0, 0};
    // key: frame or window index; state: 0 empty, 1 being produced, 2 ready
    struct Slot {
        int key = -1;
        int state = 0;
        int pins = 0;
        unsigned long long use = 0;
        cudaEvent_t ready = nullptr;
    };
    std::vector<Slot> fslot, wslot;
    float *d_frames = nullptr;  // [fcap][(final ? 2 : 1)][frame_floats]
    float *d_raw = nullptr;     // [wcap][raw_floats]
    struct Request {
        bool busy = false;
        cudaStream_t s = nullptr;
        cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // start, uploaded, filtered, done
        float *d_out = nullptr;     // one plane
        int *d_matches = nullptr;   // [2r+1][max_blk][8]
        void **d_tab = nullptr;     // [3 jobs][10 tables][2r+1 windows][tw], then [2r+1][tw] embeddings
        void **h_tab = nullptr;     // pinned mirror
        unsigned *d_fb = nullptr;   // learned matching: [2r+1][max_blk] blocks to re-search, count
        // two pinned staging buffers for the host copies, each with the event
        // of its last DMA (see staged_copy)
        void *h_stage[2] = {nullptr, nullptr};
        cudaEvent_t stage_ev[2] = {nullptr, nullptr};
        int stage_next = 0;
    };
    int nreq = kStreamRequests;  // request contexts allocated
    int nuse = kStreamRequests;  // of which in use (bm3d_b200_stream_set_concurrency)
    Request req[kStreamRequests];
    // learned matching (bm3d_b200_stream_set_proposer): embeddings of every
    // frame slot's matching plane, computed when the frame is uploaded
    bm3d_b200_proposer *prop = nullptr;
    int cells_s = 2, cells_t = 2;
    float fb_tau = 0.0f;
    MatchGeometry lgeo{};
    uint8_t *d_emb = nullptr;  // [fcap][emb_bytes]
    size_t emb_bytes = 0;
    std::unique_ptr<CopyPool> pool;  // host copies of all requests (staged_copy)
    std::mutex mu;
    std::condition_variable cv;
    unsigned long long tick = 0;
    long long uploads = 0, windows = 0, calls = 0;
    double ms_upload = 0.0, ms_filter = 0.0, ms_output = 0.0;
};

namespace {

const float *stream_slot(const bm3d_b200_stream *s, int slot) {
    return s->d_frames + (size_t)slot * (s->final_ ? 2 : 1) * s->frame_floats;
}

// Claims the slot of `key` (pinned): the slot already holding it, or an
// unpinned one (empty first, else least recently used) that the caller must
// produce (*produce = true). -1 if every slot is pinned.
int claim_slot(std::vector<bm3d_b200_stream::Slot> &v, int key, unsigned long long tick,
               bool *produce) {
    for (size_t i = 0; i < v.size(); ++i)
        if (v[i].key == key && v[i].state != 0) {
            ++v[i].pins;
            v[i].use = tick;
            *produce = false;
            return (int)i;
        }
    int victim = -1;
    for (size_t i = 0; i < v.size(); ++i) {
        if (v[i].pins) continue;
        if (victim < 0 || (v[i].state == 0 && v[victim].state != 0) ||
            (v[i].state == v[victim].state && v[i].use < v[victim].use))
            victim = (int)i;
    }
    if (victim < 0) return -1;
    v[victim].key = key;
    v[victim].state = 1;
    v[victim].pins = 1;
    v[victim].use = tick;
    *produce = true;
    return victim;
}

// One request's claims, kept for the release.
struct StreamClaims {
    std::vector<int> fs, fprod;  // frame slots pinned / produced by this request
    std::vector<int> ws, wprod;  // window slots pinned / produced
};

// Waits (lock held through lk) until slot i of v holds `key` ready; false if
// its producer gave up.
bool wait_ready(bm3d_b200_stream *s, std::unique_lock<std::mutex> &lk,
                std::vector<bm3d_b200_stream::Slot> &v, int i, int key) {
    s->cv.wait(lk, [&] { return v[i].key != key || v[i].state == 2; });
    return v[i].key == key && v[i].state == 2;
}

// Marks produced slots ready (their events recorded) or, on failure, empty.
void finish_slots(bm3d_b200_stream *s, std::vector<bm3d_b200_stream::Slot> &v,
                  const std::vector<int> &idx, bool ok) {
    std::lock_guard<std::mutex> lk(s->mu);
    for (int i : idx) {
        if (ok) {
            v[i].state = 2;
        } else {
            v[i].key = -1;
            v[i].state = 0;
        }
    }
    s->cv.notify_all();
}

constexpr size_t kStageBytes = size_t(4) << 20;  // one pinned staging buffer

// Copies a pitched plane between the caller's (pageable) host memory and the
// device through the request's two pinned staging buffers, in bands of rows:
// the host copies one band (split across the stream's copy threads) while the
// DMA of the previous band runs, and the DMAs run at pinned-memory speed on
// the request's stream. Concurrent requests each have their own buffers.
cudaError_t staged_copy(bm3d_b200_stream::Request &q, CopyPool &pool, bool to_device, void *dst,
                        size_t dpitch, const void *src, size_t spitch, size_t width_bytes,
                        int rows) {
    const int band = (int)std::max<size_t>(1, kStageBytes / width_bytes);
    // parts of at least 512 KiB per host thread
    auto host_rows = [&](char *d, size_t dp, const char *sp, size_t ss, int n) {
        const int parts = (int)std::max<size_t>(
            1, std::min<size_t>((size_t)pool.threads() + 1,
                                (size_t)n * width_bytes / (size_t(512) << 10)));
        const int per = (n + parts - 1) / parts;
        pool.run(parts, [&](int k) {
            for (int i = k * per; i < std::min(n, (k + 1) * per); ++i)
                std::memcpy(d + (size_t)i * dp, sp + (size_t)i * ss, width_bytes);
        });
    };
    int pend_b = -1, pend_r0 = 0, pend_n = 0;  // download band waiting for its host copy
    auto drain = [&]() -> cudaError_t {
        if (pend_b < 0) return cudaSuccess;
        const cudaError_t e = cudaEventSynchronize(q.stage_ev[pend_b]);
        if (e != cudaSuccess) return e;
        host_rows(static_cast<char *>(dst) + (size_t)pend_r0 * dpitch, dpitch,
                  static_cast<const char *>(q.h_stage[pend_b]), width_bytes, pend_n);
        pend_b = -1;
        return cudaSuccess;
    };
    for (int r0 = 0; r0 < rows; r0 += band) {
        const int b = q.stage_next;
        q.stage_next ^= 1;
        const int n = std::min(band, rows - r0);
        cudaError_t e = cudaEventSynchronize(q.stage_ev[b]);  // the buffer's last DMA
        if (e != cudaSuccess) return e;
        char *h = static_cast<char *>(q.h_stage[b]);
        if (to_device) {
            host_rows(h, width_bytes, static_cast<const char *>(src) + (size_t)r0 * spitch, spitch,
                      n);
            e = cudaMemcpy2DAsync(static_cast<char *>(dst) + (size_t)r0 * dpitch, dpitch, h,
                                  width_bytes, width_bytes, n, cudaMemcpyHostToDevice, q.s);
        } else {
            e = cudaMemcpy2DAsync(h, width_bytes,
                                  static_cast<const char *>(src) + (size_t)r0 * spitch, spitch,
                                  width_bytes, n, cudaMemcpyDeviceToHost, q.s);
        }
        if (e == cudaSuccess) e = cudaEventRecord(q.stage_ev[b], q.s);
        if (e == cudaSuccess && !to_device) e = drain();
        if (e != cudaSuccess) return e;
        if (!to_device) {
            pend_b = b;
            pend_r0 = r0;
            pend_n = n;
        }
    }
    return drain();
}

// Uploads frame f into frame slot `slot` (host arrays hold frames first .. ).
int stream_upload(bm3d_b200_stream *s, bm3d_b200_stream::Request &rq, int slot, int f,
                  int first, const float *const *h_src, const float *const *h_ref,
                  const int *src_strides) {
    cudaStream_t st = rq.s;
    const int k = f - first;
    for (int half = 0; half < (s->final_ ? 2 : 1); ++half) {
        const float *const *hp = half == 0 ? h_src : h_ref;
        float *dst = const_cast<float *>(stream_slot(s, slot)) + (size_t)half * s->frame_floats;
        for (int q = 0; q < s->nplanes; ++q) {
            const float *h = hp[(size_t)k * 3 + q];
            if (!h) continue;
            CUDA_TRY(staged_copy(rq, *s->pool, true, dst + s->poff[q],
                                 (size_t)s->stride * sizeof(float), h,
                                 (size_t)src_strides[(size_t)k * 3 + q],
                                 (size_t)s->pw[q] * sizeof(float), s->ph[q]));
        }
    }
    if (s->prop) {
        // proposer embeddings of the matching plane (plane 0 of the reference
        // frame in the final stage, of the source frame in the basic stage)
        const float *m = stream_slot(s, slot) + (s->final_ ? s->frame_floats : 0) + s->poff[0];
        CUDA_TRY(launch_embed(m, s->frame_floats, 1, s->pw[0], s->ph[0], s->stride,
                              proposer_frag(s->prop), proposer_bias(s->prop),
                              s->d_emb + (size_t)slot * s->emb_bytes, (long long)s->emb_bytes,
                              proposer_err(s->prop), st));
    }
    CUDA_TRY(cudaEventRecord(s->fslot[slot].ready, st));
    return BM3D_B200_OK;
}

// Block matching and filtering of the windows `wins` (their raw slots `wsl`)
// as one launch per kernel; fsl_of(f) gives the frame slot of frame f.
template <typename F>
int stream_filter(bm3d_b200_stream *s, bm3d_b200_stream::Request &q,
                  const std::vector<int> &wins, const std::vector<int> &wsl, F &&fsl_of) {
    const int k = (int)wins.size();
    if (k == 0) return BM3D_B200_OK;
    const int N = s->nframes, r = s->r, tw = s->tw;
    for (int j = 0; j < k; ++j)
        CUDA_TRY(cudaMemsetAsync(s->d_raw + (size_t)wsl[j] * s->raw_floats, 0,
                                 (size_t)s->raw_floats * sizeof(float), q.s));
    const size_t per_table = (size_t)k * tw;
    const int njobs = s->prm.chroma ? 1 : s->nplanes;
    for (int job = 0; job < njobs; ++job) {
        const int mq = job;  // matching plane (plane 0 with chroma)
        if (!s->prm.chroma && !s->process[mq]) continue;
        const int q0 = s->prm.chroma ? 0 : mq, q1 = s->prm.chroma ? 2 : mq;
        // tables of this job: [match][per plane q: src, ref, acc], each [k][tw]
        void **ht = q.h_tab + (size_t)job * 10 * per_table;
        void **dt = q.d_tab + (size_t)job * 10 * per_table;
        for (int j = 0; j < k; ++j)
            for (int z = 0; z < tw; ++z) {
                const int f = std::min(std::max(wins[j] - r + z, 0), N - 1);
                const float *fr = stream_slot(s, fsl_of(f));
                const size_t t = (size_t)j * tw + z;
                ht[t] = (void *)((s->final_ ? fr + s->frame_floats : fr) + s->poff[mq]);
                for (int qq = q0; qq <= q1; ++qq) {
                    void **hq = ht + (size_t)(1 + 3 * (qq - q0)) * per_table;
                    const size_t plane = (size_t)s->ph[qq] * s->stride;
                    hq[t] = (void *)(fr + s->poff[qq]);
                    hq[per_table + t] = s->final_ ? (void *)(fr + s->frame_floats + s->poff[qq])
                                                  : nullptr;
                    hq[2 * per_table + t] =
                        (void *)(s->d_raw + (size_t)wsl[j] * s->raw_floats + s->rawoff[qq] +
                                 (size_t)z * 2 * plane);
                }
            }
        CUDA_TRY(cudaMemcpyAsync(dt, ht, (size_t)(1 + 3 * (q1 - q0 + 1)) * per_table * sizeof(void *),
                                 cudaMemcpyHostToDevice, q.s));
        const int pq = s->prm.chroma ? 0 : mq;
        MatchParams mp = make_match_params(
            s->geo[mq], reinterpret_cast<const float *const *>(dt), q.d_matches, s->pw[mq],
            s->ph[mq], s->stride, s->prm.block_step[pq], s->prm.bm_range[pq], r,
            s->prm.ps_num[pq], s->prm.ps_range[pq]);
        mp.metric = s->metric[pq];
        if (s->prop && mq == 0) {
            // learned matching: embedding table of the windows' frames, the
            // learned search, then the exhaustive re-search of listed blocks
            void **he = q.h_tab + (size_t)3 * 10 * (2 * r + 1) * tw;
            void **de = q.d_tab + (size_t)3 * 10 * (2 * r + 1) * tw;
            for (int j = 0; j < k; ++j)
                for (int z = 0; z < tw; ++z) {
                    const int f = std::min(std::max(wins[j] - r + z, 0), N - 1);
                    he[(size_t)j * tw + z] = s->d_emb + (size_t)fsl_of(f) * s->emb_bytes;
                }
            CUDA_TRY(cudaMemcpyAsync(de, he, per_table * sizeof(void *), cudaMemcpyHostToDevice,
                                     q.s));
            const int nblk = mp.nbx * mp.nby;
            LearnedParams lp{};
            lp.embs = reinterpret_cast<const void *const *>(de);
            lp.w2 = s->pw[0] / 2;
            lp.cells_s = s->cells_s;
            lp.cells_t = s->cells_t;
            const float sg = s->prm.sigma[0] / 255.0f;
            lp.fallback_ssd = s->fb_tau > 0.0f ? s->fb_tau * 128.0f * sg * sg : 0.0f;
            unsigned *fbcount = q.d_fb + (size_t)(2 * r + 1) * s->max_blk;
            lp.fallback = q.d_fb;
            lp.fallback_count = fbcount;
            lp.fallback_capacity = (unsigned)((size_t)k * nblk);
            MatchParams lm = mp;
            lm.pitch = s->lgeo.pitch;
            lm.tile_rows = s->lgeo.tile_rows;
            CUDA_TRY(cudaMemsetAsync(fbcount, 0, sizeof(unsigned), q.s));
            CUDA_TRY(launch_learned_match(lm, lp, s->lgeo, k, q.s));
            if (lp.fallback_ssd > 0.0f) CUDA_TRY(launch_match_fallback(mp, q.d_fb, fbcount, q.s));
        } else {
            CUDA_TRY(launch_match(mp, s->geo[mq], k, q.s));
        }
        for (int qq = q0; qq <= q1; ++qq) {
            if (!s->process[qq]) continue;
            void **dq = dt + (size_t)(1 + 3 * (qq - q0)) * per_table;
            FilterParams fp{};
            fp.src = reinterpret_cast<const float *const *>(dq);
            fp.ref = s->final_ ? reinterpret_cast<const float *const *>(dq + per_table) : nullptr;
            fp.acc = reinterpret_cast<float *const *>(dq + 2 * per_table);
            fp.mult = nullptr;
            fp.matches = q.d_matches;
            fp.weight_offset = (long long)s->ph[qq] * s->stride;
            fp.acc_stride = s->stride;
            fp.stride = s->stride;
            fp.radius = r;
            fp.nblk = s->geo[mq].nbx * s->geo[mq].nby;
            fp.nbx = s->geo[mq].nbx;
            fp.corner_weight = 0;
            fp.win0 = 0;
            fp.nwin = k;
            fp.sigma = s->sigma[qq];
            fp.extractor = s->prm.extractor_exp ? std::ldexp(1.0f, s->prm.extractor_exp) : 0.0f;
            fp.t2d = s->tx2[s->prm.chroma ? 0 : qq];
            fp.t1d = s->tx1[s->prm.chroma ? 0 : qq];
            CUDA_TRY(launch_filter(fp, s->final_, q.s));
        }
    }
    for (int j = 0; j < k; ++j) CUDA_TRY(cudaEventRecord(s->wslot[wsl[j]].ready, q.s));
    return BM3D_B200_OK;
}

void stream_release(bm3d_b200_stream *s, int qi, const StreamClaims &c) {
    // the request's GPU work is complete (or abandoned) before its slots and
    // tables are handed on
    cudaStreamSynchronize(s->req[qi].s);
    std::lock_guard<std::mutex> lk(s->mu);
    for (int i : c.fs) --s->fslot[i].pins;
    for (int i : c.ws) --s->wslot[i].pins;
    s->req[qi].busy = false;
    s->cv.notify_all();
}

void stream_free_device(bm3d_b200_stream *s) {
    for (auto &q : s->req) {
        if (q.s) {
            cudaStreamSynchronize(q.s);
            cudaStreamDestroy(q.s);
        }
        for (auto &e : q.ev)
            if (e) cudaEventDestroy(e);
        cudaFree(q.d_out);
        cudaFree(q.d_matches);
        cudaFree(q.d_tab);
        cudaFreeHost(q.h_tab);
        cudaFree(q.d_fb);
        for (int b = 0; b < 2; ++b) {
            cudaFreeHost(q.h_stage[b]);
            if (q.stage_ev[b]) cudaEventDestroy(q.stage_ev[b]);
        }
        q = bm3d_b200_stream::Request{};
    }
    for (auto *v : {&s->fslot, &s->wslot})
        for (auto &sl : *v)
            if (sl.ready) cudaEventDestroy(sl.ready);
    cudaFree(s->d_frames);
    cudaFree(s->d_raw);
    cudaFree(s->d_emb);
    s->d_frames = s->d_raw = nullptr;
    s->d_emb = nullptr;
}

}  // namespace

extern "C" int bm3d_b200_stream_create(bm3d_b200_stream **out, int width, int height,
                                       int num_planes, int subsampling_w, int subsampling_h,
                                       int num_frames, const bm3d_b200_params *params, int final_,
                                       int device_id) {
    if (!out) return fail(BM3D_B200_ERR_INVALID, "BM3D: null output handle");
    *out = nullptr;
    if (!params) return fail(BM3D_B200_ERR_INVALID, "BM3D: null params");
    if (num_planes != 1 && num_planes != 3)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: clips have 1 or 3 planes");
    if (num_frames <= 0) return fail(BM3D_B200_ERR_INVALID, "BM3D: clip has no frames");
    if (subsampling_w < 0 || subsampling_h < 0 || subsampling_w > 2 || subsampling_h > 2)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid subsampling");
    const bm3d_b200_params &p = *params;
    if (p.chroma && (num_planes != 3 || subsampling_w || subsampling_h))
        return fail(BM3D_B200_ERR_INVALID, "BM3D: clip format must be YUV444 when \"chroma\" is true");
    for (int i = 0; i < 3; ++i)
        if (!(p.sigma[i] >= 0.0f)) return fail(BM3D_B200_ERR_INVALID, "BM3D: \"sigma\" must be non-negative");
    const int stride = (width + 31) / 32 * 32;
    for (int q = 0; q < num_planes; ++q) {
        const int pq = p.chroma ? 0 : q;
        const bool matched = p.chroma ? q == 0 : !(p.sigma[q] < FLT_EPSILON);
        if (!matched) continue;
        const int w = q == 0 ? width : width >> subsampling_w;
        const int h = q == 0 ? height : height >> subsampling_h;
        if (int rc = check_search(w, h, stride, p.block_step[pq], p.bm_range[pq], p.radius,
                                  p.ps_num[pq], p.ps_range[pq]))
            return rc;
    }
    int count = 0;
    CUDA_TRY(cudaGetDeviceCount(&count));
    if (device_id < 0 || device_id >= count)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid device ID (%d)", device_id);
    CUDA_TRY(cudaSetDevice(device_id));
    auto *s = new (std::nothrow) bm3d_b200_stream;
    if (!s) return fail(BM3D_B200_ERR_NOMEM, "BM3D: out of host memory");
    auto cleanup = [&](int rc) {
        bm3d_b200_stream_destroy(s);
        return rc;
    };
    s->device = device_id;
    try {
        s->pool.reset(new CopyPool(copy_pool_threads()));
    } catch (...) {
        return cleanup(fail(BM3D_B200_ERR_NOMEM, "BM3D: cannot start the host copy threads"));
    }
    s->width = width;
    s->height = height;
    s->nplanes = num_planes;
    s->ssw = subsampling_w;
    s->ssh = subsampling_h;
    s->nframes = num_frames;
    s->prm = p;
    s->final_ = final_ != 0;
    s->stride = stride;
    s->r = p.radius;
    s->tw = 2 * p.radius + 1;
    long long off = 0, roff = 0;
    for (int q = 0; q < num_planes; ++q) {
        s->pw[q] = q == 0 ? width : width >> subsampling_w;
        s->ph[q] = q == 0 ? height : height >> subsampling_h;
        s->poff[q] = off;
        s->rawoff[q] = roff;
        off += (long long)s->ph[q] * stride;
        roff += (long long)s->ph[q] * stride * 2 * s->tw;
        s->process[q] = !(p.sigma[q] < FLT_EPSILON);
        s->sigma[q] = bm3d_b200_scale_sigma(p.sigma[q], s->final_ ? 1 : 0);
        s->max_plane = std::max(s->max_plane, (size_t)s->ph[q] * stride);
        const int pq = p.chroma ? 0 : q;
        const bool matched = p.chroma ? q == 0 : s->process[q];
        if (!matched) continue;
        s->geo[q] = match_geometry(s->pw[q], s->ph[q], p.block_step[pq], p.bm_range[pq],
                                   p.radius, p.ps_range[pq]);
        s->max_blk = std::max(s->max_blk, (size_t)s->geo[q].nbx * s->geo[q].nby);
    }
    s->frame_floats = off;
    s->raw_floats = roff;
    // Concurrent requests: as many as the reference's fast=True resources,
    // fewer when one request's frames and windows pass 16 GiB.
    const int fper = 4 * p.radius + 1, wper = 2 * p.radius + 1;
    const double req_bytes = ((double)fper * (s->final_ ? 2 : 1) * s->frame_floats +
                              (double)wper * s->raw_floats) * sizeof(float);
    s->nreq = std::max(1, std::min(kStreamRequests, (int)((double)(16ull << 30) / req_bytes)));
    s->fslot.resize((size_t)s->nreq * fper);
    s->wslot.resize((size_t)s->nreq * wper);
    const size_t tab = (size_t)wper * (3 * 10 + 1) * s->tw;
    cudaError_t e = cudaMalloc(&s->d_frames, s->fslot.size() * (s->final_ ? 2 : 1) *
                                                 s->frame_floats * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_raw, s->wslot.size() * s->raw_floats * sizeof(float));
    for (auto *v : {&s->fslot, &s->wslot})
        for (auto &sl : *v)
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.ready, cudaEventDisableTiming);
    for (int i = 0; i < s->nreq && e == cudaSuccess; ++i) {
        auto &q = s->req[i];
        e = cudaStreamCreateWithFlags(&q.s, cudaStreamNonBlocking);
        for (auto &ev : q.ev)
            if (e == cudaSuccess) e = cudaEventCreate(&ev);
        if (e == cudaSuccess) e = cudaMalloc(&q.d_out, s->max_plane * sizeof(float));
        if (e == cudaSuccess)
            e = cudaMalloc(&q.d_matches, (size_t)wper * s->max_blk * 8 * sizeof(int));
        if (e == cudaSuccess) e = cudaMalloc(&q.d_tab, tab * sizeof(void *));
        if (e == cudaSuccess) e = cudaMallocHost(&q.h_tab, tab * sizeof(void *));
        if (e == cudaSuccess)
            e = cudaMalloc(&q.d_fb, ((size_t)wper * s->max_blk + 1) * sizeof(unsigned));
        for (int b = 0; b < 2; ++b) {
            if (e == cudaSuccess) e = cudaMallocHost(&q.h_stage[b], kStageBytes);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&q.stage_ev[b], cudaEventDisableTiming);
        }
    }
    s->nuse = s->nreq;
    if (e != cudaSuccess)
        return cleanup(fail(BM3D_B200_ERR_NOMEM, "BM3D: stream allocation failed: %s",
                            cudaGetErrorString(e)));
    *out = s;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_stream_set_variant(bm3d_b200_stream *s, const int *bm_error,
                                            const int *transform_2d, const int *transform_1d) {
    if (!s) return fail(BM3D_B200_ERR_INVALID, "BM3D: null stream");
    for (int q = 0; q < 3; ++q) {
        const int m = bm_error ? bm_error[q] : 0, a = transform_2d ? transform_2d[q] : 0,
                  b = transform_1d ? transform_1d[q] : 0;
        if (m < BM3D_B200_BM_SSD || m > BM3D_B200_BM_SSD_NORM)
            return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'bm_error_s': %d", m);
        if (a < BM3D_B200_TX_DCT || a > BM3D_B200_TX_BIOR1_5)
            return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'transform_2d_s': %d", a);
        if (b < BM3D_B200_TX_DCT || b > BM3D_B200_TX_BIOR1_5)
            return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid 'transform_1d_s': %d", b);
    }
    std::unique_lock<std::mutex> lk(s->mu);
    // no request in flight while the variant changes
    s->cv.wait(lk, [&] {
        for (int i = 0; i < s->nreq; ++i)
            if (s->req[i].busy) return false;
        return true;
    });
    if (s->prop && (bm_error || transform_2d || transform_1d))
        for (int q = 0; q < 3; ++q)
            if ((bm_error && bm_error[q]) || (transform_2d && transform_2d[q]) ||
                (transform_1d && transform_1d[q]))
                return fail(BM3D_B200_ERR_UNSUPPORTED,
                            "BM3D: learned matching runs with the SSD and DCT defaults only");
    for (int q = 0; q < 3; ++q) {
        s->metric[q] = bm_error ? bm_error[q] : 0;
        s->tx2[q] = transform_2d ? transform_2d[q] : 0;
        s->tx1[q] = transform_1d ? transform_1d[q] : 0;
    }
    // results computed with the previous variant are no longer valid
    for (auto &sl : s->wslot) {
        sl.key = -1;
        sl.state = 0;
    }
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_stream_frame(bm3d_b200_stream *s, int n, const float *const *h_src,
                                      const float *const *h_ref, const int *src_strides,
                                      float *const *h_dst, const int *dst_strides) {
    if (!s || !h_src || !src_strides || !h_dst || !dst_strides)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: null argument");
    if (s->final_ && !h_ref) return fail(BM3D_B200_ERR_INVALID, "BM3D: final stage needs ref frames");
    if (n < 0 || n >= s->nframes)
        return fail(BM3D_B200_ERR_INVALID, "BM3D: frame %d outside the clip", n);
    CUDA_TRY(cudaSetDevice(s->device));
    const int r = s->r, tw = s->tw, N = s->nframes;
    const int first = n - 2 * r;  // host arrays hold frames clamp(first + i), i = 0 .. 4r
    auto clampf = [&](int f) { return std::min(std::max(f, 0), N - 1); };

    // ---- claims (under the lock) -------------------------------------------
    int qi = -1;
    StreamClaims c;
    int wslot_of[2 * BM3D_B200_MAX_RADIUS + 1];
    std::vector<int> wprod_win;  // windows this request produces (with c.wprod)
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv.wait(lk, [&] {
            for (int i = 0; i < s->nuse; ++i)
                if (!s->req[i].busy) return true;
            return false;
        });
        for (int i = 0; i < s->nuse; ++i)
            if (!s->req[i].busy) {
                qi = i;
                break;
            }
        s->req[qi].busy = true;
        const unsigned long long tick = ++s->tick;
        for (int i = 0; i < tw; ++i) {
            const int w = clampf(n - r + i);
            int found = -1;
            for (int j = 0; j < i; ++j)
                if (clampf(n - r + j) == w) found = wslot_of[j];
            if (found >= 0) {
                wslot_of[i] = found;
                continue;
            }
            bool produce = false;
            const int sl = claim_slot(s->wslot, w, tick, &produce);
            if (sl < 0) {  // cannot happen: the ring holds every request's windows
                for (int k : c.ws) --s->wslot[k].pins;
                s->req[qi].busy = false;
                s->cv.notify_all();
                return fail(BM3D_B200_ERR_INVALID, "BM3D: window ring exhausted");
            }
            wslot_of[i] = sl;
            c.ws.push_back(sl);
            if (produce) {
                c.wprod.push_back(sl);
                wprod_win.push_back(w);
            }
        }
        // frames of the windows this request produces
        for (int w : wprod_win)
            for (int z = 0; z < tw; ++z) {
                const int f = clampf(w - r + z);
                bool have = false;
                for (int k : c.fs) have |= s->fslot[k].key == f;
                if (have) continue;
                bool produce = false;
                const int sl = claim_slot(s->fslot, f, tick, &produce);
                if (sl < 0) {
                    for (int k : c.ws) --s->wslot[k].pins;
                    for (int k : c.wprod) {
                        s->wslot[k].key = -1;
                        s->wslot[k].state = 0;
                    }
                    for (int k : c.fs) --s->fslot[k].pins;
                    for (int k : c.fprod) {
                        s->fslot[k].key = -1;
                        s->fslot[k].state = 0;
                    }
                    s->req[qi].busy = false;
                    s->cv.notify_all();
                    return fail(BM3D_B200_ERR_INVALID, "BM3D: frame ring exhausted");
                }
                c.fs.push_back(sl);
                if (produce) c.fprod.push_back(sl);
            }
    }
    auto &q = s->req[qi];
    // On failure: abandon what this request was producing, release the rest.
    auto abandon = [&](int rc) {
        cudaStreamSynchronize(q.s);
        finish_slots(s, s->fslot, c.fprod, false);
        finish_slots(s, s->wslot, c.wprod, false);
        stream_release(s, qi, c);
        return rc;
    };
    auto frame_slot_of = [&](int f) {
        for (int k : c.fs)
            if (s->fslot[k].key == f) return k;
        return 0;  // unreachable: every frame of a produced window is claimed
    };

    // ---- uploads of the frames this request produces -------------------------
    if (cudaEventRecord(q.ev[0], q.s) != cudaSuccess)
        return abandon(fail(BM3D_B200_ERR_CUDA, "BM3D: event record failed"));
    while (!c.fprod.empty()) {
        const int sl = c.fprod.front();
        if (int rc = stream_upload(s, q, sl, s->fslot[sl].key, first, h_src, h_ref, src_strides))
            return abandon(rc);
        std::lock_guard<std::mutex> lk(s->mu);
        s->fslot[sl].state = 2;
        ++s->uploads;
        c.fprod.erase(c.fprod.begin());  // produced: ready for every request
        s->cv.notify_all();
    }
    if (cudaEventRecord(q.ev[1], q.s) != cudaSuccess)
        return abandon(fail(BM3D_B200_ERR_CUDA, "BM3D: event record failed"));

    // ---- windows this request produces: one batched launch per kernel -------
    if (!c.wprod.empty()) {
        // frames uploaded by other requests: order this stream after them
        for (int sl : c.fs) {
            const int f = s->fslot[sl].key;
            {
                std::unique_lock<std::mutex> lk(s->mu);
                if (!wait_ready(s, lk, s->fslot, sl, f))
                    return abandon(fail(BM3D_B200_ERR_CUDA,
                                        "BM3D: a concurrent request failed to upload frame %d", f));
            }
            if (cudaStreamWaitEvent(q.s, s->fslot[sl].ready, 0) != cudaSuccess)
                return abandon(fail(BM3D_B200_ERR_CUDA, "BM3D: stream wait failed"));
        }
        if (int rc = stream_filter(s, q, wprod_win, c.wprod, frame_slot_of)) return abandon(rc);
        finish_slots(s, s->wslot, c.wprod, true);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->windows += (long long)c.wprod.size();
        }
        c.wprod.clear();
    }
    if (cudaEventRecord(q.ev[2], q.s) != cudaSuccess)
        return abandon(fail(BM3D_B200_ERR_CUDA, "BM3D: event record failed"));

    // ---- windows of other requests, then VAggregate and the download --------
    for (int i = 0; i < tw; ++i) {
        const int sl = wslot_of[i], w = clampf(n - r + i);
        {
            std::unique_lock<std::mutex> lk(s->mu);
            if (!wait_ready(s, lk, s->wslot, sl, w))
                return abandon(fail(BM3D_B200_ERR_CUDA,
                                    "BM3D: a concurrent request failed to filter window %d", w));
        }
        if (cudaStreamWaitEvent(q.s, s->wslot[sl].ready, 0) != cudaSuccess)
            return abandon(fail(BM3D_B200_ERR_CUDA, "BM3D: stream wait failed"));
    }
    for (int pq = 0; pq < s->nplanes; ++pq) {
        if (!s->process[pq] || !h_dst[pq]) continue;
        VAggregateParams vp{};
        vp.dst = q.d_out;
        for (int i = 0; i < tw; ++i)
            vp.vf[i] = s->d_raw + (size_t)wslot_of[i] * s->raw_floats + s->rawoff[pq];
        vp.dst_stride = s->stride;
        vp.raw_stride = s->stride;
        vp.width = s->pw[pq];
        vp.height = s->ph[pq];
        vp.radius = r;
        vp.n0 = n;
        vp.num_frames = N;
        vp.nout = 1;
        cudaError_t e = launch_vaggregate(vp, q.s);
        if (e == cudaSuccess)
            e = staged_copy(q, *s->pool, false, h_dst[pq], (size_t)dst_strides[pq], q.d_out,
                            (size_t)s->stride * sizeof(float), (size_t)s->pw[pq] * sizeof(float),
                            s->ph[pq]);
        if (e != cudaSuccess)
            return abandon(fail(BM3D_B200_ERR_CUDA, "BM3D: output of frame %d failed: %s", n,
                                cudaGetErrorString(e)));
    }
    cudaError_t e = cudaEventRecord(q.ev[3], q.s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(q.s);
    if (e != cudaSuccess)
        return abandon(fail(BM3D_B200_ERR_CUDA, "BM3D: frame %d failed: %s", n,
                            cudaGetErrorString(e)));
    if (s->prop)
        if (int rc = proposer_check(s->prop)) {
            // the embeddings of some frame are incomplete: nothing kept is trusted
            stream_release(s, qi, c);
            std::lock_guard<std::mutex> lk(s->mu);
            for (auto *v : {&s->fslot, &s->wslot})
                for (auto &sl : *v)
                    if (!sl.pins) {
                        sl.key = -1;
                        sl.state = 0;
                    }
            return rc;
        }
    float t[3] = {0.0f, 0.0f, 0.0f};
    for (int i = 0; i < 3; ++i) cudaEventElapsedTime(&t[i], q.ev[i], q.ev[i + 1]);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->ms_upload += t[0];
        s->ms_filter += t[1];
        s->ms_output += t[2];
        ++s->calls;
    }
    stream_release(s, qi, c);
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_stream_stats(bm3d_b200_stream *s, long long *frame_uploads,
                                      long long *windows) {
    if (!s) return fail(BM3D_B200_ERR_INVALID, "BM3D: null stream");
    std::lock_guard<std::mutex> lk(s->mu);
    if (frame_uploads) *frame_uploads = s->uploads;
    if (windows) *windows = s->windows;
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_stream_timings(bm3d_b200_stream *s, double *ms, long long *calls,
                                        int reset) {
    if (!s) return fail(BM3D_B200_ERR_INVALID, "BM3D: null stream");
    std::lock_guard<std::mutex> lk(s->mu);
    if (ms) {
        ms[0] = s->ms_upload;
        ms[1] = s->ms_filter;
        ms[2] = s->ms_output;
    }
    if (calls) *calls = s->calls;
    if (reset) {
        s->ms_upload = s->ms_filter = s->ms_output = 0.0;
        s->calls = 0;
    }
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_stream_concurrency(const bm3d_b200_stream *s) {
    return s ? s->nuse : 0;
}

namespace {

// Waits until no request is in flight (lock held through lk).
void stream_wait_idle(bm3d_b200_stream *s, std::unique_lock<std::mutex> &lk) {
    s->cv.wait(lk, [&] {
        for (int i = 0; i < s->nreq; ++i)
            if (s->req[i].busy) return false;
        return true;
    });
}

}  // namespace

extern "C" int bm3d_b200_stream_set_concurrency(bm3d_b200_stream *s, int requests) {
    if (!s) return fail(BM3D_B200_ERR_INVALID, "BM3D: null stream");
    if (requests < 1) return fail(BM3D_B200_ERR_INVALID, "BM3D: at least one request");
    std::unique_lock<std::mutex> lk(s->mu);
    stream_wait_idle(s, lk);
    s->nuse = std::min(requests, s->nreq);
    return BM3D_B200_OK;
}

extern "C" int bm3d_b200_stream_set_proposer(bm3d_b200_stream *s, bm3d_b200_proposer *p,
                                             int cells_spatial, int cells_temporal,
                                             float fallback_tau) {
    if (!s) return fail(BM3D_B200_ERR_INVALID, "BM3D: null stream");
    if (p) {
        if (cells_spatial < 1 || cells_spatial > 8 || cells_temporal < 1 || cells_temporal > 8)
            return fail(BM3D_B200_ERR_INVALID,
                        "BM3D: proposal cell counts must be in range [1, 8]");
        if (!(fallback_tau >= 0.0f))
            return fail(BM3D_B200_ERR_INVALID, "BM3D: invalid fallback_tau");
        for (int q = 0; q < 3; ++q)
            if (s->metric[q] || s->tx2[q] || s->tx1[q])
                return fail(BM3D_B200_ERR_UNSUPPORTED,
                            "BM3D: learned matching runs with the SSD and DCT defaults only");
        if (s->nplanes != 1 && !s->prm.chroma)
            return fail(BM3D_B200_ERR_UNSUPPORTED,
                        "BM3D: learned matching needs a single-plane clip or chroma matching");
        if (proposer_device(p) != s->device)
            return fail(BM3D_B200_ERR_INVALID,
                        "BM3D: proposer and stream are on different devices");
        if (s->pw[0] < 16 || s->ph[0] < 16)
            return fail(BM3D_B200_ERR_INVALID,
                        "BM3D: learned matching needs planes of 16x16 or more");
    }
    CUDA_TRY(cudaSetDevice(s->device));
    std::unique_lock<std::mutex> lk(s->mu);
    stream_wait_idle(s, lk);
    if (p) {
        const MatchGeometry lg = learned_geometry(s->pw[0], s->ph[0], s->prm.block_step[0],
                                                  s->prm.bm_range[0], s->r, s->prm.ps_range[0]);
        if (lg.smem > 220 * 1024 ||
            !learned_ordinals_fit(s->prm.bm_range[0], s->prm.ps_num[0], s->prm.ps_range[0]))
            return fail(BM3D_B200_ERR_UNSUPPORTED,
                        "BM3D: search range too large for learned matching");
        if (!s->d_emb) {
            s->emb_bytes = (size_t)(s->pw[0] / 2) * (s->ph[0] / 2) * 16;
            CUDA_TRY(cudaMalloc(&s->d_emb, s->fslot.size() * s->emb_bytes));
        }
        s->lgeo = lg;
        s->cells_s = cells_spatial;
        s->cells_t = cells_temporal;
        s->fb_tau = fallback_tau;
    }
    s->prop = p;
    // frames uploaded without embeddings and windows matched another way
    for (auto *v : {&s->fslot, &s->wslot})
        for (auto &sl : *v) {
            sl.key = -1;
            sl.state = 0;
        }
    return BM3D_B200_OK;
}

extern "C" void bm3d_b200_stream_destroy(bm3d_b200_stream *s) {
    if (!s) return;
    cudaSetDevice(s->device);
    stream_free_device(s);
    delete s;
}

// ===========================================================================
// 6. diagnostics
// ===========================================================================
namespace {

__global__ void selftest_rcp_kernel(unsigned lo, unsigned hi, unsigned long long *count,
                                    unsigned *first_bad) {
    const unsigned long long step = (unsigned long long)gridDim.x * blockDim.x;
    for (unsigned long long i = (unsigned long long)lo + blockIdx.x * blockDim.x + threadIdx.x;
         i < hi; i += step) {
        const float a = __uint_as_float((unsigned)i);
        if (__float_as_uint(rcp_rn_normal(a)) != __float_as_uint(__frcp_rn(a))) {
            atomicAdd(count, 1ULL);
            atomicMin(first_bad, (unsigned)i);
        }
    }
}

}  // namespace

extern "C" int bm3d_b200_selftest_reciprocal(unsigned lo_bits, unsigned hi_bits,
                                             unsigned long long *mismatches,
                                             unsigned *first_bad) {
    if (!mismatches || lo_bits > hi_bits)
        return fail(BM3D_B200_ERR_INVALID, "selftest: invalid arguments");
    unsigned long long *d_count = nullptr;
    CUDA_TRY(cudaMalloc(&d_count, sizeof(unsigned long long) + sizeof(unsigned)));
    unsigned *d_first = reinterpret_cast<unsigned *>(d_count + 1);
    unsigned init_first = 0xffffffffu;
    cudaError_t e = cudaMemset(d_count, 0, sizeof(unsigned long long));
    if (e == cudaSuccess)
        e = cudaMemcpy(d_first, &init_first, sizeof(unsigned), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        selftest_rcp_kernel<<<148 * 8, 256>>>(lo_bits, hi_bits, d_count, d_first);
        e = cudaGetLastError();
    }
    unsigned first = 0;
    if (e == cudaSuccess)
        e = cudaMemcpy(mismatches, d_count, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(&first, d_first, sizeof(unsigned), cudaMemcpyDeviceToHost);
    cudaFree(d_count);
    if (e != cudaSuccess)
        return fail(BM3D_B200_ERR_CUDA, "selftest: %s", cudaGetErrorString(e));
    if (first_bad) *first_bad = first;
    return BM3D_B200_OK;
}
