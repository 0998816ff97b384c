// Test infrastructure only: a harness around the reference's own CUDA BM3D
// kernel (source/kernel.cu), compiled unchanged from the reference tree by
// oracle/Makefile into oracle/_ref/. Nothing in the product links this file;
// it is the checker and the GPU reference timing, never the thing shipped.
//
// The reference file is #included as one translation unit, so its `static`
// kernel template bm3d<temporal, chroma, final_> and get_graphexec are
// callable here. Two builds: `fast` with --use_fast_math, the flags the
// reference ships with (README.md, .github/workflows/linux.yml), and `exact`
// without it (IEEE division in the weights), the parity build.
//
// Entry points (extern "C"):
//   refgpu_graph_create/launch/destroy - get_graphexec (source/kernel.cu:759-864)
//       and cudaGraphLaunch, exactly as the plugin uses them
//       (source/source.cpp:676-693, 348, 401).
//   refgpu_kernel - the graph's kernel node alone (same template and grid,
//       source/kernel.cu:808-830) on a caller's stream, for device-resident
//       kernel timing.
//   refgpu_vbm3d_twostage - the plugin's BM3Dv2 two-stage V-BM3D over a clip
//       in host memory, driven the way VapourSynth drives the plugin with
//       fast=True: worker threads run getFrame (source/source.cpp:206-441),
//       a pool of 4 GPU resources (pinned h_res, d_src, d_res, stream, graph)
//       guarded by a lock and the ticket semaphore (source/source.cpp:64-83,
//       299-303, 636-720), pinned staging by row copies (vs_bitblt), and the
//       host VAggregate filter (source/source.cpp:746-862).
#include BM3D_REF_GPU_SOURCE

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace {

thread_local std::string g_err;

int fail(const char *what, cudaError_t e) {
    g_err = std::string(what) + ": " + cudaGetErrorString(e);
    return 1;
}

#define RTRY(expr)                                 \
    do {                                           \
        cudaError_t e_ = (expr);                   \
        if (e_ != cudaSuccess) return fail(#expr, e_); \
    } while (0)

// Row copy of a pitched plane (VapourSynth's vs_bitblt for float rows).
void bitblt(float *dst, size_t dst_stride, const float *src, size_t src_stride, int width,
            int height) {
    for (int y = 0; y < height; ++y)
        std::memcpy(dst + (size_t)y * dst_stride, src + (size_t)y * src_stride,
                    (size_t)width * sizeof(float));
}

// One GPU resource of the plugin's pool (source/source.cpp:649-710, luma only).
struct Res {
    float *d_src = nullptr, *d_res = nullptr, *h_res = nullptr;
    cudaStream_t stream = nullptr;
    cudaGraphExec_t exec[2] = {nullptr, nullptr};  // basic, final
};

// The scale the plugin applies to the user's sigma (source/source.cpp:520-523).
float scaled_sigma(float s, bool final_) {
    return s * (3.f / 4.f) / 255.f * 64.f * (final_ ? 1.0f : 2.7f);
}

}  // namespace

extern "C" {

const char *refgpu_last_error(void) { return g_err.c_str(); }

void *refgpu_graph_create(float *d_res, float *d_src, float *h_res, int width, int height,
                          int stride, float sigma, int block_step, int bm_range, int radius,
                          int ps_num, int ps_range, int chroma, float sigma_u, float sigma_v,
                          int final_, float extractor) {
    return (void *)get_graphexec(d_res, d_src, h_res, width, height, stride, sigma, block_step,
                                 bm_range, radius, ps_num, ps_range, chroma != 0, sigma_u,
                                 sigma_v, final_ != 0, extractor);
}

int refgpu_graph_launch(void *exec, void *stream) {
    RTRY(cudaGraphLaunch((cudaGraphExec_t)exec, (cudaStream_t)stream));
    return 0;
}

void refgpu_graph_destroy(void *exec) {
    if (exec) cudaGraphExecDestroy((cudaGraphExec_t)exec);
}

int refgpu_kernel(float *d_res, const float *d_src, int width, int height, int stride,
                  float sigma, int block_step, int bm_range, int radius, int ps_num,
                  int ps_range, int chroma, float sigma_u, float sigma_v, int final_,
                  float extractor, void *stream) {
    const dim3 grid((width + (4 * block_step - 1)) / (4 * block_step),
                    (height + (block_step - 1)) / block_step);
    cudaStream_t s = (cudaStream_t)stream;
#define REFGPU_LAUNCH(T, C, F)                                                              \
    bm3d<T, C, F><<<grid, 32, 0, s>>>(d_res, d_src, width, height, stride, sigma, block_step, \
                                      bm_range, radius, ps_num, ps_range, sigma_u, sigma_v,  \
                                      extractor)
    const bool t = radius != 0, c = chroma != 0, f = final_ != 0;
    if (t && c && f) REFGPU_LAUNCH(true, true, true);
    else if (t && c) REFGPU_LAUNCH(true, true, false);
    else if (t && f) REFGPU_LAUNCH(true, false, true);
    else if (t) REFGPU_LAUNCH(true, false, false);
    else if (c && f) REFGPU_LAUNCH(false, true, true);
    else if (c) REFGPU_LAUNCH(false, true, false);
    else if (f) REFGPU_LAUNCH(false, false, true);
    else REFGPU_LAUNCH(false, false, false);
#undef REFGPU_LAUNCH
    RTRY(cudaGetLastError());
    return 0;
}

// Two-stage V-BM3D (vbasic = BM3Dv2(src), vfinal = BM3Dv2(src, ref=vbasic)) of
// a GRAYS clip h_src [num_frames][height][src_stride] into h_dst (same
// layout), with the reference plugin's host pipeline: `threads` worker
// threads, `resources` GPU resources (4 = fast=True). sigma is the user's
// value. extractor_exp > 0 selects the deterministic pre-rounded sums.
// stage_seconds (optional, 4 doubles): wall time of basic BM3D, its
// VAggregate, final BM3D, its VAggregate.
int refgpu_vbm3d_twostage(const float *h_src, float *h_dst, int num_frames, int width, int height,
                          int src_stride, float sigma, int block_step, int bm_range, int radius,
                          int ps_num, int ps_range, int extractor_exp, int threads,
                          int resources, int device_id, double *stage_seconds) {
    if (num_frames < 1 || width < 8 || height < 8 || radius < 1 || threads < 1 ||
        resources < 1) {
        g_err = "refgpu_vbm3d_twostage: bad arguments";
        return 1;
    }
    RTRY(cudaSetDevice(device_id));
    const int tw = 2 * radius + 1;
    const float extractor = extractor_exp ? std::ldexp(1.0f, extractor_exp) : 0.0f;

    // pool (source/source.cpp:636-710): d_src sized for the final stage
    std::vector<Res> pool(resources);
    size_t d_pitch = 0;
    int rc = 0;
    for (int i = 0; i < resources && rc == 0; ++i) {
        Res &r = pool[i];
        if (i == 0) {
            if (cudaMallocPitch(&r.d_src, &d_pitch, width * sizeof(float),
                                (size_t)2 * tw * height) != cudaSuccess)
                rc = fail("cudaMallocPitch", cudaGetLastError());
        } else if (cudaMalloc(&r.d_src, (size_t)2 * tw * height * d_pitch) != cudaSuccess) {
            rc = fail("cudaMalloc(d_src)", cudaGetLastError());
        }
        if (rc) break;
        if (cudaMalloc(&r.d_res, (size_t)tw * 2 * height * d_pitch) != cudaSuccess ||
            cudaMallocHost(&r.h_res, (size_t)2 * tw * 2 * height * d_pitch) != cudaSuccess ||
            cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking) != cudaSuccess) {
            rc = fail("resource allocation", cudaGetLastError());
            break;
        }
    }
    const int d_stride = (int)(d_pitch / sizeof(float));
    for (int i = 0; i < resources && rc == 0; ++i)
        for (int f = 0; f < 2; ++f) {
            pool[i].exec[f] = get_graphexec(pool[i].d_res, pool[i].d_src, pool[i].h_res, width,
                                            height, d_stride, scaled_sigma(sigma, f == 1),
                                            block_step, bm_range, radius, ps_num, ps_range,
                                            false, 0.0f, 0.0f, f == 1, extractor);
            if (!pool[i].exec[f]) rc = fail("get_graphexec", cudaGetLastError());
        }

    // raw V-BM3D frames [num_frames][2r+1][2][height][src_stride] and vbasic
    std::vector<float> raw, vbasic;
    if (rc == 0) {
        try {
            raw.resize((size_t)num_frames * tw * 2 * height * src_stride);
            vbasic.resize((size_t)num_frames * height * src_stride);
        } catch (...) {
            g_err = "host allocation failed";
            rc = 1;
        }
    }

    std::mutex lock;
    std::condition_variable cv;
    std::vector<int> free_res;
    for (int i = 0; i < resources; ++i) free_res.push_back(i);
    std::atomic<int> err{0};
    const size_t fsz = (size_t)height * src_stride;
    const size_t rsz = (size_t)tw * 2 * height * src_stride;

    // getFrame of BM3D for output frame n (source/source.cpp:206-441, luma)
    auto bm3d_frame = [&](int n, bool final_) {
        int ri;
        {
            std::unique_lock<std::mutex> g(lock);
            cv.wait(g, [&] { return !free_res.empty(); });
            ri = free_res.back();
            free_res.pop_back();
        }
        Res &r = pool[ri];
        float *h = r.h_res;
        const float *ref_clip = vbasic.data();
        for (int outer = 0; outer < (final_ ? 2 : 1); ++outer) {
            const float *clip = (final_ && outer == 0) ? ref_clip : h_src;
            for (int i = -radius; i <= radius; ++i) {
                const int f = std::min(std::max(n + i, 0), num_frames - 1);
                bitblt(h, d_stride, clip + (size_t)f * fsz, src_stride, width, height);
                h += (size_t)d_stride * height;
            }
        }
        if (cudaGraphLaunch(r.exec[final_ ? 1 : 0], r.stream) != cudaSuccess ||
            cudaStreamSynchronize(r.stream) != cudaSuccess)
            err.store(1);
        bitblt(raw.data() + (size_t)n * rsz, src_stride, r.h_res, d_stride, width,
               height * 2 * tw);
        {
            std::lock_guard<std::mutex> g(lock);
            free_res.push_back(ri);
        }
        cv.notify_one();
    };

    // getFrame of VAggregate for output frame n (source/source.cpp:746-862)
    auto vaggregate_frame = [&](int n, float *out) {
        std::vector<float> buffer(2 * (size_t)width);
        float *dstp = out + (size_t)n * fsz;
        for (int y = 0; y < height; ++y) {
            std::fill(buffer.begin(), buffer.end(), 0.0f);
            for (int i = 0; i < tw; ++i) {
                const int fid = std::min(std::max(n - radius + i, 0), num_frames - 1);
                const int slot = std::min(std::max(2 * radius - i, n - num_frames + 1 + radius),
                                          n + radius);
                const float *agg = raw.data() + (size_t)fid * rsz +
                                   ((size_t)slot * 2 * height + y) * src_stride;
                for (int x = 0; x < width; ++x) buffer[x] += agg[x];
                agg += (size_t)height * src_stride;
                for (int x = 0; x < width; ++x) buffer[width + x] += agg[x];
            }
            for (int x = 0; x < width; ++x) dstp[x] = buffer[x] / buffer[width + x];
            dstp += src_stride;
        }
    };

    auto parallel = [&](auto &&fn) {
        std::atomic<int> next{0};
        std::vector<std::thread> ts;
        for (int t = 0; t < threads; ++t)
            ts.emplace_back([&] {
                for (int n; (n = next.fetch_add(1)) < num_frames;) fn(n);
            });
        for (auto &t : ts) t.join();
    };

    if (rc == 0) {
        double secs[4] = {0, 0, 0, 0};
        auto now = [] { return std::chrono::steady_clock::now(); };
        auto t0 = now();
        parallel([&](int n) { bm3d_frame(n, false); });
        auto t1 = now();
        parallel([&](int n) { vaggregate_frame(n, vbasic.data()); });
        auto t2 = now();
        parallel([&](int n) { bm3d_frame(n, true); });
        auto t3 = now();
        parallel([&](int n) { vaggregate_frame(n, h_dst); });
        auto t4 = now();
        secs[0] = std::chrono::duration<double>(t1 - t0).count();
        secs[1] = std::chrono::duration<double>(t2 - t1).count();
        secs[2] = std::chrono::duration<double>(t3 - t2).count();
        secs[3] = std::chrono::duration<double>(t4 - t3).count();
        if (stage_seconds) std::memcpy(stage_seconds, secs, sizeof(secs));
        if (err.load()) {
            g_err = "cudaGraphLaunch / cudaStreamSynchronize failed";
            rc = 1;
        }
    }

    for (Res &r : pool) {
        for (auto &e : r.exec)
            if (e) cudaGraphExecDestroy(e);
        if (r.stream) cudaStreamDestroy(r.stream);
        cudaFreeHost(r.h_res);
        cudaFree(r.d_res);
        cudaFree(r.d_src);
    }
    return rc;
}

}  // extern "C"
