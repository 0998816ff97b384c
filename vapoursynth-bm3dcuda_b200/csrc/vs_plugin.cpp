// VapourSynth filter layer of the B200 engine: BM3D, VAggregate and BM3Dv2
// registered under the reference plugin's identifier and namespace, with the
// reference's argument strings, defaults, carry-forward rules, error messages,
// output formats and frame properties (source/source.cpp:457-1027). Compute
// goes through the engine's C ABI (include/bm3d_b200.h):
//   BM3D       one bm3d_b200_graph per (device resource, plane job), the
//              replacement of the reference's per-resource CUDA graphs;
//              radius 0 is aggregated on the device (bm3d_b200_aggregate).
//   VAggregate the temporal aggregation on the device (bm3d_b200_vaggregate).
//   BM3Dv2     BM3D followed by VAggregate when radius > 0, streamed
//              (bm3d_b200_stream): frames uploaded once, windows filtered once.
//
// Beyond the reference's arguments, BM3D / BM3Dv2 accept three optional
// ones that default to the reference's behaviour: proposer (a file written
// by bm3dcuda.learned.Proposer.save: the network parameters and embedding
// quantisation of a trained match proposer), proposer_cells (cells scored
// per spatial / temporal search, default 2, 2) and proposer_tau (exhaustive
// re-search threshold, default 4). A proposer makes the block matching of
// BM3Dv2 with radius > 0 learned; other calls reject it.
//
// Build against the VapourSynth SDK's VapourSynth.h (API v3) for a loadable
// plugin; the in-repo declarations under vsapi_min/ serve the test harness.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include <VSHelper.h>
#include <VapourSynth.h>

#include "bm3d_b200.h"

namespace {

// Built twice: as bm3dcuda (source/source.cpp) and, with BM3D_RTC_PLUGIN, as
// the run-time-compiled plugin's surface bm3dcuda_rtc (rtc_source/source.cpp),
// whose BM3D / BM3Dv2 add bm_error_s, transform_2d_s and transform_1d_s and
// whose messages start with "BM3D_RTC: ".
#ifdef BM3D_RTC_PLUGIN
constexpr const char *kPluginId = "com.wolframrhodium.bm3dcuda_rtc";
constexpr const char *kNamespace = "bm3dcuda_rtc";
constexpr const char *kPrefix = "BM3D_RTC: ";
#else
constexpr const char *kPluginId = "com.wolframrhodium.bm3dcuda";
constexpr const char *kNamespace = "bm3dcuda";
constexpr const char *kPrefix = "BM3D: ";
#endif
constexpr int kFastResources = 4;

// ---------------------------------------------------------------------------
// argument helpers (source/source.cpp:503-634)
// ---------------------------------------------------------------------------
template <typename T, typename Get, typename Ok>
bool per_plane(T (&out)[3], T def, Get get, Ok ok) {
    for (int i = 0; i < 3; ++i) {
        int err = 0;
        T v = get(i, &err);
        if (err) {
            v = i == 0 ? def : out[i - 1];
        } else if (!ok(v)) {
            return false;
        }
        out[i] = v;
    }
    return true;
}

int scalar_int(const VSAPI *vsapi, const VSMap *in, const char *key, int def) {
    int err = 0;
    const int v = int64ToIntS(vsapi->propGetInt(in, key, 0, &err));
    return err ? def : v;
}

// One device resource: staging buffers, a stream and the engine graphs.
struct Resource {
    float *d_src = nullptr;  // [(final?2:1)][planes][2r+1][H][stride]
    float *d_res = nullptr;  // [planes][2r+1][2][H][stride]
    float *d_out = nullptr;  // [H][stride] aggregated plane (radius 0)
    float *h_res = nullptr;  // pinned staging, max of both layouts
    cudaStream_t stream = nullptr;
    bm3d_b200_graph *graph[3] = {nullptr, nullptr, nullptr};

    void release() {
        for (auto &g : graph) {
            bm3d_b200_graph_destroy(g);
            g = nullptr;
        }
        if (stream) cudaStreamDestroy(stream);
        cudaFree(d_src);
        cudaFree(d_res);
        cudaFree(d_out);
        cudaFreeHost(h_res);
        stream = nullptr;
        d_src = d_res = d_out = h_res = nullptr;
    }
};

// Fixed pool of resources handed out to concurrent getFrame calls.
class ResourcePool {
public:
    void put(Resource *r) {
        std::lock_guard<std::mutex> lk(mu_);
        free_.push_back(r);
        cv_.notify_one();
    }
    Resource *take() {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !free_.empty(); });
        Resource *r = free_.back();
        free_.pop_back();
        return r;
    }

private:
    std::mutex mu_;
    std::condition_variable cv_;
    std::vector<Resource *> free_;
};

struct BM3DData {
    VSNodeRef *node = nullptr;
    VSNodeRef *ref_node = nullptr;
    const VSVideoInfo *vi = nullptr;
    int radius = 0;
    bool chroma = false;
    bool final_ = false;
    bool zero_init = true;
    bool process[3] = {false, false, false};
    int device_id = 0;
    int d_stride = 0;  // floats per row of the device buffers
    std::vector<Resource> resources;
    ResourcePool pool;

    ~BM3DData() {
        if (!resources.empty()) cudaSetDevice(device_id);
        for (auto &r : resources) r.release();
    }
};

std::string cuda_msg(const char *what, cudaError_t e) {
    return std::string("'") + what + "' failed: " + cudaGetErrorString(e);
}

#define TRY_CUDA(expr)                                                  \
    do {                                                                \
        cudaError_t e_ = (expr);                                        \
        if (e_ != cudaSuccess) return cuda_msg(#expr, e_);              \
    } while (0)

#define TRY_ENGINE(expr)                                                \
    do {                                                                \
        if ((expr) != BM3D_B200_OK) return std::string(bm3d_b200_last_error()); \
    } while (0)

int plane_width(const VSVideoInfo *vi, int p) {
    return p == 0 ? vi->width : vi->width >> vi->format->subSamplingW;
}
int plane_height(const VSVideoInfo *vi, int p) {
    return p == 0 ? vi->height : vi->height >> vi->format->subSamplingH;
}

// ---------------------------------------------------------------------------
// BM3D
// ---------------------------------------------------------------------------
void VS_CC bm3d_init(VSMap *, VSMap *, void **instanceData, VSNode *node, VSCore *,
                     const VSAPI *vsapi) {
    auto *d = static_cast<BM3DData *>(*instanceData);
    if (d->radius) {
        VSVideoInfo vi = *d->vi;
        vi.height *= 2 * (2 * d->radius + 1);  // raw stack (source/source.cpp:197-200)
        vsapi->setVideoInfo(&vi, 1, node);
    } else {
        vsapi->setVideoInfo(d->vi, 1, node);
    }
}

// Runs one plane job (chroma: all three planes) of one frame window.
// frames: (final ? 2 : 1) * (2r+1) VS frames, ref frames first.
std::string bm3d_job(BM3DData *d, Resource &res, const std::vector<const VSFrameRef *> &frames,
                     VSFrameRef *dst, int job, const VSAPI *vsapi) {
    const int tw = 2 * d->radius + 1;
    const int nin = (d->final_ ? 2 : 1);
    const int plane0 = d->chroma ? 0 : job;
    const int np = d->chroma ? 3 : 1;
    const int width = plane_width(d->vi, plane0), height = plane_height(d->vi, plane0);
    const int d_pitch = d->d_stride * (int)sizeof(float);
    // stage [(final?2:1)][planes][2r+1][H][stride] into pinned memory
    float *h = res.h_res;
    for (int half = 0; half < nin; ++half)
        for (int q = 0; q < np; ++q) {
            const int plane = plane0 + q;
            for (int z = 0; z < tw; ++z) {
                if (!d->chroma || q == 0 || d->process[q]) {
                    const VSFrameRef *f = frames[half * tw + z];
                    vs_bitblt(h, d_pitch, vsapi->getReadPtr(f, plane), vsapi->getStride(f, plane),
                              (size_t)width * sizeof(float), height);
                }
                h += (size_t)d->d_stride * height;
            }
        }
    cudaStream_t s = res.stream;
    bm3d_b200_graph *g = res.graph[job];
    if (d->radius > 0) {
        // the full graph: upload, BM3D, download of the accumulator stack
        TRY_ENGINE(bm3d_b200_graph_launch(g, s));
        TRY_CUDA(cudaStreamSynchronize(s));
        const float *src = res.h_res;
        for (int q = 0; q < np; ++q) {
            const int plane = plane0 + q;
            if (d->process[plane])
                vs_bitblt(vsapi->getWritePtr(dst, plane), vsapi->getStride(dst, plane), src,
                          d_pitch, (size_t)width * sizeof(float), (size_t)height * 2 * tw);
            src += (size_t)d->d_stride * height * 2 * tw;
        }
        return {};
    }
    const size_t rows_in = (size_t)nin * np * tw * height;
    TRY_CUDA(cudaMemcpy2DAsync(res.d_src, d_pitch, res.h_res, d_pitch, (size_t)width * sizeof(float),
                               rows_in, cudaMemcpyHostToDevice, s));
    TRY_ENGINE(bm3d_b200_graph_launch_device(g, s));
    for (int q = 0; q < np; ++q) {
        const int plane = plane0 + q;
        if (!d->process[plane]) continue;
        const float *acc = res.d_res + (size_t)q * 2 * tw * height * d->d_stride;
        TRY_ENGINE(bm3d_b200_aggregate(res.d_out, d->d_stride, acc, d->d_stride, width, height, s));
        TRY_CUDA(cudaMemcpy2DAsync(res.h_res, d_pitch, res.d_out, d_pitch,
                                   (size_t)width * sizeof(float), height, cudaMemcpyDeviceToHost,
                                   s));
        TRY_CUDA(cudaStreamSynchronize(s));
        vs_bitblt(vsapi->getWritePtr(dst, plane), vsapi->getStride(dst, plane), res.h_res, d_pitch,
                  (size_t)width * sizeof(float), height);
    }
    return {};
}

const VSFrameRef *VS_CC bm3d_get_frame(int n, int activationReason, void **instanceData, void **,
                                       VSFrameContext *frameCtx, VSCore *core,
                                       const VSAPI *vsapi) {
    auto *d = static_cast<BM3DData *>(*instanceData);
    const int nframes = d->vi->numFrames;
    if (activationReason == arInitial) {
        const int first = std::max(n - d->radius, 0), last = std::min(n + d->radius, nframes - 1);
        for (int i = first; i <= last; ++i) vsapi->requestFrameFilter(i, d->node, frameCtx);
        if (d->final_)
            for (int i = first; i <= last; ++i) vsapi->requestFrameFilter(i, d->ref_node, frameCtx);
        return nullptr;
    }
    if (activationReason != arAllFramesReady) return nullptr;

    if (cudaError_t e = cudaSetDevice(d->device_id); e != cudaSuccess) {
        vsapi->setFilterError((std::string(kPrefix) + cudaGetErrorString(e)).c_str(), frameCtx);
        return nullptr;
    }
    const int tw = 2 * d->radius + 1;
    std::vector<const VSFrameRef *> frames;  // ref frames first, then src frames
    for (VSNodeRef *nd : {d->ref_node, d->node}) {
        if (!nd) continue;
        for (int i = -d->radius; i <= d->radius; ++i)
            frames.push_back(vsapi->getFrameFilter(std::min(std::max(n + i, 0), nframes - 1), nd,
                                                   frameCtx));
    }
    const VSFrameRef *src = frames[(d->final_ ? tw : 0) + d->radius];
    VSFrameRef *dst = nullptr;
    if (d->radius) {
        dst = vsapi->newVideoFrame(d->vi->format, d->vi->width, d->vi->height * 2 * tw, src, core);
        for (int p = 0; p < d->vi->format->numPlanes; ++p)
            if (d->zero_init && !d->process[p])
                memset(vsapi->getWritePtr(dst, p), 0,
                       (size_t)vsapi->getFrameHeight(dst, p) * vsapi->getStride(dst, p));
    } else {
        const VSFrameRef *fr[] = {d->process[0] ? nullptr : src, d->process[1] ? nullptr : src,
                                  d->process[2] ? nullptr : src};
        const int pl[] = {0, 1, 2};
        dst = vsapi->newVideoFrame2(d->vi->format, d->vi->width, d->vi->height, fr, pl, src, core);
    }

    Resource *res = d->pool.take();
    std::string err;
    const int njobs = d->chroma ? 1 : d->vi->format->numPlanes;
    for (int job = 0; job < njobs && err.empty(); ++job) {
        if (!d->chroma && !d->process[job]) continue;
        err = bm3d_job(d, *res, frames, dst, job, vsapi);
    }
    d->pool.put(res);
    for (auto *f : frames) vsapi->freeFrame(f);
    if (!err.empty()) {
        vsapi->freeFrame(dst);
        vsapi->setFilterError((kPrefix + err).c_str(), frameCtx);
        return nullptr;
    }
    if (d->radius) {
        VSMap *props = vsapi->getFramePropsRW(dst);
        vsapi->propSetInt(props, "BM3D_V_radius", d->radius, paReplace);
        const int64_t process[3] = {d->process[0], d->process[1], d->process[2]};
        vsapi->propSetIntArray(props, "BM3D_V_process", process, 3);
    }
    return dst;
}

void VS_CC bm3d_free(void *instanceData, VSCore *, const VSAPI *vsapi) {
    auto *d = static_cast<BM3DData *>(instanceData);
    vsapi->freeNode(d->node);
    vsapi->freeNode(d->ref_node);
    delete d;
}

// Parsed arguments of BM3D / BM3Dv2 (source/source.cpp:457-634), with the
// rtc plugin's variant strings in its build (rtc_source/source.cpp:854-911).
struct BM3DArgs {
    VSNodeRef *node = nullptr, *ref_node = nullptr;
    const VSVideoInfo *vi = nullptr;
    bool final_ = false;
    float sigma[3] = {3.0f, 3.0f, 3.0f};  // user-level values
    bool process[3] = {true, true, true};
    int block_step[3] = {8, 8, 8}, bm_range[3] = {9, 9, 9}, ps_num[3] = {2, 2, 2},
        ps_range[3] = {4, 4, 4};
    int radius = 0;
    bool chroma = false;
    int device_id = 0;
    bool fast = true;
    int extractor_exp = 0;
    bool zero_init = true;
    int bm_error[3] = {0, 0, 0}, tx2[3] = {0, 0, 0}, tx1[3] = {0, 0, 0};
    // learned match proposal (optional, no counterpart in the reference)
    std::string proposer;
    int proposer_cells[2] = {2, 2};
    float proposer_tau = 4.0f;
};

// Validates in the reference's order; returns "" or the message without the
// plugin prefix. a.node / a.ref_node hold references either way.
std::string parse_bm3d_args(const VSMap *in, const VSAPI *vsapi, BM3DArgs &a) {
    a.node = vsapi->propGetNode(in, "clip", 0, nullptr);
    a.vi = vsapi->getVideoInfo(a.node);
    const VSFormat *fmt = a.vi->format;
    if (!isConstantFormat(a.vi) || fmt->sampleType == stInteger ||
        (fmt->sampleType == stFloat && fmt->bitsPerSample != 32))
        return "only constant format 32bit float input supported";
    int err = 0;
    a.ref_node = vsapi->propGetNode(in, "ref", 0, &err);
    if (err) {
        a.ref_node = nullptr;
    } else {
        const VSVideoInfo *rvi = vsapi->getVideoInfo(a.ref_node);
        if (rvi->format->id != fmt->id) return "\"ref\" must be of the same format as \"clip\"";
        if (rvi->width != a.vi->width || rvi->height != a.vi->height)
            return "\"ref\" must be of the same dimensions as \"clip\"";
        if (rvi->numFrames != a.vi->numFrames)
            return "\"ref\" must be of the same number of frames as \"clip\"";
    }
    a.final_ = a.ref_node != nullptr;
    if (!per_plane(a.sigma, 3.0f,
                   [&](int i, int *e) { return (float)vsapi->propGetFloat(in, "sigma", i, e); },
                   [](float v) { return v >= 0.0f; }))
        return "\"sigma\" must be non-negative";
    for (int i = 0; i < 3; ++i)
        a.process[i] = !(a.sigma[i] < std::numeric_limits<float>::epsilon());
    auto get_int = [&](const char *key) {
        return [=](int i, int *e) { return int64ToIntS(vsapi->propGetInt(in, key, i, e)); };
    };
    if (!per_plane(a.block_step, 8, get_int("block_step"), [](int v) { return v > 0 && v <= 8; }))
        return "\"block_step\" must be in range [1, 8]";
    if (!per_plane(a.bm_range, 9, get_int("bm_range"), [](int v) { return v > 0; }))
        return "\"bm_range\" must be positive";
    a.radius = scalar_int(vsapi, in, "radius", 0);
    if (a.radius < 0) return "\"radius\" must be non-negative";
    if (!per_plane(a.ps_num, 2, get_int("ps_num"), [](int v) { return v > 0 && v <= 8; }))
        return "\"ps_num\" must be in range [1, 8]";
    if (!per_plane(a.ps_range, 4, get_int("ps_range"), [](int v) { return v > 0; }))
        return "\"ps_range\" must be positive";
    a.chroma = scalar_int(vsapi, in, "chroma", 0) != 0;
    if (a.chroma && fmt->id != pfYUV444PS)
        return "clip format must be YUV444 when \"chroma\" is true";
    a.device_id = scalar_int(vsapi, in, "device_id", 0);
    int count = 0;
    if (cudaError_t e = cudaGetDeviceCount(&count); e != cudaSuccess)
        return cuda_msg("cudaGetDeviceCount(&device_count)", e);
    if (a.device_id < 0 || a.device_id >= count)
        return "invalid device ID (" + std::to_string(a.device_id) + ")";
    if (cudaError_t e = cudaSetDevice(a.device_id); e != cudaSuccess)
        return cuda_msg("cudaSetDevice(device_id)", e);
    a.fast = scalar_int(vsapi, in, "fast", 1) != 0;
    a.extractor_exp = scalar_int(vsapi, in, "extractor_exp", 0);
#ifdef BM3D_RTC_PLUGIN
    {
        auto parse = [&](const char *key, int (&dst)[3], const char *const *names, int n,
                         std::string *bad) {
            for (int i = 0; i < 3; ++i) {
                int e = 0;
                const char *v = vsapi->propGetData(in, key, i, &e);
                if (e) {
                    dst[i] = i == 0 ? 0 : dst[i - 1];
                    continue;
                }
                std::string t(v ? v : "");
                for (char &c : t) c = (char)std::tolower((unsigned char)c);
                int k = -1;
                for (int j = 0; j < n; ++j)
                    if (t == names[j]) k = j;
                if (k < 0) {
                    *bad = t;
                    return false;
                }
                dst[i] = k;
            }
            return true;
        };
        static const char *const bm_names[] = {"ssd", "sad", "zssd", "zsad", "ssd/norm"};
        static const char *const tx_names[] = {"dct", "haar", "wht", "bior1.5"};
        std::string bad;
        if (!parse("bm_error_s", a.bm_error, bm_names, 5, &bad))
            return "invalid 'bm_error_s': " + bad;
        if (!parse("transform_2d_s", a.tx2, tx_names, 4, &bad))
            return "invalid 'transform_2d_s': " + bad;
        if (!parse("transform_1d_s", a.tx1, tx_names, 4, &bad))
            return "invalid 'transform_1d_s': " + bad;
    }
#endif
    a.zero_init = scalar_int(vsapi, in, "zero_init", 1) != 0;
    {
        int e = 0;
        const char *path = vsapi->propGetData(in, "proposer", 0, &e);
        if (!e && path) a.proposer = path;
        for (int i = 0; i < 2; ++i) {
            const int v = int64ToIntS(vsapi->propGetInt(in, "proposer_cells", i, &e));
            a.proposer_cells[i] = e ? (i == 0 ? 2 : a.proposer_cells[0]) : v;
            if (!e && (v < 1 || v > 8)) return "\"proposer_cells\" must be in range [1, 8]";
        }
        const double tau = vsapi->propGetFloat(in, "proposer_tau", 0, &e);
        if (!e) {
            if (!(tau >= 0.0)) return "\"proposer_tau\" must be non-negative";
            a.proposer_tau = (float)tau;
        }
    }
    return {};
}

// A trained proposer from the file `path` (float32 little-endian: the
// network's BM3D_B200_PROPOSER_PARAMS parameters, then the 17 quantisation
// values), on the current device; "" or an error message.
std::string load_proposer(const std::string &path, int device_id, bm3d_b200_proposer **out) {
    *out = nullptr;
    const int np = bm3d_b200_proposer_num_params();
    std::vector<float> buf((size_t)np + 17);
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return "cannot open \"proposer\" file " + path;
    const size_t got = std::fread(buf.data(), sizeof(float), buf.size(), f);
    const bool extra = std::fgetc(f) != EOF;
    std::fclose(f);
    if (got != buf.size() || extra)
        return "\"proposer\" file " + path + " is not a saved proposer (" +
               std::to_string(buf.size() * sizeof(float)) + " bytes expected)";
    bm3d_b200_proposer *p = nullptr;
    if (bm3d_b200_proposer_create(&p, buf.data(), device_id) != BM3D_B200_OK ||
        bm3d_b200_proposer_set_quant(p, buf.data() + np) != BM3D_B200_OK) {
        std::string m = bm3d_b200_last_error();
        bm3d_b200_proposer_destroy(p);
        if (m.rfind("BM3D: ", 0) == 0) m = m.substr(6);
        return m;
    }
    *out = p;
    return {};
}

void VS_CC bm3d_create(const VSMap *in, VSMap *out, void *, VSCore *core, const VSAPI *vsapi) {
    auto d = std::make_unique<BM3DData>();
    auto fail = [&](const std::string &msg) {
        vsapi->setError(out, (kPrefix + msg).c_str());
        vsapi->freeNode(d->node);
        vsapi->freeNode(d->ref_node);
        d->node = d->ref_node = nullptr;
    };
    BM3DArgs a;
    const std::string perr = parse_bm3d_args(in, vsapi, a);
    d->node = a.node;
    d->ref_node = a.ref_node;
    if (!perr.empty()) return fail(perr);
    if (!a.proposer.empty()) return fail("\"proposer\" applies to BM3Dv2 with radius > 0");
    d->vi = a.vi;
    const VSFormat *fmt = d->vi->format;
    d->final_ = a.final_;
    for (int i = 0; i < 3; ++i) d->process[i] = a.process[i];
    float sigma[3];
    for (int i = 0; i < 3; ++i) sigma[i] = bm3d_b200_scale_sigma(a.sigma[i], d->final_);
    int block_step[3], bm_range[3], ps_num[3], ps_range[3];
    int bm_error[3], tx2[3], tx1[3];
    for (int i = 0; i < 3; ++i) {
        block_step[i] = a.block_step[i];
        bm_range[i] = a.bm_range[i];
        ps_num[i] = a.ps_num[i];
        ps_range[i] = a.ps_range[i];
        bm_error[i] = a.bm_error[i];
        tx2[i] = a.tx2[i];
        tx1[i] = a.tx1[i];
    }
    d->radius = a.radius;
    d->chroma = a.chroma;
    d->device_id = a.device_id;
    const bool fast = a.fast;
    const float extractor = a.extractor_exp ? std::ldexp(1.0f, a.extractor_exp) : 0.0f;
    d->zero_init = a.zero_init;

    // device resources (source/source.cpp:636-713)
    const int tw = 2 * d->radius + 1;
    const int np = d->chroma ? 3 : 1;
    const int max_w = d->process[0] ? d->vi->width : d->vi->width >> fmt->subSamplingW;
    const int max_h = d->process[0] ? d->vi->height : d->vi->height >> fmt->subSamplingH;
    d->d_stride = (std::max(max_w, d->vi->width) + 31) / 32 * 32;
    const size_t plane = (size_t)d->d_stride * std::max(max_h, d->vi->height);
    const size_t src_floats = (size_t)(d->final_ ? 2 : 1) * np * tw * plane;
    const size_t res_floats = (size_t)np * tw * 2 * plane;
    d->resources.resize(fast ? kFastResources : 1);
    for (auto &r : d->resources) {
        cudaError_t e = cudaMalloc(&r.d_src, src_floats * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&r.d_res, res_floats * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&r.d_out, plane * sizeof(float));
        if (e == cudaSuccess) e = cudaMallocHost(&r.h_res, std::max(src_floats, res_floats) * sizeof(float));
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&r.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(cuda_msg("device resource allocation", e));
        for (int p = 0; p < fmt->numPlanes; ++p) {
            const int job = d->chroma ? 0 : p;
            if (d->chroma ? p != 0 : !d->process[p]) continue;
            const int pw = d->chroma ? d->vi->width : plane_width(d->vi, p);
            const int ph = d->chroma ? d->vi->height : plane_height(d->vi, p);
            const int q = d->chroma ? 0 : p;
            if (bm3d_b200_graph_create_rtc(&r.graph[job], r.d_res, r.d_src, r.h_res, pw, ph,
                                           d->d_stride, sigma[q], block_step[q], bm_range[q],
                                           d->radius, ps_num[q], ps_range[q], d->chroma, sigma[1],
                                           sigma[2], d->final_, extractor, bm_error[q], tx2[q],
                                           tx1[q]) != BM3D_B200_OK) {
                std::string m = bm3d_b200_last_error();
                if (m.rfind("BM3D: ", 0) == 0) m = m.substr(6);
                return fail(m);
            }
        }
        d->pool.put(&r);
    }
    vsapi->createFilter(in, out, "BM3D", bm3d_init, bm3d_get_frame, bm3d_free, fmParallel, 0,
                        d.release(), core);
}

// ---------------------------------------------------------------------------
// VAggregate (source/source.cpp:722-909), on the device
// ---------------------------------------------------------------------------
struct VAggBuffers {
    float *d_raw = nullptr;  // (2r+1) raw frames of one plane; only the read slabs are filled
    float *d_out = nullptr;
    float *h_out = nullptr;
    cudaStream_t stream = nullptr;
};

struct VAggData {
    VSNodeRef *node = nullptr;
    VSNodeRef *src_node = nullptr;
    const VSVideoInfo *src_vi = nullptr;
    bool process[3] = {false, false, false};
    int radius = 0;
    int device_id = 0;
    int d_stride = 0;
    std::vector<VAggBuffers> buffers;
    std::mutex mu;
    std::condition_variable cv;
    std::vector<VAggBuffers *> idle;

    ~VAggData() {
        if (!buffers.empty()) cudaSetDevice(device_id);
        for (auto &b : buffers) {
            if (b.stream) cudaStreamDestroy(b.stream);
            cudaFree(b.d_raw);
            cudaFree(b.d_out);
            cudaFreeHost(b.h_out);
        }
    }
};

void VS_CC vagg_init(VSMap *, VSMap *, void **instanceData, VSNode *node, VSCore *,
                     const VSAPI *vsapi) {
    auto *d = static_cast<VAggData *>(*instanceData);
    vsapi->setVideoInfo(d->src_vi, 1, node);
}

std::string vagg_plane(VAggData *d, VAggBuffers &b, const std::vector<const VSFrameRef *> &raw,
                       VSFrameRef *dst, int plane, int n, const VSAPI *vsapi) {
    const int r = d->radius, tw = 2 * r + 1, N = d->src_vi->numFrames;
    const int w = plane_width(d->src_vi, plane), h = plane_height(d->src_vi, plane);
    const size_t pitch = (size_t)d->d_stride * sizeof(float);
    const size_t raw_frame = (size_t)tw * 2 * h * d->d_stride;
    const float *vframes[2 * BM3D_B200_MAX_RADIUS + 1];
    for (int i = 0; i < tw; ++i) {
        // upload only the wdst/weight slab pair that VAggregate reads
        const int s = std::min(std::max(2 * r - i, n - N + 1 + r), n + r);
        float *base = b.d_raw + (size_t)i * raw_frame;
        const uint8_t *sp = vsapi->getReadPtr(raw[i], plane) +
                            (size_t)s * 2 * h * vsapi->getStride(raw[i], plane);
        TRY_CUDA(cudaMemcpy2DAsync(base + (size_t)s * 2 * h * d->d_stride, pitch, sp,
                                   vsapi->getStride(raw[i], plane), (size_t)w * sizeof(float),
                                   (size_t)2 * h, cudaMemcpyHostToDevice, b.stream));
        vframes[i] = base;
    }
    TRY_ENGINE(bm3d_b200_vaggregate(b.d_out, d->d_stride, vframes, d->d_stride, w, h, r, n, N,
                                    b.stream));
    TRY_CUDA(cudaMemcpy2DAsync(b.h_out, pitch, b.d_out, pitch, (size_t)w * sizeof(float), h,
                               cudaMemcpyDeviceToHost, b.stream));
    TRY_CUDA(cudaStreamSynchronize(b.stream));
    vs_bitblt(vsapi->getWritePtr(dst, plane), vsapi->getStride(dst, plane), b.h_out, (int)pitch,
              (size_t)w * sizeof(float), h);
    return {};
}

const VSFrameRef *VS_CC vagg_get_frame(int n, int activationReason, void **instanceData, void **,
                                       VSFrameContext *frameCtx, VSCore *core,
                                       const VSAPI *vsapi) {
    auto *d = static_cast<VAggData *>(*instanceData);
    const int N = d->src_vi->numFrames;
    if (activationReason == arInitial) {
        for (int i = std::max(n - d->radius, 0); i <= std::min(n + d->radius, N - 1); ++i)
            vsapi->requestFrameFilter(i, d->node, frameCtx);
        vsapi->requestFrameFilter(n, d->src_node, frameCtx);
        return nullptr;
    }
    if (activationReason != arAllFramesReady) return nullptr;
    if (cudaError_t e = cudaSetDevice(d->device_id); e != cudaSuccess) {
        vsapi->setFilterError((std::string("VAggregate: ") + cudaGetErrorString(e)).c_str(),
                              frameCtx);
        return nullptr;
    }
    const VSFrameRef *src = vsapi->getFrameFilter(n, d->src_node, frameCtx);
    std::vector<const VSFrameRef *> raw;
    for (int i = n - d->radius; i <= n + d->radius; ++i)
        raw.push_back(vsapi->getFrameFilter(std::min(std::max(i, 0), N - 1), d->node, frameCtx));
    const VSFrameRef *fr[] = {d->process[0] ? nullptr : src, d->process[1] ? nullptr : src,
                              d->process[2] ? nullptr : src};
    const int pl[] = {0, 1, 2};
    VSFrameRef *dst = vsapi->newVideoFrame2(d->src_vi->format, d->src_vi->width,
                                            d->src_vi->height, fr, pl, src, core);
    VAggBuffers *b;
    {
        std::unique_lock<std::mutex> lk(d->mu);
        d->cv.wait(lk, [&] { return !d->idle.empty(); });
        b = d->idle.back();
        d->idle.pop_back();
    }
    std::string err;
    for (int p = 0; p < d->src_vi->format->numPlanes && err.empty(); ++p)
        if (d->process[p]) err = vagg_plane(d, *b, raw, dst, p, n, vsapi);
    {
        std::lock_guard<std::mutex> lk(d->mu);
        d->idle.push_back(b);
        d->cv.notify_one();
    }
    for (auto *f : raw) vsapi->freeFrame(f);
    vsapi->freeFrame(src);
    if (!err.empty()) {
        vsapi->freeFrame(dst);
        vsapi->setFilterError(("VAggregate: " + err).c_str(), frameCtx);
        return nullptr;
    }
    return dst;
}

void VS_CC vagg_free(void *instanceData, VSCore *, const VSAPI *vsapi) {
    auto *d = static_cast<VAggData *>(instanceData);
    vsapi->freeNode(d->src_node);
    vsapi->freeNode(d->node);
    delete d;
}

void VS_CC vagg_create(const VSMap *in, VSMap *out, void *, VSCore *core, const VSAPI *vsapi) {
    auto d = std::make_unique<VAggData>();
    d->node = vsapi->propGetNode(in, "clip", 0, nullptr);
    const VSVideoInfo *vi = vsapi->getVideoInfo(d->node);
    d->src_node = vsapi->propGetNode(in, "src", 0, nullptr);
    d->src_vi = vsapi->getVideoInfo(d->src_node);
    d->radius = (vi->height / d->src_vi->height - 2) / 4;  // source/source.cpp:892
    const int nplanes = vsapi->propNumElements(in, "planes");
    for (int i = 0; i < nplanes; ++i) {
        const int p = int64ToIntS(vsapi->propGetInt(in, "planes", i, nullptr));
        if (p >= 0 && p < 3) d->process[p] = true;
    }
    auto fail = [&](const std::string &msg) {
        vsapi->setError(out, ("VAggregate: " + msg).c_str());
        vsapi->freeNode(d->node);
        vsapi->freeNode(d->src_node);
        d->node = d->src_node = nullptr;
    };
    if (d->radius < 0 || d->radius > BM3D_B200_MAX_RADIUS)
        return fail("clip is not a V-BM3D output of src");
    cudaGetDevice(&d->device_id);
    const int tw = 2 * d->radius + 1;
    d->d_stride = (d->src_vi->width + 31) / 32 * 32;
    const size_t plane = (size_t)d->d_stride * d->src_vi->height;
    d->buffers.resize(kFastResources);
    for (auto &b : d->buffers) {
        cudaError_t e = cudaMalloc(&b.d_raw, (size_t)tw * tw * 2 * plane * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&b.d_out, plane * sizeof(float));
        if (e == cudaSuccess) e = cudaMallocHost(&b.h_out, plane * sizeof(float));
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) return fail(cuda_msg("device buffer allocation", e));
        d->idle.push_back(&b);
    }
    vsapi->createFilter(in, out, "VAggregate", vagg_init, vagg_get_frame, vagg_free, fmParallel, 0,
                        d.release(), core);
}

// ---------------------------------------------------------------------------
// BM3Dv2 (source/source.cpp:911-989)
// ---------------------------------------------------------------------------
// ---------------------------------------------------------------------------
// BM3Dv2 with radius > 0, streamed (bm3d_b200_stream): frames uploaded once,
// windows filtered once, VAggregate on the device, one frame back per call.
// Same output as BM3D followed by VAggregate (source/source.cpp:911-989).
// ---------------------------------------------------------------------------
struct StreamData {
    VSNodeRef *node = nullptr, *ref_node = nullptr;
    const VSVideoInfo *vi = nullptr;
    int radius = 0;
    bool process[3] = {false, false, false};
    int device_id = 0;
    bm3d_b200_stream *stream = nullptr;
    bm3d_b200_proposer *proposer = nullptr;

    ~StreamData() {
        cudaSetDevice(device_id);
        if (stream) bm3d_b200_stream_destroy(stream);
        if (proposer) bm3d_b200_proposer_destroy(proposer);
    }
};

void VS_CC stream_init(VSMap *, VSMap *, void **instanceData, VSNode *node, VSCore *,
                       const VSAPI *vsapi) {
    vsapi->setVideoInfo(static_cast<StreamData *>(*instanceData)->vi, 1, node);
}

const VSFrameRef *VS_CC stream_get_frame(int n, int activationReason, void **instanceData,
                                         void **, VSFrameContext *frameCtx, VSCore *core,
                                         const VSAPI *vsapi) {
    auto *d = static_cast<StreamData *>(*instanceData);
    const int nframes = d->vi->numFrames, r = d->radius;
    if (activationReason == arInitial) {
        // the windows n-r .. n+r read frames n-2r .. n+2r
        const int first = std::max(n - 2 * r, 0), last = std::min(n + 2 * r, nframes - 1);
        for (int i = first; i <= last; ++i) vsapi->requestFrameFilter(i, d->node, frameCtx);
        if (d->ref_node)
            for (int i = first; i <= last; ++i) vsapi->requestFrameFilter(i, d->ref_node, frameCtx);
        return nullptr;
    }
    if (activationReason != arAllFramesReady) return nullptr;
    if (cudaError_t e = cudaSetDevice(d->device_id); e != cudaSuccess) {
        vsapi->setFilterError((std::string(kPrefix) + cudaGetErrorString(e)).c_str(), frameCtx);
        return nullptr;
    }
    const int nw = 4 * r + 1;
    const int np = d->vi->format->numPlanes;
    std::vector<const VSFrameRef *> src(nw), ref(d->ref_node ? nw : 0);
    std::vector<const float *> hs((size_t)nw * 3, nullptr), hr(d->ref_node ? (size_t)nw * 3 : 0);
    std::vector<int> strides((size_t)nw * 3, 0);
    for (int i = 0; i < nw; ++i) {
        const int f = std::min(std::max(n - 2 * r + i, 0), nframes - 1);
        src[i] = vsapi->getFrameFilter(f, d->node, frameCtx);
        if (d->ref_node) ref[i] = vsapi->getFrameFilter(f, d->ref_node, frameCtx);
        for (int p = 0; p < np; ++p) {
            hs[(size_t)i * 3 + p] = reinterpret_cast<const float *>(vsapi->getReadPtr(src[i], p));
            strides[(size_t)i * 3 + p] = vsapi->getStride(src[i], p);
            if (d->ref_node)
                hr[(size_t)i * 3 + p] =
                    reinterpret_cast<const float *>(vsapi->getReadPtr(ref[i], p));
        }
    }
    const VSFrameRef *center = src[2 * r];
    const VSFrameRef *fr[] = {d->process[0] ? nullptr : center, d->process[1] ? nullptr : center,
                              d->process[2] ? nullptr : center};
    const int pl[] = {0, 1, 2};
    VSFrameRef *dst =
        vsapi->newVideoFrame2(d->vi->format, d->vi->width, d->vi->height, fr, pl, center, core);
    float *hd[3] = {nullptr, nullptr, nullptr};
    int ds[3] = {0, 0, 0};
    for (int p = 0; p < np; ++p) {
        if (!d->process[p]) continue;
        hd[p] = reinterpret_cast<float *>(vsapi->getWritePtr(dst, p));
        ds[p] = vsapi->getStride(dst, p);
    }
    const int rc = bm3d_b200_stream_frame(d->stream, n, hs.data(),
                                          d->ref_node ? hr.data() : nullptr, strides.data(), hd,
                                          ds);
    for (auto *f : src) vsapi->freeFrame(f);
    for (auto *f : ref) vsapi->freeFrame(f);
    if (rc != BM3D_B200_OK) {
        std::string m = bm3d_b200_last_error();
        if (m.rfind("BM3D: ", 0) == 0) m = m.substr(6);
        vsapi->setFilterError((kPrefix + m).c_str(), frameCtx);
        vsapi->freeFrame(dst);
        return nullptr;
    }
    return dst;
}

void VS_CC stream_free(void *instanceData, VSCore *, const VSAPI *vsapi) {
    auto *d = static_cast<StreamData *>(instanceData);
    vsapi->freeNode(d->node);
    vsapi->freeNode(d->ref_node);
    delete d;
}

// BM3Dv2 radius > 0: parses like BM3D, then builds the streamed filter.
void stream_create(const VSMap *in, VSMap *out, VSCore *core, const VSAPI *vsapi) {
    BM3DArgs a;
    const std::string perr = parse_bm3d_args(in, vsapi, a);
    auto d = std::make_unique<StreamData>();
    d->node = a.node;
    d->ref_node = a.ref_node;
    auto fail = [&](const std::string &msg) {
        vsapi->setError(out, (kPrefix + msg).c_str());
        vsapi->freeNode(d->node);
        vsapi->freeNode(d->ref_node);
        d->node = d->ref_node = nullptr;
    };
    if (!perr.empty()) return fail(perr);
    d->vi = a.vi;
    d->radius = a.radius;
    d->device_id = a.device_id;
    const VSFormat *fmt = a.vi->format;
    for (int i = 0; i < 3; ++i) d->process[i] = i < fmt->numPlanes && a.process[i];
    bm3d_b200_params p;
    bm3d_b200_params_default(&p);
    for (int i = 0; i < 3; ++i) {
        p.sigma[i] = a.sigma[i];
        p.block_step[i] = a.block_step[i];
        p.bm_range[i] = a.bm_range[i];
        p.ps_num[i] = a.ps_num[i];
        p.ps_range[i] = a.ps_range[i];
    }
    p.radius = a.radius;
    p.chroma = a.chroma;
    p.extractor_exp = a.extractor_exp;
    p.zero_init = a.zero_init;
    if (bm3d_b200_stream_create(&d->stream, a.vi->width, a.vi->height, fmt->numPlanes,
                                fmt->subSamplingW, fmt->subSamplingH, a.vi->numFrames, &p,
                                a.final_, a.device_id) != BM3D_B200_OK ||
        bm3d_b200_stream_set_variant(d->stream, a.bm_error, a.tx2, a.tx1) != BM3D_B200_OK ||
        bm3d_b200_stream_set_concurrency(d->stream, a.fast ? kFastResources : 1) !=
            BM3D_B200_OK) {
        std::string m = bm3d_b200_last_error();
        if (m.rfind("BM3D: ", 0) == 0) m = m.substr(6);
        return fail(m);
    }
    if (!a.proposer.empty()) {
        const std::string perr2 = load_proposer(a.proposer, a.device_id, &d->proposer);
        if (!perr2.empty()) return fail(perr2);
        if (bm3d_b200_stream_set_proposer(d->stream, d->proposer, a.proposer_cells[0],
                                          a.proposer_cells[1], a.proposer_tau) != BM3D_B200_OK) {
            std::string m = bm3d_b200_last_error();
            if (m.rfind("BM3D: ", 0) == 0) m = m.substr(6);
            return fail(m);
        }
    }
    vsapi->createFilter(in, out, "BM3Dv2", stream_init, stream_get_frame, stream_free,
                        fmParallel, 0, d.release(), core);
}

void VS_CC bm3dv2_create(const VSMap *in, VSMap *out, void *, VSCore *core, const VSAPI *vsapi) {
    bool process[3] = {true, true, true};
    const int nsigma = vsapi->propNumElements(in, "sigma");
    for (int i = 0; i < std::min(3, nsigma); ++i)
        if (vsapi->propGetFloat(in, "sigma", i, nullptr) < std::numeric_limits<float>::epsilon())
            process[i] = false;
    if (nsigma > 0)
        for (int i = nsigma; i < 3; ++i) process[i] = process[i - 1];
    VSNodeRef *src = vsapi->propGetNode(in, "clip", 0, nullptr);
    const VSVideoInfo *vi = vsapi->getVideoInfo(src);
    bool skip = true;
    for (int i = 0; i < vi->format->numPlanes; ++i) skip = skip && !process[i];
    if (skip) {
        vsapi->propSetNode(out, "clip", src, paReplace);
        vsapi->freeNode(src);
        return;
    }
    {
        int err = 0;
        const int r = int64ToIntS(vsapi->propGetInt(in, "radius", 0, &err));
        if (!err && r > 0) {
            vsapi->freeNode(src);
            return stream_create(in, out, core, vsapi);
        }
    }
    VSPlugin *plugin = vsapi->getPluginById(kPluginId, core);
    VSMap *map = vsapi->invoke(plugin, "BM3D", in);
    if (const char *e = vsapi->getError(map)) {
        vsapi->setError(out, e);
        vsapi->freeMap(map);
        vsapi->freeNode(src);
        return;
    }
    int err = 0;
    int radius = int64ToIntS(vsapi->propGetInt(in, "radius", 0, &err));
    if (err) radius = 0;
    if (radius == 0) {
        VSNodeRef *node = vsapi->propGetNode(map, "clip", 0, nullptr);
        vsapi->freeMap(map);
        vsapi->propSetNode(out, "clip", node, paReplace);
        vsapi->freeNode(node);
        vsapi->freeNode(src);
        return;
    }
    vsapi->propSetNode(map, "src", src, paReplace);
    vsapi->freeNode(src);
    for (int i = 0; i < 3; ++i)
        if (process[i]) vsapi->propSetInt(map, "planes", i, paAppend);
    VSMap *map2 = vsapi->invoke(plugin, "VAggregate", map);
    vsapi->freeMap(map);
    if (const char *e = vsapi->getError(map2)) {
        vsapi->setError(out, e);
        vsapi->freeMap(map2);
        return;
    }
    VSNodeRef *node = vsapi->propGetNode(map2, "clip", 0, nullptr);
    vsapi->freeMap(map2);
    vsapi->propSetNode(out, "clip", node, paReplace);
    vsapi->freeNode(node);
}

}  // namespace

VS_EXTERNAL_API(void) VapourSynthPluginInit(VSConfigPlugin configFunc,
                                            VSRegisterFunction registerFunc, VSPlugin *plugin) {
    configFunc(kPluginId, kNamespace, "BM3D algorithm implemented in CUDA (B200 engine)",
               VAPOURSYNTH_API_VERSION, 1, plugin);
    // argument strings of source/source.cpp:1001-1026
    const char *bm3d_args =
        "clip:clip;"
        "ref:clip:opt;"
        "sigma:float[]:opt;"
        "block_step:int[]:opt;"
        "bm_range:int[]:opt;"
        "radius:int:opt;"
        "ps_num:int[]:opt;"
        "ps_range:int[]:opt;"
        "chroma:int:opt;"
        "device_id:int:opt;"
        "fast:int:opt;"
        "extractor_exp:int:opt;"
#ifdef BM3D_RTC_PLUGIN
        "bm_error_s:data[]:opt;"
        "transform_2d_s:data[]:opt;"
        "transform_1d_s:data[]:opt;"
#endif
        "zero_init:int:opt;"
        // optional learned match proposal (no counterpart in the reference)
        "proposer:data:opt;"
        "proposer_cells:int[]:opt;"
        "proposer_tau:float:opt;";
    registerFunc("BM3D", bm3d_args, bm3d_create, nullptr, plugin);
    registerFunc("VAggregate", "clip:clip;src:clip;planes:int[];", vagg_create, nullptr, plugin);
    registerFunc("BM3Dv2", bm3d_args, bm3dv2_create, nullptr, plugin);
}
