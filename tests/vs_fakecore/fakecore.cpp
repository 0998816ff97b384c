// Test harness: an in-process stand-in for a VapourSynth core, implementing
// the VSAPI members the bm3dcuda plugin calls (vsapi_min/VapourSynth.h).
// Frames are evaluated synchronously and recursively: a filter's getFrame is
// called with arInitial, every requested frame is produced, then getFrame is
// called with arAllFramesReady. A small C API lets pytest build source clips
// from numpy data, load the plugin, invoke its functions and read frames back.
#include <dlfcn.h>

#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include <VSHelper.h>
#include <VapourSynth.h>

namespace {

thread_local std::string g_err;

struct Node;

struct Value {
    char type = 0;  // 'i' int, 'f' float, 'n' node, 's' data
    std::vector<int64_t> ints;
    std::vector<double> floats;
    std::vector<Node *> nodes;
    std::vector<std::string> data;
};

}  // namespace

struct VSMap {
    std::map<std::string, Value> kv;
    std::string error;
    bool has_error = false;
    ~VSMap();
};

struct VSFrameRef {
    const VSFormat *format = nullptr;
    int w[3] = {0, 0, 0}, h[3] = {0, 0, 0}, stride[3] = {0, 0, 0};
    std::vector<uint8_t> data[3];
    VSMap props;
    int refs = 1;
};

struct VSFrameContext {
    std::vector<std::pair<Node *, int>> requested;
    std::map<std::pair<Node *, int>, const VSFrameRef *> ready;
    std::string error;
    bool failed = false;
};

struct VSCore {
    std::map<std::string, std::pair<std::string, std::pair<VSPublicFunction, void *>>> funcs;
    std::string plugin_id, ns;
    void *dl = nullptr;
};

struct VSPlugin {
    VSCore *core = nullptr;
};

namespace {

struct Node {
    VSVideoInfo vi{};
    int refs = 1;
    // source clip
    std::vector<VSFrameRef *> frames;
    // filter
    VSFilterGetFrame get_frame = nullptr;
    VSFilterFree free_fn = nullptr;
    void *instance = nullptr;
    VSCore *core = nullptr;
};

const VSAPI *api();

void node_addref(Node *n) { ++n->refs; }
void node_release(Node *n) {
    if (!n || --n->refs > 0) return;
    if (n->free_fn) n->free_fn(n->instance, n->core, api());
    for (auto *f : n->frames) {
        if (--f->refs == 0) delete f;
    }
    delete n;
}

}  // namespace

VSMap::~VSMap() {
    for (auto &kv2 : kv)
        for (Node *n : kv2.second.nodes) node_release(n);
}

namespace {

// VSNodeRef handles are the Node pointers themselves, one reference each.
VSNodeRef *as_ref(Node *n) { return reinterpret_cast<VSNodeRef *>(n); }
Node *as_node(VSNodeRef *r) { return reinterpret_cast<Node *>(r); }
Node *as_node(VSNode *r) { return reinterpret_cast<Node *>(r); }

// formats
VSFormat make_format(const char *name, int id, int family, int st, int bits, int ssw, int ssh,
                     int np) {
    VSFormat f{};
    snprintf(f.name, sizeof(f.name), "%s", name);
    f.id = id;
    f.colorFamily = family;
    f.sampleType = st;
    f.bitsPerSample = bits;
    f.bytesPerSample = (bits + 7) / 8;
    f.subSamplingW = ssw;
    f.subSamplingH = ssh;
    f.numPlanes = np;
    return f;
}

const VSFormat g_formats[] = {
    make_format("GrayS", pfGrayS, cmGray, stFloat, 32, 0, 0, 1),
    make_format("YUV444PS", pfYUV444PS, cmYUV, stFloat, 32, 0, 0, 3),
    make_format("RGBS", pfRGBS, cmRGB, stFloat, 32, 0, 0, 3),
    make_format("YUV420PS", pfYUV420PS, cmYUV, stFloat, 32, 1, 1, 3),
    make_format("Gray8", 1000001, cmGray, stInteger, 8, 0, 0, 1),
    make_format("GrayH", 1000012, cmGray, stFloat, 16, 0, 0, 1),
};

const VSFormat *format_by_id(int id) {
    for (const auto &f : g_formats)
        if (f.id == id) return &f;
    return nullptr;
}

VSFrameRef *alloc_frame(const VSFormat *fmt, int w, int h) {
    auto *f = new VSFrameRef;
    f->format = fmt;
    for (int p = 0; p < fmt->numPlanes; ++p) {
        f->w[p] = p ? w >> fmt->subSamplingW : w;
        f->h[p] = p ? h >> fmt->subSamplingH : h;
        f->stride[p] = (f->w[p] * fmt->bytesPerSample + 63) / 64 * 64;
        f->data[p].assign((size_t)f->stride[p] * f->h[p], 0);
    }
    return f;
}

void copy_props(VSFrameRef *dst, const VSFrameRef *src) {
    if (!src) return;
    for (const auto &kv : src->props.kv) {
        dst->props.kv[kv.first] = kv.second;
        for (Node *n : kv.second.nodes) node_addref(n);
    }
}

// synchronous frame evaluation
const VSFrameRef *produce(Node *n, int i, std::string &err) {
    if (i < 0 || i >= n->vi.numFrames) {
        err = "frame index out of range";
        return nullptr;
    }
    if (!n->get_frame) {
        VSFrameRef *f = n->frames[i];
        ++f->refs;
        return f;
    }
    VSFrameContext ctx;
    void *frame_data = nullptr;
    n->get_frame(i, arInitial, &n->instance, &frame_data, &ctx, n->core, api());
    for (const auto &req : ctx.requested) {
        if (ctx.ready.count(req)) continue;
        const VSFrameRef *f = produce(req.first, req.second, err);
        if (!f) return nullptr;
        ctx.ready[req] = f;
    }
    const VSFrameRef *out =
        n->get_frame(i, arAllFramesReady, &n->instance, &frame_data, &ctx, n->core, api());
    for (auto &kv : ctx.ready) {
        VSFrameRef *f = const_cast<VSFrameRef *>(kv.second);
        if (--f->refs == 0) delete f;
    }
    if (ctx.failed || !out) {
        err = ctx.failed ? ctx.error : "filter returned no frame";
        return nullptr;
    }
    return out;
}

// ---------------------------------------------------------------------------
// VSAPI members
// ---------------------------------------------------------------------------
VSNodeRef *VS_CC propGetNode(const VSMap *m, const char *key, int index, int *error) {
    auto it = m->kv.find(key);
    if (it == m->kv.end() || it->second.type != 'n' || index >= (int)it->second.nodes.size()) {
        if (error) *error = 1;
        return nullptr;
    }
    if (error) *error = 0;
    Node *n = it->second.nodes[index];
    node_addref(n);
    return as_ref(n);
}
const VSVideoInfo *VS_CC getVideoInfo(VSNodeRef *r) { return &as_node(r)->vi; }
void VS_CC setVideoInfo(const VSVideoInfo *vi, int, VSNode *node) { as_node(node)->vi = *vi; }
void VS_CC freeNode(VSNodeRef *r) { node_release(as_node(r)); }
int VS_CC propNumElements(const VSMap *m, const char *key) {
    auto it = m->kv.find(key);
    if (it == m->kv.end()) return -1;
    const Value &v = it->second;
    return v.type == 'i' ? (int)v.ints.size() : v.type == 'f' ? (int)v.floats.size()
                                              : v.type == 's' ? (int)v.data.size()
                                                              : (int)v.nodes.size();
}
const char *VS_CC propGetData(const VSMap *m, const char *key, int index, int *error) {
    auto it = m->kv.find(key);
    if (it == m->kv.end() || it->second.type != 's' || index >= (int)it->second.data.size()) {
        if (error) *error = 1;
        return nullptr;
    }
    if (error) *error = 0;
    return it->second.data[index].c_str();
}
int64_t VS_CC propGetInt(const VSMap *m, const char *key, int index, int *error) {
    auto it = m->kv.find(key);
    if (it == m->kv.end() || it->second.type != 'i' || index >= (int)it->second.ints.size()) {
        if (error) *error = 1;
        return 0;
    }
    if (error) *error = 0;
    return it->second.ints[index];
}
double VS_CC propGetFloat(const VSMap *m, const char *key, int index, int *error) {
    auto it = m->kv.find(key);
    if (it == m->kv.end() || index >= propNumElements(m, key)) {
        if (error) *error = 1;
        return 0.0;
    }
    if (error) *error = 0;
    const Value &v = it->second;
    return v.type == 'f' ? v.floats[index] : (double)v.ints[index];
}
int VS_CC propSetInt(VSMap *m, const char *key, int64_t i, int append) {
    Value &v = m->kv[key];
    if (append != paAppend) v = Value{};
    v.type = 'i';
    v.ints.push_back(i);
    return 0;
}
int VS_CC propSetIntArray(VSMap *m, const char *key, const int64_t *i, int size) {
    Value &v = m->kv[key];
    v = Value{};
    v.type = 'i';
    v.ints.assign(i, i + size);
    return 0;
}
int VS_CC propSetNode(VSMap *m, const char *key, VSNodeRef *node, int append) {
    Value &v = m->kv[key];
    if (append != paAppend) {
        for (Node *n : v.nodes) node_release(n);
        v = Value{};
    }
    v.type = 'n';
    node_addref(as_node(node));
    v.nodes.push_back(as_node(node));
    return 0;
}
void VS_CC setError(VSMap *m, const char *msg) {
    m->has_error = true;
    m->error = msg ? msg : "";
}
const char *VS_CC getError(const VSMap *m) { return m->has_error ? m->error.c_str() : nullptr; }
void VS_CC freeMap(VSMap *m) { delete m; }

void VS_CC createFilter(const VSMap *in, VSMap *out, const char *, VSFilterInit init,
                        VSFilterGetFrame getFrame, VSFilterFree free_fn, int, int,
                        void *instanceData, VSCore *core) {
    auto *n = new Node;
    n->get_frame = getFrame;
    n->free_fn = free_fn;
    n->instance = instanceData;
    n->core = core;
    init(const_cast<VSMap *>(in), out, &n->instance, reinterpret_cast<VSNode *>(n), core, api());
    propSetNode(out, "clip", as_ref(n), paReplace);
    node_release(n);
}
VSPlugin *VS_CC getPluginById(const char *id, VSCore *core) {
    static VSPlugin plugin;
    plugin.core = core;
    return core->plugin_id == id ? &plugin : nullptr;
}
VSMap *VS_CC invoke(VSPlugin *plugin, const char *name, const VSMap *args) {
    auto *out = new VSMap;
    VSCore *core = plugin->core;
    auto it = core->funcs.find(name);
    if (it == core->funcs.end()) {
        setError(out, "function not found");
        return out;
    }
    it->second.second.first(args, out, it->second.second.second, core, api());
    return out;
}
void VS_CC getCoreInfo2(VSCore *, VSCoreInfo *info) {
    memset(info, 0, sizeof(*info));
    info->numThreads = 1;
}
void VS_CC setFilterError(const char *msg, VSFrameContext *ctx) {
    ctx->failed = true;
    ctx->error = msg ? msg : "";
}
void VS_CC requestFrameFilter(int n, VSNodeRef *node, VSFrameContext *ctx) {
    ctx->requested.emplace_back(as_node(node), n);
}
const VSFrameRef *VS_CC getFrameFilter(int n, VSNodeRef *node, VSFrameContext *ctx) {
    auto it = ctx->ready.find({as_node(node), n});
    if (it == ctx->ready.end()) return nullptr;
    const_cast<VSFrameRef *>(it->second)->refs++;
    return it->second;
}
void VS_CC freeFrame(const VSFrameRef *f) {
    if (!f) return;
    auto *m = const_cast<VSFrameRef *>(f);
    if (--m->refs == 0) delete m;
}
VSFrameRef *VS_CC newVideoFrame(const VSFormat *fmt, int w, int h, const VSFrameRef *propSrc,
                                VSCore *) {
    VSFrameRef *f = alloc_frame(fmt, w, h);
    copy_props(f, propSrc);
    return f;
}
VSFrameRef *VS_CC newVideoFrame2(const VSFormat *fmt, int w, int h, const VSFrameRef **planeSrc,
                                 const int *planes, const VSFrameRef *propSrc, VSCore *core) {
    VSFrameRef *f = newVideoFrame(fmt, w, h, propSrc, core);
    for (int p = 0; p < fmt->numPlanes; ++p)
        if (planeSrc && planeSrc[p]) {
            const VSFrameRef *s = planeSrc[p];
            vs_bitblt(f->data[p].data(), f->stride[p], s->data[planes[p]].data(),
                      s->stride[planes[p]], (size_t)f->w[p] * fmt->bytesPerSample, f->h[p]);
        }
    return f;
}
int VS_CC getStride(const VSFrameRef *f, int p) { return f->stride[p]; }
const uint8_t *VS_CC getReadPtr(const VSFrameRef *f, int p) { return f->data[p].data(); }
uint8_t *VS_CC getWritePtr(VSFrameRef *f, int p) { return f->data[p].data(); }
int VS_CC getFrameWidth(const VSFrameRef *f, int p) { return f->w[p]; }
int VS_CC getFrameHeight(const VSFrameRef *f, int p) { return f->h[p]; }
VSMap *VS_CC getFramePropsRW(VSFrameRef *f) { return &f->props; }

const VSAPI g_api = [] {
    VSAPI a{};
    a.propGetNode = propGetNode;
    a.getVideoInfo = getVideoInfo;
    a.setVideoInfo = setVideoInfo;
    a.freeNode = freeNode;
    a.propNumElements = propNumElements;
    a.propGetInt = propGetInt;
    a.propGetFloat = propGetFloat;
    a.propGetData = propGetData;
    a.propSetInt = propSetInt;
    a.propSetIntArray = propSetIntArray;
    a.propSetNode = propSetNode;
    a.setError = setError;
    a.getError = getError;
    a.freeMap = freeMap;
    a.createFilter = createFilter;
    a.getPluginById = getPluginById;
    a.invoke = invoke;
    a.getCoreInfo2 = getCoreInfo2;
    a.setFilterError = setFilterError;
    a.requestFrameFilter = requestFrameFilter;
    a.getFrameFilter = getFrameFilter;
    a.freeFrame = freeFrame;
    a.newVideoFrame = newVideoFrame;
    a.newVideoFrame2 = newVideoFrame2;
    a.getStride = getStride;
    a.getReadPtr = getReadPtr;
    a.getWritePtr = getWritePtr;
    a.getFrameWidth = getFrameWidth;
    a.getFrameHeight = getFrameHeight;
    a.getFramePropsRW = getFramePropsRW;
    return a;
}();

const VSAPI *api() { return &g_api; }

VSCore *g_loading = nullptr;

void VS_CC config_plugin(const char *id, const char *ns, const char *, int, int, VSPlugin *) {
    g_loading->plugin_id = id;
    g_loading->ns = ns;
}
void VS_CC register_function(const char *name, const char *args, VSPublicFunction fn, void *data,
                             VSPlugin *) {
    g_loading->funcs[name] = {args, {fn, data}};
}

}  // namespace

// ---------------------------------------------------------------------------
// C API for the tests
// ---------------------------------------------------------------------------
extern "C" {

const char *fc_last_error() { return g_err.c_str(); }

VSCore *fc_core_new() { return new VSCore; }

int fc_load_plugin(VSCore *core, const char *path) {
    core->dl = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!core->dl) {
        g_err = dlerror();
        return -1;
    }
    auto init = reinterpret_cast<VSInitPlugin>(dlsym(core->dl, "VapourSynthPluginInit"));
    if (!init) {
        g_err = "VapourSynthPluginInit not exported";
        return -1;
    }
    g_loading = core;
    init(config_plugin, register_function, nullptr);
    g_loading = nullptr;
    return 0;
}

const char *fc_plugin_id(VSCore *core) { return core->plugin_id.c_str(); }
const char *fc_plugin_ns(VSCore *core) { return core->ns.c_str(); }
const char *fc_function_args(VSCore *core, const char *name) {
    auto it = core->funcs.find(name);
    return it == core->funcs.end() ? nullptr : it->second.first.c_str();
}

VSMap *fc_map_new() { return new VSMap; }
void fc_map_free(VSMap *m) { delete m; }
void fc_map_set_int(VSMap *m, const char *key, long long v, int append) {
    propSetInt(m, key, v, append);
}
void fc_map_set_float(VSMap *m, const char *key, double v, int append) {
    Value &val = m->kv[key];
    if (!append) val = Value{};
    val.type = 'f';
    val.floats.push_back(v);
}
void fc_map_set_node(VSMap *m, const char *key, VSNodeRef *n) { propSetNode(m, key, n, paReplace); }
void fc_map_set_data(VSMap *m, const char *key, const char *v, int append) {
    Value &val = m->kv[key];
    if (!append) val = Value{};
    val.type = 's';
    val.data.push_back(v);
}
const char *fc_map_error(VSMap *m) { return getError(m); }
VSNodeRef *fc_map_get_node(VSMap *m, const char *key) { return propGetNode(m, key, 0, nullptr); }

VSMap *fc_invoke(VSCore *core, const char *name, VSMap *args) {
    VSPlugin plugin{core};
    return invoke(&plugin, name, args);
}

// A source clip of zeroed frames; fill planes with fc_clip_set_plane.
VSNodeRef *fc_clip_new(int format_id, int width, int height, int num_frames) {
    const VSFormat *fmt = format_by_id(format_id);
    if (!fmt) {
        g_err = "unknown format";
        return nullptr;
    }
    auto *n = new Node;
    n->vi.format = fmt;
    n->vi.width = width;
    n->vi.height = height;
    n->vi.numFrames = num_frames;
    n->vi.fpsNum = 24;
    n->vi.fpsDen = 1;
    for (int i = 0; i < num_frames; ++i) n->frames.push_back(alloc_frame(fmt, width, height));
    return as_ref(n);
}

// data: plane rows of width_p samples, contiguous.
int fc_clip_set_plane(VSNodeRef *r, int n, int plane, const void *data) {
    Node *node = as_node(r);
    VSFrameRef *f = node->frames.at(n);
    vs_bitblt(f->data[plane].data(), f->stride[plane], data,
              f->w[plane] * f->format->bytesPerSample,
              (size_t)f->w[plane] * f->format->bytesPerSample, f->h[plane]);
    return 0;
}

void fc_node_free(VSNodeRef *r) { freeNode(r); }

void fc_video_info(VSNodeRef *r, int *w, int *h, int *frames, int *format_id) {
    const VSVideoInfo *vi = getVideoInfo(r);
    *w = vi->width;
    *h = vi->height;
    *frames = vi->numFrames;
    *format_id = vi->format ? vi->format->id : 0;
}

const VSFrameRef *fc_get_frame(VSNodeRef *r, int n) {
    g_err.clear();
    return produce(as_node(r), n, g_err);
}

void fc_frame_dims(const VSFrameRef *f, int plane, int *w, int *h) {
    *w = f->w[plane];
    *h = f->h[plane];
}

// Copies a float plane into dst (rows of width_p floats, contiguous).
void fc_frame_read(const VSFrameRef *f, int plane, float *dst) {
    vs_bitblt(dst, f->w[plane] * 4, f->data[plane].data(), f->stride[plane],
              (size_t)f->w[plane] * 4, f->h[plane]);
}

long long fc_frame_prop_int(const VSFrameRef *f, const char *key, int index, int *error) {
    return propGetInt(&f->props, key, index, error);
}

void fc_frame_free(const VSFrameRef *f) { freeFrame(f); }

}  // extern "C"
