/*
 * Minimal, project-written declarations of the VapourSynth C API (v3 surface)
 * that the bm3d plugin layer and the oracle harness refer to BY NAME.
 *
 * This is NOT the VapourSynth SDK header. Only the identifiers that the
 * BM3D/VAggregate/BM3Dv2 filter code uses are declared, and the member order
 * of `VSAPI` here is this project's own. Code compiled against this file is
 * source-compatible with the real SDK (every access goes through a member
 * name), but a plugin binary meant to be loaded by a real VapourSynth core
 * must be rebuilt against the real `VapourSynth.h` (API v3) so the function
 * table layout matches. Inside this repository the header serves two jobs:
 *   1. compiling the reference CPU implementation unchanged for the oracle;
 *   2. compiling the plugin layer against an in-process fake core in tests.
 */
#ifndef BM3D_B200_VSAPI_MIN_H
#define BM3D_B200_VSAPI_MIN_H

#include <stdint.h>

#define VAPOURSYNTH_API_MAJOR 3
#define VAPOURSYNTH_API_MINOR 6
#define VAPOURSYNTH_API_VERSION ((VAPOURSYNTH_API_MAJOR << 16) | (VAPOURSYNTH_API_MINOR))

#if defined(_WIN32)
#define VS_CC __stdcall
#else
#define VS_CC
#endif

#ifdef __cplusplus
#define VS_EXTERN_C extern "C"
#else
#define VS_EXTERN_C
#endif
#define VS_EXTERNAL_API(ret) VS_EXTERN_C __attribute__((visibility("default"))) ret VS_CC

typedef struct VSFrameRef VSFrameRef;
typedef struct VSNodeRef VSNodeRef;
typedef struct VSCore VSCore;
typedef struct VSPlugin VSPlugin;
typedef struct VSNode VSNode;
typedef struct VSFuncRef VSFuncRef;
typedef struct VSMap VSMap;
typedef struct VSFrameContext VSFrameContext;

typedef enum VSColorFamily {
    cmGray = 1000000,
    cmRGB = 2000000,
    cmYUV = 3000000,
    cmYCoCg = 4000000,
    cmCompat = 9000000
} VSColorFamily;

typedef enum VSSampleType {
    stInteger = 0,
    stFloat = 1
} VSSampleType;

/* Preset ids follow the v3 numbering scheme (family + running index). */
typedef enum VSPresetFormat {
    pfNone = 0,
    pfGrayS = cmGray + 13,
    pfYUV420PS = cmYUV + 20,
    pfYUV444PS = cmYUV + 21,
    pfRGBS = cmRGB + 22
} VSPresetFormat;

typedef enum VSFilterMode {
    fmParallel = 100,
    fmParallelRequests = 200,
    fmUnordered = 300,
    fmSerial = 400
} VSFilterMode;

typedef enum VSActivationReason {
    arInitial = 0,
    arFrameReady = 1,
    arAllFramesReady = 2,
    arError = -1
} VSActivationReason;

typedef enum VSPropAppendMode {
    paReplace = 0,
    paAppend = 1,
    paTouch = 2
} VSPropAppendMode;

typedef struct VSFormat {
    char name[32];
    int id;
    int colorFamily;
    int sampleType;
    int bitsPerSample;
    int bytesPerSample;
    int subSamplingW;
    int subSamplingH;
    int numPlanes;
} VSFormat;

typedef struct VSVideoInfo {
    const VSFormat *format;
    int64_t fpsNum;
    int64_t fpsDen;
    int width;
    int height;
    int numFrames;
    int flags;
} VSVideoInfo;

typedef struct VSCoreInfo {
    const char *versionString;
    int core;
    int api;
    int numThreads;
    int64_t maxFramebufferSize;
    int64_t usedFramebufferSize;
} VSCoreInfo;

typedef struct VSAPI VSAPI;

typedef void (VS_CC *VSPublicFunction)(const VSMap *in, VSMap *out, void *userData, VSCore *core, const VSAPI *vsapi);
typedef void (VS_CC *VSRegisterFunction)(const char *name, const char *args, VSPublicFunction argsFunc, void *functionData, VSPlugin *plugin);
typedef void (VS_CC *VSConfigPlugin)(const char *identifier, const char *defaultNamespace, const char *name, int apiVersion, int readonly, VSPlugin *plugin);
typedef void (VS_CC *VSInitPlugin)(VSConfigPlugin configFunc, VSRegisterFunction registerFunc, VSPlugin *plugin);
typedef void (VS_CC *VSFilterInit)(VSMap *in, VSMap *out, void **instanceData, VSNode *node, VSCore *core, const VSAPI *vsapi);
typedef const VSFrameRef *(VS_CC *VSFilterGetFrame)(int n, int activationReason, void **instanceData, void **frameData, VSFrameContext *frameCtx, VSCore *core, const VSAPI *vsapi);
typedef void (VS_CC *VSFilterFree)(void *instanceData, VSCore *core, const VSAPI *vsapi);

/* Function table: only the members the bm3d filters call, by name. */
struct VSAPI {
    /* nodes and clips */
    VSNodeRef *(VS_CC *propGetNode)(const VSMap *map, const char *key, int index, int *error);
    const VSVideoInfo *(VS_CC *getVideoInfo)(VSNodeRef *node);
    void (VS_CC *setVideoInfo)(const VSVideoInfo *vi, int numOutputs, VSNode *node);
    void (VS_CC *freeNode)(VSNodeRef *node);
    /* argument maps */
    int (VS_CC *propNumElements)(const VSMap *map, const char *key);
    int64_t (VS_CC *propGetInt)(const VSMap *map, const char *key, int index, int *error);
    double (VS_CC *propGetFloat)(const VSMap *map, const char *key, int index, int *error);
    int (VS_CC *propSetInt)(VSMap *map, const char *key, int64_t i, int append);
    int (VS_CC *propSetIntArray)(VSMap *map, const char *key, const int64_t *i, int size);
    int (VS_CC *propSetNode)(VSMap *map, const char *key, VSNodeRef *node, int append);
    void (VS_CC *setError)(VSMap *map, const char *errorMessage);
    const char *(VS_CC *getError)(const VSMap *map);
    void (VS_CC *freeMap)(VSMap *map);
    /* filters and plugins */
    void (VS_CC *createFilter)(const VSMap *in, VSMap *out, const char *name, VSFilterInit init, VSFilterGetFrame getFrame, VSFilterFree free, int filterMode, int flags, void *instanceData, VSCore *core);
    VSPlugin *(VS_CC *getPluginById)(const char *identifier, VSCore *core);
    VSMap *(VS_CC *invoke)(VSPlugin *plugin, const char *name, const VSMap *args);
    void (VS_CC *getCoreInfo2)(VSCore *core, VSCoreInfo *info);
    void (VS_CC *setFilterError)(const char *errorMessage, VSFrameContext *frameCtx);
    /* frames */
    void (VS_CC *requestFrameFilter)(int n, VSNodeRef *node, VSFrameContext *frameCtx);
    const VSFrameRef *(VS_CC *getFrameFilter)(int n, VSNodeRef *node, VSFrameContext *frameCtx);
    void (VS_CC *freeFrame)(const VSFrameRef *f);
    VSFrameRef *(VS_CC *newVideoFrame)(const VSFormat *format, int width, int height, const VSFrameRef *propSrc, VSCore *core);
    VSFrameRef *(VS_CC *newVideoFrame2)(const VSFormat *format, int width, int height, const VSFrameRef **planeSrc, const int *planes, const VSFrameRef *propSrc, VSCore *core);
    int (VS_CC *getStride)(const VSFrameRef *f, int plane);
    const uint8_t *(VS_CC *getReadPtr)(const VSFrameRef *f, int plane);
    uint8_t *(VS_CC *getWritePtr)(VSFrameRef *f, int plane);
    int (VS_CC *getFrameWidth)(const VSFrameRef *f, int plane);
    int (VS_CC *getFrameHeight)(const VSFrameRef *f, int plane);
    VSMap *(VS_CC *getFramePropsRW)(VSFrameRef *f);
    /* string (data) arguments: the rtc plugin's bm_error_s / transform_*_s */
    const char *(VS_CC *propGetData)(const VSMap *map, const char *key, int index, int *error);
};

#endif /* BM3D_B200_VSAPI_MIN_H */
