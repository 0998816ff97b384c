/*
 * bm3d_b200 — C ABI of the B200 (sm_100a) BM3D / V-BM3D engine.
 *
 * Plain C: pointers, ints and floats only. Streams are passed as `void *`
 * holding a cudaStream_t (NULL = the legacy default stream). Every function
 * returns BM3D_B200_OK (0) or an error code; bm3d_b200_last_error() returns
 * the message of the calling thread's last failure.
 *
 * Three groups of entry points:
 *
 *  1. The device pipeline behind the reference plugin's graph executable.
 *     The reference's VapourSynth filter (source/source.cpp) builds one CUDA
 *     graph per (resource, plane) with
 *         get_graphexec(d_res, d_src, h_res, width, height, stride, sigma,
 *                       block_step, bm_range, radius, ps_num, ps_range,
 *                       chroma, sigma_u, sigma_v, final_, extractor)
 *     (declared source/source.cpp:45-52, defined source/kernel.cu:759-864)
 *     and runs it with cudaGraphLaunch (source/source.cpp:348, 401).
 *     bm3d_b200_graph_create / _launch take exactly those arguments and
 *     buffers, with the same layouts, and do the same work.
 *
 *  2. The host-side aggregation of that plugin, moved to the device:
 *     Aggregation (source/source.cpp:170-188) and the VAggregate filter's
 *     per-frame loop (source/source.cpp:814-850).
 *
 *  3. A device-resident clip pipeline: all frames of a clip in HBM, every
 *     stage batched over all frames in one launch per kernel, V-BM3D
 *     accumulation straight into each output frame's accumulator (the
 *     VAggregate sum fused into the scatter). This is what the plugin's
 *     BM3Dv2 path and the Python module use for whole clips.
 */
#ifndef BM3D_B200_H
#define BM3D_B200_H

#if defined(__GNUC__)
#define BM3D_B200_API __attribute__((visibility("default")))
#else
#define BM3D_B200_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define BM3D_B200_OK 0
#define BM3D_B200_ERR_INVALID 1     /* an argument is out of range */
#define BM3D_B200_ERR_CUDA 2        /* a CUDA runtime call failed */
#define BM3D_B200_ERR_UNSUPPORTED 3 /* valid for the reference, not supported here */
#define BM3D_B200_ERR_NOMEM 4

/* Largest supported plane side and temporal radius (match positions are
 * packed as 14-bit x, 14-bit y, 4-bit temporal slot). */
#define BM3D_B200_MAX_DIM 16383
#define BM3D_B200_MAX_RADIUS 7

/* Message of the calling thread's most recent failing call ("" if none). */
BM3D_B200_API const char *bm3d_b200_last_error(void);

/* 1-based ABI version of this header. */
BM3D_B200_API int bm3d_b200_abi_version(void);

/* Effective threshold sigma from the user's sigma, as BM3DCreate scales it
 * (source/source.cpp:520-523): sigma * (3/4) / 255 * 64 * (final_ ? 1 : 2.7). */
BM3D_B200_API float bm3d_b200_scale_sigma(float sigma, int final_);

/* ------------------------------------------------------------------------
 * 1. Reference graph replacement
 * ------------------------------------------------------------------------
 * Buffers (all pitched with `stride` floats per row, as in the reference):
 *   d_src: device, [(final_ ? 2 : 1)][planes][2r+1][height][stride];
 *          for final_, the first half is the reference (basic estimate)
 *          clip and the second half the noisy clip.
 *   d_res: device, [planes][2r+1][2][height][stride] accumulators
 *          (wdst slab, then weight slab, per temporal slot).
 *   h_res: host (pinned for async copies), large enough for either layout.
 *   planes = chroma ? 3 : 1. sigma, sigma_u, sigma_v are effective
 *   (already scaled) values; a chroma plane with sigma < FLT_EPSILON is
 *   skipped (source/kernel.cu:664-670). extractor = 2^extractor_exp or 0.
 * The object owns its block-matching scratch memory and a CUDA graph.
 */
typedef struct bm3d_b200_graph bm3d_b200_graph;

BM3D_B200_API int bm3d_b200_graph_create(bm3d_b200_graph **out, float *d_res, float *d_src, float *h_res,
                           int width, int height, int stride, float sigma, int block_step,
                           int bm_range, int radius, int ps_num, int ps_range, int chroma,
                           float sigma_u, float sigma_v, int final_, float extractor);

/* Block-distance and transform variants of the run-time-compiled plugin
 * bm3dcuda_rtc, whose BM3D adds bm_error_s, transform_2d_s and
 * transform_1d_s (rtc_source/source.cpp:854-911, 1370-1387; README.md:118-135)
 * and builds one kernel per plane with them (rtc_source/source.cpp:191-214,
 * 985-1060; rtc_source/kernel.hpp:200-504). The values are the plugin's
 * strings: "ssd", "sad", "zssd", "zsad", "ssd/norm"; "dct", "haar", "wht",
 * "bior1.5". With chroma the plane-0 choices apply to all planes. */
#define BM3D_B200_BM_SSD 0
#define BM3D_B200_BM_SAD 1
#define BM3D_B200_BM_ZSSD 2
#define BM3D_B200_BM_ZSAD 3
#define BM3D_B200_BM_SSD_NORM 4
#define BM3D_B200_TX_DCT 0
#define BM3D_B200_TX_HAAR 1
#define BM3D_B200_TX_WHT 2
#define BM3D_B200_TX_BIOR1_5 3

/* bm3d_b200_graph_create with the variant of one plane's compiled kernel
 * (the rtc plugin's compile() + get_graphexec, rtc_source/source.cpp:191-380). */
BM3D_B200_API int bm3d_b200_graph_create_rtc(bm3d_b200_graph **out, float *d_res, float *d_src,
                                             float *h_res, int width, int height, int stride,
                                             float sigma, int block_step, int bm_range, int radius,
                                             int ps_num, int ps_range, int chroma, float sigma_u,
                                             float sigma_v, int final_, float extractor,
                                             int bm_error, int transform_2d, int transform_1d);

/* h_res -> d_src, zero d_res, BM3D, d_res -> h_res; asynchronous on `stream`
 * (the reference's cudaGraphLaunch of its four-node graph). */
BM3D_B200_API int bm3d_b200_graph_launch(bm3d_b200_graph *g, void *stream);

/* The device part only: zero d_res and run BM3D from d_src into d_res. */
BM3D_B200_API int bm3d_b200_graph_launch_device(bm3d_b200_graph *g, void *stream);

/* Copies the match lists of the last launch to host memory:
 * [planes == 1 ? 1 : 1][nblocks][8][3] ints (x, y, temporal slot), blocks in
 * the reference's scan order. Synchronous. *nblocks receives the count. */
BM3D_B200_API int bm3d_b200_graph_matches(bm3d_b200_graph *g, int *h_xyz, int capacity_blocks, int *nblocks);

BM3D_B200_API void bm3d_b200_graph_destroy(bm3d_b200_graph *g);

/* Allocation-free form of bm3d_b200_graph_launch_device. No counterpart in
 * the reference. For callers that cannot let a library allocate device
 * memory during processing - a host application that owns the whole
 * device-memory budget through its own pool, or a real-time pipeline that
 * cannot absorb the device-wide synchronisation cudaMalloc/cudaFree may
 * cause. Same arguments and buffers as bm3d_b200_graph_create (d_src, d_res
 * provided by the caller); zeroes d_res and runs BM3D on `stream`,
 * asynchronously. Its scratch (pointer tables, block-matching lists) lives in
 * an 8 MiB array inside the library on every device that loads it, so frames
 * are limited to 262016 reference blocks (e.g. 3840x2160 at block_step 8);
 * larger ones return BM3D_B200_ERR_UNSUPPORTED. The first call on a device
 * resolves the array's address there (cudaGetSymbolAddress) and keeps it for
 * the life of the process; make that first call before any stream capture,
 * and do not call this entry point on a device again after cudaDeviceReset
 * there (the kept address would be stale). All calls on a device share the array:
 * calls whose GPU work overlaps (other streams or host threads) race, so
 * issue them in order on one stream. Nothing in the array needs to start at
 * zero - every call writes all of it that it reads. */
BM3D_B200_API int bm3d_b200_window_noalloc(float *d_res, const float *d_src, int width, int height,
                                           int stride, float sigma, int block_step, int bm_range,
                                           int radius, int ps_num, int ps_range, int chroma,
                                           float sigma_u, float sigma_v, int final_,
                                           float extractor, void *stream);

/* ------------------------------------------------------------------------
 * 2. Aggregation on the device
 * ------------------------------------------------------------------------ */

/* d_dst[y][x] = wdst[y][x] / weight[y][x], where d_res points at a wdst slab
 * followed `height` rows later by its weight slab (source/source.cpp:170-188). */
BM3D_B200_API int bm3d_b200_aggregate(float *d_dst, int dst_stride, const float *d_res, int res_stride,
                        int width, int height, void *stream);

/* VAggregate of output frame n of a clip of num_frames frames
 * (source/source.cpp:814-850). vframes: HOST array of 2r+1 DEVICE pointers,
 * the raw BM3D outputs ([2r+1][2][height][raw_stride]) of frames
 * clamp(n-r .. n+r). Replication padding at the clip ends as the reference. */
BM3D_B200_API int bm3d_b200_vaggregate(float *d_dst, int dst_stride, const float *const *vframes,
                         int raw_stride, int width, int height, int radius, int n,
                         int num_frames, void *stream);

/* ------------------------------------------------------------------------
 * 3. Device-resident clip pipeline
 * ------------------------------------------------------------------------
 * Frame layout (device and host): frame f holds its planes back to back,
 * plane p being height_p rows of `stride` floats, height_p = height for
 * p == 0 and height >> subsampling_h otherwise (width likewise). A clip is
 * num_frames such frames. Raw V-BM3D output (dst_mode RAW) holds, per frame
 * and plane, (2r+1) pairs of (wdst, weight) slabs of height_p rows: the
 * reference's BM3D output with height * 2 * (2r+1) (source/source.cpp:190-204).
 */
typedef struct bm3d_b200_params {
    float sigma[3];     /* user-level sigma per plane; < FLT_EPSILON: plane untouched */
    int block_step[3];  /* [1, 8] */
    int bm_range[3];    /* > 0 */
    int ps_num[3];      /* [1, 8] */
    int ps_range[3];    /* > 0 */
    int radius;         /* [0, BM3D_B200_MAX_RADIUS] */
    int chroma;         /* CBM3D: 3 planes of equal size, matching on plane 0 */
    int extractor_exp;  /* 0: atomic order free; > 0: pre-rounded deterministic sums */
    int zero_init;      /* RAW output: zero unprocessed planes (default 1) */
} bm3d_b200_params;

/* Fills the reference's defaults: sigma 3, block_step 8, bm_range 9,
 * ps_num 2, ps_range 4, radius 0, chroma 0, extractor_exp 0, zero_init 1. */
BM3D_B200_API void bm3d_b200_params_default(bm3d_b200_params *p);

#define BM3D_B200_DST_AGGREGATED 0 /* denoised frames (BM3Dv2 output) */
#define BM3D_B200_DST_RAW 1        /* raw V-BM3D stacks (BM3D output, radius > 0) */

typedef struct bm3d_b200_clip bm3d_b200_clip;

BM3D_B200_API int bm3d_b200_clip_create(bm3d_b200_clip **out, int width, int height, int num_planes,
                          int subsampling_w, int subsampling_h, int num_frames,
                          const bm3d_b200_params *params, int device_id);

/* Floats per frame of the source layout, and of the RAW output layout. */
BM3D_B200_API long long bm3d_b200_clip_frame_floats(const bm3d_b200_clip *c);
BM3D_B200_API long long bm3d_b200_clip_raw_frame_floats(const bm3d_b200_clip *c);
BM3D_B200_API int bm3d_b200_clip_stride(const bm3d_b200_clip *c);

/* One BM3D call over every frame, device buffers. d_ref NULL = basic
 * estimate, else final (Wiener) estimate against d_ref. Asynchronous. */
BM3D_B200_API int bm3d_b200_clip_run(bm3d_b200_clip *c, const float *d_src, const float *d_ref, float *d_dst,
                       int dst_mode, void *stream);

/* Same from/to host buffers: the copies and the work run on `stream` (NULL:
 * the clip's own stream), which is synchronised before returning. Pinned
 * (page-locked) host buffers give overlapped, full-bandwidth copies. */
BM3D_B200_API int bm3d_b200_clip_run_host(bm3d_b200_clip *c, const float *h_src, const float *h_ref,
                            float *h_dst, int dst_mode, void *stream);

/* Two-stage V-BM3D (README.md:44-53): vbasic = BM3Dv2(src), vfinal =
 * BM3Dv2(src, ref=vbasic), with the intermediate kept on the device.
 * Host buffers in the source layout; runs on `stream` (NULL: the clip's
 * own) and synchronises it before returning. */
BM3D_B200_API int bm3d_b200_clip_twostage_host(bm3d_b200_clip *c, const float *h_src, float *h_dst,
                                               void *stream);

/* The same, returning once the work is queued on `stream` (no counterpart in
 * the reference). h_src and h_dst must be pinned (page-locked) and stay
 * untouched until the stream has completed. Calls on one clip run in order,
 * on whatever streams they are given (each waits for the clip's previous call).
 * Two clips used in turn, each on its own stream, keep one clip's copies in
 * flight while the other computes; for that use this call pipelines a
 * single-plane clip in three equal chunks (the synchronous call uses more,
 * smaller chunks: the latency of one call). After the stream has completed,
 * bm3d_b200_clip_status reports a tensor-core wait that gave up. */
BM3D_B200_API int bm3d_b200_clip_twostage_host_async(bm3d_b200_clip *c, const float *h_src,
                                                     float *h_dst, void *stream);

/* Device-buffer form of the two-stage run; d_basic receives vbasic.
 * Asynchronous on `stream`. */
BM3D_B200_API int bm3d_b200_clip_twostage(bm3d_b200_clip *c, const float *d_src, float *d_basic,
                            float *d_dst, void *stream);

/* Per-stage device timers (CUDA events recorded on the launching stream
 * around every kernel launch of the clip pipeline). Off by default. */
#define BM3D_B200_STAGE_MATCH 0     /* block matching (basic stage) */
#define BM3D_B200_STAGE_FILTER 1    /* 3-D transform, shrinkage, scatter (basic stage) */
#define BM3D_B200_STAGE_AGGREGATE 2 /* division into the output frames */
#define BM3D_B200_STAGE_PROPOSE 3   /* proposer embeddings (learned matching only) */
#define BM3D_B200_STAGE_MATCH_FINAL 4  /* block matching of the final (Wiener) stage */
#define BM3D_B200_STAGE_FILTER_FINAL 5 /* filtering of the final (Wiener) stage */
#define BM3D_B200_STAGE_FALLBACK 6  /* exhaustive re-search after learned matching */
#define BM3D_B200_NUM_STAGES 7
BM3D_B200_API int bm3d_b200_clip_set_profiling(bm3d_b200_clip *c, int enable);

/* Accumulated milliseconds and kernel launches per stage since the last reset
 * (synchronises with the recorded events). ms / launches: arrays of
 * BM3D_B200_NUM_STAGES entries, either may be NULL. */
BM3D_B200_API int bm3d_b200_clip_stage_times(bm3d_b200_clip *c, double *ms, long long *launches,
                                             int reset);

BM3D_B200_API void bm3d_b200_clip_destroy(bm3d_b200_clip *c);

/* Arithmetic of the collaborative filter's 3-D transforms (no counterpart in
 * the reference). FP32 (default): the reference's 8-point factorisation, step
 * for step. SPLIT_BF16: each pass is a batch of 8x8 contractions on the
 * tensor cores, operands split into three BF16 parts with the six
 * significant products accumulated in FP32 (about FP32 accuracy). TC_F16:
 * the 2-D transform of each patch is one 64 x 64 matrix (the Kronecker
 * product of the 8-point transform with itself) applied to 128 patches per
 * tcgen05 MMA, FP16 operands (patches, transform, shrunk spectra) with FP32
 * accumulation (coefficient errors of about 1e-3 relative); the transform
 * across the group, the shrinkage and the scatter stay FP32. Block matching,
 * ranking and the Wiener division stay FP32 in every mode. */
#define BM3D_B200_PRECISION_FP32 0
#define BM3D_B200_PRECISION_SPLIT_BF16 1
#define BM3D_B200_PRECISION_TC_F16 2
BM3D_B200_API int bm3d_b200_clip_set_precision(bm3d_b200_clip *c, int precision);

/* OK, or BM3D_B200_ERR_CUDA when a tensor-core kernel of the clip's last runs
 * (TC_F16 filter, proposer inference) gave up waiting for its MMAs after
 * about a second and skipped its work. The host-buffer entry points check
 * this themselves; call it after synchronising a device-buffer run. */
BM3D_B200_API int bm3d_b200_clip_status(bm3d_b200_clip *c);

/* Per-plane block distance and transforms of the rtc plugin (BM3D_B200_BM_*,
 * BM3D_B200_TX_*; arrays of 3, NULL = the defaults "ssd" / "dct" / "dct").
 * The variants run on the exhaustive FP32 path: not with a proposer attached
 * nor with the split-BF16 precision (BM3D_B200_ERR_UNSUPPORTED). */
BM3D_B200_API int bm3d_b200_clip_set_variant(bm3d_b200_clip *c, const int *bm_error,
                                             const int *transform_2d, const int *transform_1d);

/* Match lists [nblocks][8][3] (x, y, temporal slot) of window n from the
 * clip's last block matching of plane 0 (synchronises the device); with
 * h_xyz NULL or too small only *nblocks is set. */
BM3D_B200_API int bm3d_b200_clip_matches(bm3d_b200_clip *c, int n, int *h_xyz,
                                         int capacity_blocks, int *nblocks);

/* ------------------------------------------------------------------------
 * 3b. Frame-by-frame V-BM3D for streaming hosts
 * ------------------------------------------------------------------------
 * The reference plugin's BM3Dv2 with radius > 0 is BM3D then VAggregate
 * (source/source.cpp:911-989): each output frame uploads its 2r+1 window
 * frames into a fresh resource (4 resources with fast=True,
 * source/source.cpp:636-713), downloads the window's raw (2r+1) x 2 stack
 * (source/source.cpp:348-372) and VAggregate reads 2r+1 of those stacks again
 * (source/source.cpp:746-862). A stream keeps source (and reference) frames
 * in a device ring keyed by frame index, each uploaded once, and each
 * window's raw stack in a ring of window slots, each computed once; output
 * frame n is the VAggregate of windows clamp(n-r .. n+r) on the device and
 * only it crosses back to the host. Same planes, parameters and results as
 * bm3d_b200_clip_run with DST_AGGREGATED (bit-identical with extractor_exp).
 * final_: final (Wiener) stage, reference frames given alongside.
 * Calls may come from several host threads at once (VapourSynth's fmParallel
 * getFrame): up to bm3d_b200_stream_concurrency(s) requests run concurrently,
 * each on its own CUDA stream, sharing the rings (a frame or window needed by
 * several requests is produced once and waited for by the others). */
typedef struct bm3d_b200_stream bm3d_b200_stream;
typedef struct bm3d_b200_proposer bm3d_b200_proposer;

BM3D_B200_API int bm3d_b200_stream_create(bm3d_b200_stream **out, int width, int height,
                                          int num_planes, int subsampling_w, int subsampling_h,
                                          int num_frames, const bm3d_b200_params *params,
                                          int final_, int device_id);
/* Output frame n. h_src / h_ref: HOST plane pointers [4r+1][3] of frames
 * clamp(n-2r .. n+2r) (planes not processed may be NULL; h_ref NULL for the
 * basic stage), src_strides [4r+1][3] their row pitches in bytes; h_dst[3]
 * receives the processed planes (dst_strides in bytes; other planes are left
 * alone). Synchronous: h_dst is written when the call returns. Thread-safe;
 * concurrent calls overlap their copies and kernels (the windows a call has
 * to compute run as one launch per kernel). */
BM3D_B200_API int bm3d_b200_stream_frame(bm3d_b200_stream *s, int n, const float *const *h_src,
                                         const float *const *h_ref, const int *src_strides,
                                         float *const *h_dst, const int *dst_strides);
/* The rtc plugin's per-plane variants (as bm3d_b200_clip_set_variant). */
BM3D_B200_API int bm3d_b200_stream_set_variant(bm3d_b200_stream *s, const int *bm_error,
                                               const int *transform_2d, const int *transform_1d);
/* Frames uploaded and windows filtered so far (each frame and window once
 * while requests move through the clip in order). */
BM3D_B200_API int bm3d_b200_stream_stats(bm3d_b200_stream *s, long long *frame_uploads,
                                         long long *windows);
/* Device time of the completed calls since the last reset, from CUDA events
 * on each call's stream: ms[0] uploads, ms[1] window filtering (with waits
 * for frames other calls upload), ms[2] VAggregate and download (with waits
 * for windows other calls filter); *calls their number. */
BM3D_B200_API int bm3d_b200_stream_timings(bm3d_b200_stream *s, double *ms, long long *calls,
                                           int reset);
/* Requests that run concurrently (4, as the reference's fast=True resources,
 * fewer when one request's frames and windows exceed 16 GiB). */
BM3D_B200_API int bm3d_b200_stream_concurrency(const bm3d_b200_stream *s);
/* Caps the concurrent requests at `requests` (at most the allocated number;
 * the plugin passes fast ? 4 : 1, source/source.cpp:613-621). Waits for the
 * requests in flight. */
BM3D_B200_API int bm3d_b200_stream_set_concurrency(bm3d_b200_stream *s, int requests);
/* Learned match proposal for the stream (no counterpart in the reference; see
 * bm3d_b200_clip_set_proposer for the arguments): every uploaded frame's
 * matching plane gets its embeddings, every window's block matching becomes
 * learned, with the exhaustive re-search of blocks farther than the fallback
 * threshold. NULL detaches. Waits for the requests in flight and drops the
 * frames and windows kept so far. A call whose proposer inference gave up
 * waiting returns BM3D_B200_ERR_CUDA. The proposer must outlive the stream. */
BM3D_B200_API int bm3d_b200_stream_set_proposer(bm3d_b200_stream *s, bm3d_b200_proposer *p,
                                                int cells_spatial, int cells_temporal,
                                                float fallback_tau);
BM3D_B200_API void bm3d_b200_stream_destroy(bm3d_b200_stream *s);

/* ------------------------------------------------------------------------
 * 4. Batches of uneven clips (no counterpart in the reference)
 * ------------------------------------------------------------------------
 * Many single-plane clips of different sizes and parameters run the
 * two-stage V-BM3D (vbasic = BM3Dv2(src), vfinal = BM3Dv2(src, ref=vbasic))
 * together: each pipeline stage is one persistent launch over all clips and
 * the whole run is one CUDA graph. Clip buffers are device memory with
 * `num_frames` planes of `height` rows of stride (width + 31) / 32 * 32
 * floats; d_dst receives vfinal. Only sigma[0], block_step[0], bm_range[0],
 * ps_num[0], ps_range[0], radius and extractor_exp of the params are used. */
typedef struct bm3d_b200_batch bm3d_b200_batch;

BM3D_B200_API int bm3d_b200_batch_create(bm3d_b200_batch **out, int device_id);
BM3D_B200_API int bm3d_b200_batch_add(bm3d_b200_batch *b, int width, int height, int num_frames,
                                      const bm3d_b200_params *params, const float *d_src,
                                      float *d_dst, int *clip_index);
/* Autotuner (synchronous): times the block-matching stage of the batch for
 * CTA widths of 1, 2, 4 warps and strip widths 8..12, then the persistent
 * filter launches (basic, final) with 1..4 and the aggregation launch with
 * 1, 2, 4, 8 resident CTAs per SM (capped at the occupancy limit), and keeps
 * the fastest of each. No counterpart in the reference (its launch shape is
 * fixed, source/kernel.cu:823-828). */
BM3D_B200_API int bm3d_b200_batch_autotune(bm3d_b200_batch *b, void *stream);
/* The chosen CTA width (warps) and strip width. */
BM3D_B200_API int bm3d_b200_batch_config(const bm3d_b200_batch *b, int *cta_warps, int *strip);
/* The autotuned resident CTAs per SM of the persistent filter (basic, final)
 * and aggregation launches (0: as many as fit, before autotuning). */
BM3D_B200_API int bm3d_b200_batch_grids(const bm3d_b200_batch *b, int *filter_basic_per_sm,
                                        int *filter_final_per_sm, int *aggregate_per_sm);
/* Runs the whole batch on `stream` (asynchronous; the first call records the graph). */
BM3D_B200_API int bm3d_b200_batch_run(bm3d_b200_batch *b, void *stream);
/* The basic estimate (vbasic) of clip clip_index from the last run, copied
 * into d_basic (device, the clip's source layout) on `stream`
 * (asynchronous). No counterpart in the reference. */
BM3D_B200_API int bm3d_b200_batch_basic(bm3d_b200_batch *b, int clip_index, float *d_basic,
                                        void *stream);
/* Per clip, the device time in ms from the batch's first work item to the
 * clip's last final frame (synchronises the device). */
BM3D_B200_API int bm3d_b200_batch_latencies(bm3d_b200_batch *b, double *ms, int capacity);
BM3D_B200_API void bm3d_b200_batch_destroy(bm3d_b200_batch *b);

/* ------------------------------------------------------------------------
 * 5. Learned match proposal (no counterpart in the reference)
 * ------------------------------------------------------------------------
 * A proposer is a small CNN (three 3x3 convolutions, 1 -> 16 -> 16 -> 16
 * channels, ReLU after the first two) over the 2x-downsampled plane. Its
 * output at half-resolution pixel (u/2 + 2, v/2 + 2) embeds the block whose
 * origin (u, v) lies in cell (u/2, v/2). With a proposer attached, a clip's
 * block matching ranks the cells of each search window by embedding
 * distance and computes the exact block distance only for the 4 origins of
 * each of the best cells_spatial (centre frame) / cells_temporal (each
 * neighbour frame, over the union of its ps_num windows) cells. Blocks whose
 * best match other than themselves is farther than fallback_ssd get the
 * exhaustive search instead.
 *
 * Parameters: BM3D_B200_PROPOSER_PARAMS floats, w1 [3][3][1][16], b1 [16],
 * w2 [3][3][16][16], b2 [16], w3 [3][3][16][16], b3 [16], with w[dy][dx][ci][co]
 * weighting input pixel (y + dy - 1, x + dx - 1). Training is FP32 on the
 * device; inference runs the layers on the tensor cores with BF16 operands
 * and FP32 accumulation and stores 8-bit embeddings
 * q[c] = clamp(rint(v[c] * qscale + qoff[c]), 0, 255); cells are ranked by
 * the exact integer squared distance of their q vectors. */
#define BM3D_B200_PROPOSER_PARAMS 4800

/* bm3d_b200_proposer is declared with the streams above. */

BM3D_B200_API int bm3d_b200_proposer_num_params(void);
/* params NULL: the "coarse" network whose 16 outputs are 8x the 4x4
 * half-resolution pixels of the block (ranking by downsampled SSD). */
BM3D_B200_API int bm3d_b200_proposer_create(bm3d_b200_proposer **out, const float *params,
                                            int device_id);
BM3D_B200_API int bm3d_b200_proposer_get_params(bm3d_b200_proposer *p, float *h_params);
/* Replaces the parameters (NULL: coarse) and resets the optimiser state;
 * the quantisation is left as it is. */
BM3D_B200_API int bm3d_b200_proposer_set_params(bm3d_b200_proposer *p, const float *h_params);
BM3D_B200_API void bm3d_b200_proposer_destroy(bm3d_b200_proposer *p);

/* Embedding quantisation: 17 floats, qscale then qoff[16]. NULL sets the
 * coarse network's (qscale 20, qoff -100). */
BM3D_B200_API int bm3d_b200_proposer_get_quant(bm3d_b200_proposer *p, float *h_quant);
BM3D_B200_API int bm3d_b200_proposer_set_quant(bm3d_b200_proposer *p, const float *h_quant);
/* Sets the quantisation from the FP32 embeddings of sample planes
 * [nframes][height][stride] (device): qscale = 127 / (4 * largest channel
 * standard deviation), qoff[c] = 128 - qscale * mean[c]. Synchronous. */
BM3D_B200_API int bm3d_b200_proposer_calibrate(bm3d_b200_proposer *p, const float *d_frames,
                                               int nframes, int width, int height, int stride,
                                               void *stream);

/* Training (distillation from the exhaustive search). d_frames holds nframes
 * planes [height][stride] (device). d_samples: device int[nsamples][4] =
 * (fc, fz, x, y): a reference block at origin (x, y) of frame fc, whose
 * candidate cells are (x/2 + u, y/2 + v), |u|, |v| <= U, of frame fz.
 * d_teacher: device float[nsamples][(2U+1)^2], per cell (index
 * (v+U)*(2U+1) + (u+U)) the smallest exact block distance to the cell's
 * block origins in the plane, +inf for cells without one
 * (bm3d_b200_proposer_teacher computes it). With d the squared embedding
 * distance of a cell to the reference cell, p = softmax(-d) and
 * q = softmax(-(s - min s) / temperature) over the sample's cells, the loss is
 * the mean over samples of KL(q || p).
 * teacher: fills d_teacher on `stream` (no proposer needed). Asynchronous.
 * loss_grad: the loss and its gradient (FP32 forward/backward kernels) at the
 * current parameters, copied to h_loss / h_grad (either may be NULL). */
BM3D_B200_API int bm3d_b200_proposer_teacher(const float *d_frames, int nframes, int width,
                                             int height, int stride, const int *d_samples,
                                             int nsamples, int U, float *d_teacher,
                                             void *stream);
BM3D_B200_API int bm3d_b200_proposer_loss_grad(bm3d_b200_proposer *p, const float *d_frames,
                                               int nframes, int width, int height, int stride,
                                               const int *d_samples, const float *d_teacher,
                                               int nsamples, int U, float temperature,
                                               float *h_loss, float *h_grad, void *stream);
/* `steps` Adam steps (learning rate lr) on the same data, then a calibration
 * of the quantisation on the training frames; h_losses (optional) receives
 * each step's loss. Synchronous. */
BM3D_B200_API int bm3d_b200_proposer_train(bm3d_b200_proposer *p, const float *d_frames,
                                           int nframes, int width, int height, int stride,
                                           const int *d_samples, const float *d_teacher,
                                           int nsamples, int U, float temperature, int steps,
                                           float lr, float *h_losses, void *stream);
/* Inference embeddings of nframes planes: d_emb receives, per frame,
 * [height/2][width/2][16] bytes (quantised, see above). Asynchronous. */
BM3D_B200_API int bm3d_b200_proposer_embed(bm3d_b200_proposer *p, const float *d_frames,
                                           int nframes, int width, int height, int stride,
                                           void *d_emb, void *stream);
/* BM3D_B200_OK, or BM3D_B200_ERR_CUDA when an inference launch of this
 * proposer gave up waiting for its tensor-core work (each wait is bounded to
 * about a second; the embeddings of that launch are then incomplete). Read
 * after the stream that ran the launches has been synchronised; once set, the
 * status stays set for the proposer's lifetime. The clip entry points with
 * host buffers check it themselves. No counterpart in the reference (the
 * proposer is an addition). */
BM3D_B200_API int bm3d_b200_proposer_status(const bm3d_b200_proposer *p);
/* The FP32 training network's embeddings (float, same layout). Synchronous. */
BM3D_B200_API int bm3d_b200_proposer_embed_f32(bm3d_b200_proposer *p, const float *d_frames,
                                               int nframes, int width, int height, int stride,
                                               float *d_emb, void *stream);

/* Learned block matching of one temporal window: d_frames / d_embs are HOST
 * arrays of 2r+1 DEVICE pointers (matching planes, and their 8-bit
 * embeddings from bm3d_b200_proposer_embed). h_xyz receives
 * [nblocks][8][3] (x, y, slot) like bm3d_b200_graph_matches, h_fallback
 * (optional) one flag per block: 1 if the block fell back to the exhaustive
 * search. fallback_ssd <= 0 disables the fallback. Synchronous. */
BM3D_B200_API int bm3d_b200_learned_match(const float *const *d_frames, const void *const *d_embs,
                                          int width, int height, int stride, int block_step,
                                          int bm_range, int radius, int ps_num, int ps_range,
                                          int cells_spatial, int cells_temporal,
                                          float fallback_ssd, int *h_xyz, int *h_fallback,
                                          int capacity_blocks, int *nblocks);

/* Attaches a proposer to a single-plane clip (NULL detaches): its block
 * matching becomes learned with the given cell counts (1..8). fallback_tau
 * > 0 sets fallback_ssd = fallback_tau * 128 * (sigma / 255)^2 for each
 * stage, sigma the user-level sigma: tau times the expected distance of two
 * noisy copies of the same block. The proposer must outlive the attachment. */
BM3D_B200_API int bm3d_b200_clip_set_proposer(bm3d_b200_clip *c, bm3d_b200_proposer *p,
                                              int cells_spatial, int cells_temporal,
                                              float fallback_tau);
/* Block matching of the final stage in the two-stage entry points
 * (bm3d_b200_clip_twostage, bm3d_b200_clip_twostage_host) of a clip with a
 * proposer attached. No counterpart in the reference. SEARCH (default): the
 * learned search on the basic estimate (proposer embeddings of the basic
 * estimate, exhaustive fallback). BASIC_LISTS: every block keeps the 8
 * positions the basic stage matched and re-orders them by their block
 * distance on the basic estimate (the reference's distance); no proposer
 * inference and no cell ranking in the final stage. BASIC_ORDER: the basic
 * stage's lists unchanged, in their basic-stage order (no final-stage
 * matching work at all). Single-plane clips; other runs and clips without a
 * proposer always search. */
#define BM3D_B200_FINAL_MATCH_SEARCH 0
#define BM3D_B200_FINAL_MATCH_BASIC_LISTS 1
#define BM3D_B200_FINAL_MATCH_BASIC_ORDER 2
BM3D_B200_API int bm3d_b200_clip_set_final_matching(bm3d_b200_clip *c, int mode);

/* Blocks matched and blocks that fell back since the last reset
 * (synchronises the clip's work). */
BM3D_B200_API int bm3d_b200_clip_learned_stats(bm3d_b200_clip *c, long long *blocks,
                                               long long *fallbacks, int reset);

/* ------------------------------------------------------------------------
 * Diagnostics
 * ------------------------------------------------------------------------
 * Compares the engine's FMA-corrected reciprocal (used by the Wiener
 * shrinkage) with the IEEE round-to-nearest reciprocal for every float whose
 * bit pattern lies in [lo_bits, hi_bits) on the current device. *mismatches
 * receives the count, *first_bad (optional) the smallest mismatching pattern
 * (0xffffffff if none). Synchronous. */
BM3D_B200_API int bm3d_b200_selftest_reciprocal(unsigned lo_bits, unsigned hi_bits,
                                                unsigned long long *mismatches,
                                                unsigned *first_bad);

#ifdef __cplusplus
}
#endif

#endif /* BM3D_B200_H */
