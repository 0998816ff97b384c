// Internal launch interfaces of the BM3D kernels (not part of the C ABI).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <mutex>

struct bm3d_b200_proposer;

namespace bm3d {

// Raises the dynamic shared-memory limit of kernel `fn` on the current device
// to at least `bytes` (never lowers it). `cfg` is the calling site's record of
// the limit set per device; the check and the update hold one lock, so host
// threads launching at the same time keep the record consistent. Launches
// recorded into CUDA graphs repeat no attribute call once the limit is set.
inline cudaError_t raise_smem_limit(int (&cfg)[64], const void *fn, size_t bytes) {
    static std::mutex mu;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < 64 && cfg[dev] >= (int)bytes) return cudaSuccess;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess && dev >= 0 && dev < 64) cfg[dev] = (int)bytes;
    return e;
}

// Inference weights of a proposer (bm3d_proposer.cu).
const uint32_t *proposer_frag(const bm3d_b200_proposer *p);
const float *proposer_bias(const bm3d_b200_proposer *p);
unsigned *proposer_err(const bm3d_b200_proposer *p);
// 0, or the error status recorded for an inference launch (read after a sync)
int proposer_check(const bm3d_b200_proposer *p);
int proposer_device(const bm3d_b200_proposer *p);

// Block matching over a batch of temporal windows.
struct MatchParams {
    const float *const *frames;  // [nwin][2r+1] matching planes (src, or ref for final)
    int *matches;                // [nwin][nby][nbx][8] packed (x, y, z)
    int width, height, stride;
    int block_step, bm_range, radius, ps_num, ps_range;
    int nbx, nby;
    int win0;        // first window of this launch (grid z covers win0 ...)
    int pitch;       // shared-memory tile pitch (words)
    int tile_rows;   // rows of the shared-memory tile
    int extra_cols;  // strip overrun columns beyond the widest window
    int nsub_s, nsub_t;
    int metric;      // block distance: 0 SSD; 1 SAD, 2 ZSSD, 3 ZSAD, 4 SSD/NORM
};

struct MatchGeometry {
    int nbx, nby;
    int ks, kt, nsub_s, nsub_t, extra_cols;
    int wx;  // warps per CTA along x
    int pitch;
    int tile_rows;
    size_t smem;
};

MatchGeometry match_geometry(int width, int height, int block_step, int bm_range, int radius,
                             int ps_range);
// Geometry with a given CTA width (warps) and strip width K (autotuner).
MatchGeometry match_geometry_with(int width, int height, int block_step, int bm_range, int radius,
                                  int ps_range, int wx, int K);
// CTA tiles of one launch over nwin windows.
long long match_tiles(const MatchGeometry &g, int nwin);
cudaError_t launch_match(const MatchParams &p, const MatchGeometry &g, int nwin,
                         cudaStream_t stream);

// Learned block matching (bm3d_learned.cu): candidate cells ranked by the
// proposer's embeddings, the best ones scored exactly; blocks whose best
// non-centre match stays above fallback_ssd are listed for the exhaustive
// re-search (launch_match_fallback), which reproduces launch_match's list.
struct LearnedParams {
    const void *const *embs;  // [nwin][2r+1] 8-bit embeddings [height/2][width/2][16]
    int w2;                   // embedding row length in cells (width / 2)
    int cells_s, cells_t;     // cells scored exactly per spatial / temporal search (1..8)
    float fallback_ssd;       // > 0: re-search blocks whose best other match exceeds it
    unsigned *fallback;       // [capacity] window * nblk + block, or null
    unsigned *fallback_count;  // zero before the launch
    unsigned fallback_capacity;
};
MatchGeometry learned_geometry(int width, int height, int block_step, int bm_range, int radius,
                               int ps_range);
cudaError_t launch_learned_match(const MatchParams &p, const LearnedParams &lp,
                                 const MatchGeometry &g, int nwin, cudaStream_t stream);
// Whether every candidate cell of a stage gets a distinct 12-bit ordinal
// (spatial: (bm_range + 2)^2 cells at most; temporal: ps_num windows of
// (ps_range + 2)^2), which the learned matcher's ranking keys need.
bool learned_ordinals_fit(int bm_range, int ps_num, int ps_range);
// Final-stage lists from the basic stage's: the 8 positions of every block's
// list in p.matches (windows p.win0 .. p.win0 + nwin - 1) scored on p.frames
// with the reference's block distance and sorted in place (stable).
cudaError_t launch_rescore(const MatchParams &p, int nwin, cudaStream_t stream);
// Exhaustive re-search of the blocks listed by the learned matcher.
cudaError_t launch_match_fallback(const MatchParams &p, const unsigned *list,
                                  const unsigned *count, cudaStream_t stream);

// Proposer network inference (bm3d_proposer.cu): 8-bit embeddings of nframes
// planes, frame_floats apart, into emb (emb_frame bytes apart); *err (device
// address of the proposer's error word) gets a nonzero bit if a CTA gave up
// waiting for its tensor-core work.
cudaError_t launch_embed(const float *src, long long frame_floats, int nframes, int width,
                         int height, int stride, const uint32_t *frag, const float *bias,
                         uint8_t *emb, long long emb_frame, unsigned *err, cudaStream_t s);

// Persistent block matching over a batch of clips (one launch).
struct MatchBatch {
    const MatchParams *clips;      // [nclips] per-clip parameters (device)
    const long long *item_off;     // [nclips + 1] prefix sums of CTA tiles (device)
    int nclips;
    unsigned long long *counter;   // work counter, zero at launch
    unsigned long long *start_ns;  // globaltimer stamp of the first tile
};
cudaError_t launch_match_batch(const MatchBatch &b, int K, int wx, size_t smem,
                               cudaStream_t stream);

// Collaborative filtering + scatter of one plane over a batch of windows.
struct FilterParams {
    const float *const *src;  // [nwin][2r+1] noisy planes of the filtered plane
    const float *const *ref;  // [nwin][2r+1] basic-estimate planes (final stage) or null
    float *const *acc;        // [nwin][2r+1] wdst plane receiving slot z, or null (dropped)
    const float *mult;        // [nwin][2r+1] multiplicity of slot z in its target, or null (1)
    const int *matches;       // [nwin][nblk][8]
    long long weight_offset;  // floats from a wdst plane to its weight plane
    int acc_stride;
    int stride;
    int radius;
    int nblk;
    int nbx;  // blocks per block row (groups are scheduled row-major across windows)
    int win0;  // first window of this launch
    int nwin;  // windows win0 .. win0 + nwin - 1
    int corner_weight;  // 1: add each patch's weight once at its top-left pixel
    float sigma;        // effective sigma (already scaled)
    float extractor;    // 2^extractor_exp, or 0
    int precision;      // 0: FP32, the reference's factorisation; 1: split-BF16 tensor
                        // cores; 2: FP16 Kronecker-form 2-D transforms on tcgen05
    int t2d, t1d;       // transforms (rows/columns, group): 0 DCT, 1 Haar, 2 WHT, 3 bior1.5
    unsigned *err;      // precision 2: set to nonzero when a CTA gave up waiting for its MMAs
};

cudaError_t launch_filter(const FilterParams &p, bool final_, cudaStream_t stream);
// precision 2 (bm3d_filter_tc.cu)
cudaError_t launch_filter_tc(const FilterParams &p, bool final_, cudaStream_t stream);

// dst[y][x] = wdst[y][x] / weight[y][x] over a batch of planes.
struct AggregateParams {
    float *dst;
    const float *wdst;
    long long dst_plane_stride;  // floats between consecutive output planes
    long long acc_plane_stride;  // floats between consecutive accumulator pairs
    long long weight_offset;
    int dst_stride, acc_stride;
    int width, height, nplanes;
    int corner_weight;  // weight plane holds per-patch corner weights (8x8 box sum)
    bool vec;           // set by launch_aggregate: rows allow float4 access
};
cudaError_t launch_aggregate(const AggregateParams &p, cudaStream_t stream);

// Persistent filtering / aggregation over a batch of clips (one launch each).
struct FilterBatch {
    const FilterParams *clips;    // [nclips] (device)
    const long long *item_off;    // [nclips + 1] prefix sums of CTA group ranges
    int nclips;
    unsigned long long *counter;  // zero at launch
};
struct AggregateBatch {
    const AggregateParams *clips;  // [nclips] (device); vec precomputed per clip
    const long long *item_off;     // [nclips + 1] prefix sums of tiles
    int nclips;
    unsigned long long *counter;   // zero at launch
    unsigned *remaining;           // [nclips] tiles left, or null (no stamps)
    unsigned long long *end_ns;    // [nclips] globaltimer when a clip's last tile is done
};
// ctas_per_sm: resident CTAs per SM of the persistent grid (<= 0: as many
// as fit; the batch autotuner picks it)
cudaError_t launch_filter_batch(const FilterBatch &b, bool final_, cudaStream_t stream,
                                int ctas_per_sm = 0);
cudaError_t launch_aggregate_batch(const AggregateBatch &b, cudaStream_t stream,
                                   int ctas_per_sm = 0);
long long filter_ctas(const FilterParams &p);
long long aggregate_tiles(const AggregateParams &p);
bool aggregate_vec(const AggregateParams &p);

// VAggregate (source/source.cpp:746-862) for a batch of output frames.
struct VAggregateParams {
    float *dst;  // [nout] planes, dst_plane_stride apart
    // Raw V-BM3D outputs ([2r+1][2][height][raw_stride] each): either one
    // pointer per window slot for a single output frame (vf), or a clip base
    // with one raw frame every raw_frame_floats floats (base != null).
    const float *vf[2 * 7 + 1];
    const float *base;
    long long raw_frame_floats;
    long long dst_plane_stride;
    int dst_stride, raw_stride;
    int width, height, radius;
    int n0;  // index of the first output frame
    int num_frames;
    int nout;
};
cudaError_t launch_vaggregate(const VAggregateParams &p, cudaStream_t stream);

}  // namespace bm3d
