// Collaborative filtering (3-D transform, shrinkage, inverse) and weighted
// scatter for BM3D / V-BM3D on sm_100a, plus the per-pixel aggregation
// kernels (spatial division and VAggregate).
//
// One group (8 matched 8x8 patches of one reference block) is handled by 8
// threads. The 3-D transform runs in the reference's pass order - rows, then
// columns, then across the group - with the reference's 1-D factorisation
// (source/kernel.cu:256-363, cpu_source/source.cpp:596-670):
//
//   thread = column c, holds (patch, row):  vertical pass in registers
//   exchange through shared memory -> thread = row r: horizontal pass
//   exchange back -> thread = column c: group pass, shrinkage
//   inverse: vertical pass, exchange, horizontal pass and group pass
//            (thread = row), exchange back -> thread = column: scatter
//
// The shrinkage runs with the coefficient layout the reference uses (lane =
// column frequency, in-register index = group frequency * 8 + row frequency),
// so the Wiener weight's sum of squares is accumulated in the same order.
//
// Scatter: the 8 threads of a group add 8 contiguous pixels of a patch row per
// instruction, so a warp's reduction touches 4-8 sectors instead of 32. With
// corner weights the weight of a patch is added once, at its top-left pixel;
// the aggregation kernel then sums each pixel's 8x8 neighbourhood of corners,
// which equals the per-pixel weight sum (exactly so with pre-rounding).
//
// Groups are scheduled block-row-major across windows: CTAs running together
// work on the same rows of every window, so the gathered patches and the
// accumulator rows they hit stay resident in L2.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "bm3d_device.cuh"
#include "bm3d_internal.h"

namespace bm3d {

namespace {

constexpr int kXchgGroup = 584;  // words per group in the exchange buffer (8*72 + 8)
constexpr int kCoefGroup = 520;  // words per group of parked Wiener coefficients
constexpr int kGroupsPerCta = 16;

// thread = column `me`, v[p][row] -> thread = row `me`, v[p][col]
__device__ __forceinline__ void col_to_row(float (&v)[8][8], float *S, int me) {
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int i = 0; i < 8; ++i) S[p * 72 + i * 9 + me] = v[p][i];
    __syncwarp();
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int j = 0; j < 8; ++j) v[p][j] = S[p * 72 + me * 9 + j];
    __syncwarp();
}

// thread = row `me`, v[p][col] -> thread = column `me`, v[p][row]
__device__ __forceinline__ void row_to_col(float (&v)[8][8], float *S, int me) {
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int j = 0; j < 8; ++j) S[p * 72 + me * 9 + j] = v[p][j];
    __syncwarp();
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int i = 0; i < 8; ++i) v[p][i] = S[p * 72 + i * 9 + me];
    __syncwarp();
}

// The 8-point passes run two lines per packed FP32x2 instruction stream
// (lines of patches p and p + 1 within the patches; lines of elements i and
// i + 1 across the group); the results are those of the scalar codelets.
__device__ __forceinline__ void pass_in_patch(float (&v)[8][8], bool forward) {
#pragma unroll
    for (int p = 0; p < 8; p += 2) {
        f32x2 t[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) t[k] = pack2(v[p][k], v[p + 1][k]);
        if (forward) dct8_fwd2(t); else dct8_inv2(t);
#pragma unroll
        for (int k = 0; k < 8; ++k) unpack2(t[k], v[p][k], v[p + 1][k]);
    }
}

__device__ __forceinline__ void pass_across_group(float (&v)[8][8], bool forward) {
#pragma unroll
    for (int i = 0; i < 8; i += 2) {
        f32x2 t[8];
#pragma unroll
        for (int p = 0; p < 8; ++p) t[p] = pack2(v[p][i], v[p][i + 1]);
        if (forward) dct8_fwd2(t); else dct8_inv2(t);
#pragma unroll
        for (int p = 0; p < 8; ++p) unpack2(t[p], v[p][i], v[p][i + 1]);
    }
}

// The same passes with run-time transform kinds (the run-time-compiled
// plugin's transform_2d_s / transform_1d_s; kinds are uniform per launch).
__device__ __forceinline__ void pass_in_patch_var(float (&v)[8][8], bool forward, int kind) {
#pragma unroll
    for (int p = 0; p < 8; ++p) tx8(v[p], kind, forward);
}

__device__ __forceinline__ void pass_across_group_var(float (&v)[8][8], bool forward, int kind) {
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        float t[8];
#pragma unroll
        for (int p = 0; p < 8; ++p) t[p] = v[p][i];
        tx8(t, kind, forward);
#pragma unroll
        for (int p = 0; p < 8; ++p) v[p][i] = t[p];
    }
}

__device__ __forceinline__ void forward3d_var(float (&v)[8][8], float *S, int me, int t2d,
                                              int t1d) {
    pass_in_patch_var(v, true, t2d);
    col_to_row(v, S, me);
    pass_in_patch_var(v, true, t2d);
    row_to_col(v, S, me);
    pass_across_group_var(v, true, t1d);
}

// Forward 3-D transform: in thread = column layout, out thread = column layout.
__device__ __forceinline__ void forward3d(float (&v)[8][8], float *S, int me) {
    pass_in_patch(v, true);   // rows (vertical)
    col_to_row(v, S, me);
    pass_in_patch(v, true);   // columns (horizontal)
    row_to_col(v, S, me);
    pass_across_group(v, true);
}

// ---------------------------------------------------------------------------
// Split-BF16 tensor-core transform (precision 1).
//
// The reference's 8-point factorisation is the linear map
//   C[k][n] = 2 c_k cos(pi (2n + 1) k / 16),  c_0 = 1/sqrt(2), c_k = 1,
// and its inverse is C^T (C^T C = 16 I, fwd(inv(x)) = 16 x). Each pass of the
// 3-D transform multiplies the 64 lines of a group along one axis by C (or
// C^T): a [64 x 8] x [8 x 8] contraction, four m16n8k8 BF16 tensor-core tiles.
// Operands are split into three BF16 parts (x = xh + xm + xl, each part the
// rounding of what the previous ones leave) and the six products of order up
// to 2^-16 relative are accumulated in FP32, smallest first:
//   xl Dh + xm Dm + xh Dl + xm Dh + xh Dm + xh Dh,
// which keeps the product accurate to about FP32 rounding (2^-24). The group
// sits in the warp's exchange buffer as G[p*72 + r*9 + c]; the four groups of
// a warp are transformed by the whole warp, one m16n8k8 tile at a time.
// ---------------------------------------------------------------------------
struct SplitB {
    uint32_t h, m, l;  // B fragments (k = 2t, 2t+1; n = lane / 4) of the three parts
};

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi) {
    return (uint32_t)__bfloat16_as_ushort(lo) | ((uint32_t)__bfloat16_as_ushort(hi) << 16);
}

// B fragments of the forward (C) or inverse (C^T) map for this lane: the mma
// computes out[line][n] = sum_k in[line][k] * B[k][n], B[k][n] = D[n][k].
__device__ __forceinline__ SplitB dct_fragment(bool forward, int lane) {
    const int n = lane >> 2, t = lane & 3;
    __nv_bfloat16 h[2], m[2], l[2];
    for (int j = 0; j < 2; ++j) {
        const int k = 2 * t + j;
        const int fr = forward ? n : k, ps = forward ? k : n;  // frequency, position
        const double c = fr == 0 ? 0.70710678118654752440 : 1.0;
        const double d = 2.0 * c * cos(3.14159265358979323846 * (2 * ps + 1) * fr / 16.0);
        h[j] = __double2bfloat16(d);
        const double r1 = d - (double)__bfloat162float(h[j]);
        m[j] = __double2bfloat16(r1);
        l[j] = __double2bfloat16(r1 - (double)__bfloat162float(m[j]));
    }
    return SplitB{pack_bf16(h[0], h[1]), pack_bf16(m[0], m[1]), pack_bf16(l[0], l[1])};
}

__device__ __forceinline__ void split3(float x, __nv_bfloat16 &h, __nv_bfloat16 &m,
                                       __nv_bfloat16 &l) {
    h = __float2bfloat16_rn(x);
    const float r1 = __fsub_rn(x, __bfloat162float(h));
    m = __float2bfloat16_rn(r1);
    l = __float2bfloat16_rn(__fsub_rn(r1, __bfloat162float(m)));
}

__device__ __forceinline__ void mma_k8(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t b) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5}, {%6}, "
        "{%0,%1,%2,%3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(b));
}

// word offset of element k of line l of a pass along `axis`
// (0: along rows r, 1: along columns c, 2: across the group p)
__device__ __forceinline__ int tc_addr(int axis, int l, int k) {
    return axis == 0 ? (l >> 3) * 72 + k * 9 + (l & 7)
                     : axis == 1 ? (l >> 3) * 72 + (l & 7) * 9 + k
                                 : k * 72 + (l >> 3) * 9 + (l & 7);
}

// One pass along `axis` for the warp's four groups (buffers kXchgGroup apart).
__device__ __forceinline__ void tc_pass(float *W, int axis, const SplitB &B, int lane) {
    const int gq = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int gi = 0; gi < 4; ++gi) {
        float *G = W + gi * kXchgGroup;
#pragma unroll
        for (int mt = 0; mt < 4; ++mt) {
            const int l0 = mt * 16 + gq, l1 = l0 + 8;
            const int o00 = tc_addr(axis, l0, 2 * t), o01 = tc_addr(axis, l0, 2 * t + 1);
            const int o10 = tc_addr(axis, l1, 2 * t), o11 = tc_addr(axis, l1, 2 * t + 1);
            __nv_bfloat16 h[4], m[4], l[4];
            split3(G[o00], h[0], m[0], l[0]);
            split3(G[o01], h[1], m[1], l[1]);
            split3(G[o10], h[2], m[2], l[2]);
            split3(G[o11], h[3], m[3], l[3]);
            const uint32_t ah0 = pack_bf16(h[0], h[1]), ah1 = pack_bf16(h[2], h[3]);
            const uint32_t am0 = pack_bf16(m[0], m[1]), am1 = pack_bf16(m[2], m[3]);
            const uint32_t al0 = pack_bf16(l[0], l[1]), al1 = pack_bf16(l[2], l[3]);
            float acc[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            mma_k8(acc, al0, al1, B.h);
            mma_k8(acc, am0, am1, B.m);
            mma_k8(acc, ah0, ah1, B.l);
            mma_k8(acc, am0, am1, B.h);
            mma_k8(acc, ah0, ah1, B.m);
            mma_k8(acc, ah0, ah1, B.h);
            G[o00] = acc[0];
            G[o01] = acc[1];
            G[o10] = acc[2];
            G[o11] = acc[3];
        }
    }
}

// 3-D transform of the warp's groups on the tensor cores: in with thread =
// column `me` of group S (v[p][row]); out the same way, or (READ_BACK false)
// left in S as S[p*72 + r*9 + c]. W = the warp's first buffer.
template <bool READ_BACK = true>
__device__ __forceinline__ void tc_transform3d(float (&v)[8][8], float *S, float *W, int me,
                                               int lane, const SplitB &B) {
#pragma unroll
    for (int p = 0; p < 8; ++p)
#pragma unroll
        for (int r = 0; r < 8; ++r) S[p * 72 + r * 9 + me] = v[p][r];
    __syncwarp();
    tc_pass(W, 0, B, lane);
    __syncwarp();
    tc_pass(W, 1, B, lane);
    __syncwarp();
    tc_pass(W, 2, B, lane);
    __syncwarp();
    if constexpr (READ_BACK) {
#pragma unroll
        for (int p = 0; p < 8; ++p)
#pragma unroll
            for (int r = 0; r < 8; ++r) v[p][r] = S[p * 72 + r * 9 + me];
        __syncwarp();
    }
}

__device__ __forceinline__ void load_group(float (&v)[8][8], const float *const *planes,
                                           const int (&pos)[8], int stride, int c) {
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const float *b = planes[pos_z(pos[p])] + (size_t)pos_y(pos[p]) * stride + pos_x(pos[p]) + c;
#pragma unroll
        for (int r = 0; r < 8; ++r) v[p][r] = __ldg(b + (size_t)r * stride);
    }
}

// The same pixels as load_group, copied asynchronously into C[(p*8 + r)*8 + c]
// (the thread's own slots of the parked-coefficient buffer): they land while
// the thread works on something else, and only this thread reads them.
__device__ __forceinline__ void prefetch_group(float *C, const float *const *planes,
                                               const int (&pos)[8], int stride, int c) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(C + c);
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const float *b = planes[pos_z(pos[p])] + (size_t)pos_y(pos[p]) * stride + pos_x(pos[p]) + c;
#pragma unroll
        for (int r = 0; r < 8; ++r)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d + 4u * (p * 64 + r * 8)),
                         "l"(b + (size_t)r * stride)
                         : "memory");
    }
}

template <bool FINAL>
constexpr size_t filter_smem() {
    return (size_t)kGroupsPerCta * (kXchgGroup + (FINAL ? kCoefGroup : 0)) * sizeof(float);
}

// The kGroupsPerCta groups of CTA index `cta` of one filter launch; TC runs
// the transforms on the tensor cores (split BF16), else in FP32 with the
// reference's factorisation; VAR takes the transform kinds from prm.t2d /
// prm.t1d (FP32).
template <bool FINAL, bool TC, bool VAR = false>
__device__ __forceinline__ void filter_cta(const FilterParams &prm, long long cta, float *fsm) {
    float *xbuf = fsm;
    float *cbuf = fsm + kGroupsPerCta * kXchgGroup;

    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int g = lane >> 3;
    const int me = lane & 7;
    const long long row_groups = (long long)prm.nwin * prm.nbx;  // one block row, all windows
    const long long ngroups = row_groups * (prm.nblk / prm.nbx);
    const long long gid = cta * kGroupsPerCta + warp * 4 + g;
    const bool active = gid < ngroups;
    const long long gidc = active ? gid : 0;
    const int brow = (int)(gidc / row_groups);
    const long long rem = gidc - (long long)brow * row_groups;
    const int wrel = (int)(rem / prm.nbx);
    const int blk = brow * prm.nbx + (int)(rem - (long long)wrel * prm.nbx);
    const int win = prm.win0 + wrel;
    const int tw = 2 * prm.radius + 1;
    float *S = xbuf + (warp * 4 + g) * kXchgGroup;
    float *W = xbuf + warp * 4 * kXchgGroup;
    SplitB Bf{}, Bi{};
    if (TC) {
        Bf = dct_fragment(true, lane);
        Bi = dct_fragment(false, lane);
    }

    int pos[8];
    {
        const int4 *m = reinterpret_cast<const int4 *>(prm.matches +
                                                       ((size_t)win * prm.nblk + blk) * 8);
        const int4 a = __ldg(m), b = __ldg(m + 1);
        pos[0] = a.x; pos[1] = a.y; pos[2] = a.z; pos[3] = a.w;
        pos[4] = b.x; pos[5] = b.y; pos[6] = b.z; pos[7] = b.w;
    }

    const float inv4096 = 1.0f / 4096.0f;
    const float sigma = prm.sigma;
    float v[8][8];
    float weight;

    if (FINAL) {
        // empirical Wiener shrinkage against the basic estimate's spectrum
        // (source/kernel.cu:284-326, cpu_source/source.cpp:617-643). The
        // noisy patches are copied asynchronously into C while the basic
        // estimate's group is loaded and transformed; then each thread swaps
        // its own slots of C: the basic spectrum's Wiener coefficients in,
        // the noisy pixels out, and the noisy group is transformed and
        // scaled by 1/4096 and its coefficient (the reference's two roundings).
        float *C = cbuf + (warp * 4 + g) * kCoefGroup;
        prefetch_group(C, prm.src + (size_t)win * tw, pos, prm.stride, me);
        load_group(v, prm.ref + (size_t)win * tw, pos, prm.stride, me);
        const float sqr_sigma = __fmul_rn(sigma, sigma);
        float norm = 0.0f;
        // both forward transforms run through one copy of the code (a rolled
        // loop keeps the kernel small enough for the instruction caches)
#pragma unroll 1
        for (int it = 0; it < 2; ++it) {
            if (TC) tc_transform3d(v, S, W, me, lane, Bf);
            else if (VAR) forward3d_var(v, S, me, prm.t2d, prm.t1d);
            else forward3d(v, S, me);
            if (it == 1) break;
            asm volatile("cp.async.wait_all;" ::: "memory");
            // Two coefficients (rows r, r + 1) per packed FP32x2 instruction
            // stream; every lane is the scalar IEEE operation, and the
            // weight's sum of squares still runs in the reference's order
            // (p, then r).
            const f32x2 sig2 = splat2(sqr_sigma), one2 = splat2(1.0f);
#pragma unroll
            for (int p = 0; p < 8; ++p) {
#pragma unroll
                for (int r = 0; r < 8; r += 2) {
                    const f32x2 x = pack2(v[p][r], v[p][r + 1]);
                    const f32x2 sq = mul2(x, x);
                    // sq + sigma^2 >= sigma^2 >= (FLT_EPSILON * 0.188)^2: a normal float
                    const f32x2 den = add2(sq, sig2);
                    f32x2 y = pack2(rcp_approx(lo2(den)), rcp_approx(hi2(den)));
                    f32x2 e = fma2(neg2(den), y, one2);  // reciprocal as rcp_rn_normal
                    y = fma2(e, y, y);
                    e = fma2(neg2(den), y, one2);
                    y = fma2(e, y, y);
                    float c0, c1;
                    unpack2(mul2(sq, y), c0, c1);
                    if (p == 0 && r == 0 && me == 0) c0 = 1.0f;  // DC passes unchanged
                    norm = __fmaf_rn(c0, c0, norm);
                    norm = __fmaf_rn(c1, c1, norm);
                    float *slot = C + (p * 8 + r) * 8 + me;
                    v[p][r] = slot[0];
                    v[p][r + 1] = slot[8];
                    slot[0] = c0;
                    slot[8] = c1;
                }
            }
        }
#pragma unroll
        for (int p = 0; p < 8; ++p)
#pragma unroll
            for (int r = 0; r < 8; ++r)
                v[p][r] = __fmul_rn(__fmul_rn(v[p][r], inv4096), C[(p * 8 + r) * 8 + me]);
        norm = __fadd_rn(norm, __shfl_xor_sync(0xffffffffu, norm, 1, 8));
        norm = __fadd_rn(norm, __shfl_xor_sync(0xffffffffu, norm, 2, 8));
        norm = __fadd_rn(norm, __shfl_xor_sync(0xffffffffu, norm, 4, 8));
        weight = __fdiv_rn(1.0f, norm);
    } else {
        // hard thresholding (source/kernel.cu:208-252, cpu_source/source.cpp:562-594)
        load_group(v, prm.src + (size_t)win * tw, pos, prm.stride, me);
        if (TC) tc_transform3d(v, S, W, me, lane, Bf);
        else if (VAR) forward3d_var(v, S, me, prm.t2d, prm.t1d);
        else forward3d(v, S, me);
        int nnz = 0;
#pragma unroll
        for (int p = 0; p < 8; ++p) {
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const float thr = (p == 0 && r == 0 && me == 0) ? 0.0f : sigma;  // DC kept
                const float x = v[p][r];
                const bool keep = fabsf(x) >= thr;
                nnz += keep ? 1 : 0;
                v[p][r] = keep ? __fmul_rn(x, inv4096) : 0.0f;
            }
        }
        nnz += __shfl_xor_sync(0xffffffffu, nnz, 1, 8);
        nnz += __shfl_xor_sync(0xffffffffu, nnz, 2, 8);
        nnz += __shfl_xor_sync(0xffffffffu, nnz, 4, 8);
        weight = __fdiv_rn(1.0f, (float)nnz);
    }

    // inverse: rows, columns, group; the result is left in the exchange
    // buffer as S[p*72 + r*9 + c]
    if (TC) {
        tc_transform3d<false>(v, S, W, me, lane, Bi);
    } else {
        if (VAR) {
            pass_in_patch_var(v, false, prm.t2d);
            col_to_row(v, S, me);
            pass_in_patch_var(v, false, prm.t2d);
            pass_across_group_var(v, false, prm.t1d);
        } else {
            pass_in_patch(v, false);
            col_to_row(v, S, me);
            pass_in_patch(v, false);
            pass_across_group(v, false);
        }
#pragma unroll
        for (int p = 0; p < 8; ++p)
#pragma unroll
            for (int j = 0; j < 8; ++j) S[p * 72 + me * 9 + j] = v[p][j];
        __syncwarp();
    }

    // weighted scatter (source/kernel.cu:717-756); thread `me` owns column
    // `me` of every patch and adds one patch per iteration of a rolled loop
    // (the patch position comes from lane `p` of the group). Pre-rounding with
    // 2^extractor_exp makes the sums independent of the atomic order; a
    // multiplicity of 1 multiplies exactly.
    // Lane `me` resolves patch `me`'s target (plane pointer, multiplicity)
    // once; the loop takes patch p's from lane p of the group.
    int pos_me = pos[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) pos_me = me == k ? pos[k] : pos_me;
    const int z_me = pos_z(pos_me);
    float *const plane_me = prm.acc[(size_t)win * tw + z_me];
    const float mul_me = prm.mult ? prm.mult[(size_t)win * tw + z_me] : 1.0f;
    const unsigned long long dst_me =
        plane_me ? reinterpret_cast<unsigned long long>(
                       plane_me + (size_t)pos_y(pos_me) * prm.acc_stride + pos_x(pos_me))
                 : 0ull;
    const float ext = prm.extractor;
    const float wq = __fsub_rn(__fadd_rn(weight, ext), ext);
#pragma unroll 1
    for (int p = 0; p < 8; ++p) {
        float *wd = reinterpret_cast<float *>(__shfl_sync(0xffffffffu, dst_me, p, 8));
        const float mul = __shfl_sync(0xffffffffu, mul_me, p, 8);
        if (!active || wd == nullptr) continue;
        const float wm = __fmul_rn(wq, mul);
        float *wt = wd + prm.weight_offset;
        const float *sp = S + p * 72 + me;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            float val = __fmul_rn(weight, sp[r * 9]);
            val = __fsub_rn(__fadd_rn(val, ext), ext);
            atomicAdd(wd + (size_t)r * prm.acc_stride + me, __fmul_rn(val, mul));
            if (!prm.corner_weight) atomicAdd(wt + (size_t)r * prm.acc_stride + me, wm);
        }
        if (prm.corner_weight && me == 0) atomicAdd(wt, wm);
    }
}

// Resident CTAs per SM the register allocation aims at: the hard-threshold
// FP32 kernel fits 96 registers without spills (5 CTAs: 1.30 ms against 1.33
// at 4 for the 30-window launch); the Wiener kernel's shared memory allows 3.
template <bool FINAL, bool TC, bool VAR>
constexpr int filter_ctas_per_sm() {
    return FINAL ? 3 : (TC || VAR ? 4 : 5);
}

template <bool FINAL, bool TC, bool VAR = false>
__global__ void __launch_bounds__(128, filter_ctas_per_sm<FINAL, TC, VAR>())
    filter_kernel(FilterParams prm) {
    extern __shared__ float fsm[];
    filter_cta<FINAL, TC, VAR>(prm, blockIdx.x, fsm);
}

// Persistent form over a batch of clips: resident CTAs take CTA-sized group
// ranges from a shared counter, clip-major.
template <bool FINAL>
__global__ void __launch_bounds__(128, 3) filter_batch_kernel(FilterBatch b) {
    extern __shared__ float fsm[];
    __shared__ FilterParams ps;
    __shared__ long long item_s;
    const long long total = b.item_off[b.nclips];
    for (;;) {
        if (threadIdx.x == 0) item_s = (long long)atomicAdd(b.counter, 1ULL);
        __syncthreads();
        const long long item = item_s;
        if (item >= total) break;
        int lo = 0, hi = b.nclips;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (b.item_off[mid] <= item) lo = mid; else hi = mid;
        }
        if (threadIdx.x == 0) ps = b.clips[lo];
        __syncthreads();
        filter_cta<FINAL, false>(ps, item - b.item_off[lo], fsm);
        __syncthreads();
    }
}

// dst = wdst / weight; with corner weights the weight of a pixel is the sum of
// the corner plane over its 8x8 up-left neighbourhood. A CTA handles a 32x8
// output tile; corner sums run vertically then horizontally in a fixed order.
// A CTA of 256 threads covers a 128 x 16 tile; each thread 8 consecutive
// pixels of one row, loaded and stored as float4 pairs when aligned.
constexpr int kAggTx = 128, kAggTy = 16, kAggThreads = 256;

__device__ __forceinline__ void load8(float (&v)[8], const float *src, int x, int width,
                                      bool vec) {
    if (vec && x + 8 <= width) {
        const float4 u = *reinterpret_cast<const float4 *>(src);
        const float4 w = *reinterpret_cast<const float4 *>(src + 4);
        v[0] = u.x; v[1] = u.y; v[2] = u.z; v[3] = u.w;
        v[4] = w.x; v[5] = w.y; v[6] = w.z; v[7] = w.w;
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) v[k] = x + k < width ? src[k] : 1.0f;
    }
}

// corner tile: columns x0-8 .. x0+kAggTx-1 (float4 aligned when x0 is), rows
// y0-7 .. y0+kAggTy-1; the smem pitch keeps every row 16-byte aligned
constexpr int kAggCq = (kAggTx + 8) / 4;                      // float4 per corner row
constexpr int kAggCp = kAggTx + 12;                           // smem pitch (floats)
constexpr int kAggCItems = (kAggTy + 7) * kAggCq;             // float4 per tile
constexpr int kAggCIter = (kAggCItems + kAggThreads - 1) / kAggThreads;

__device__ __forceinline__ void aggregate_tile(const AggregateParams &p, int tile_x, int tile_y,
                                               int pl) {
    __shared__ __align__(16) float corner[kAggTy + 7][kAggCp];
    __shared__ float colsum[kAggTy][kAggTx + 8];
    const int x0 = tile_x * kAggTx, y0 = tile_y * kAggTy;
    const float *wd = p.wdst + pl * p.acc_plane_stride;
    const float *wt = wd + p.weight_offset;
    const int tid = threadIdx.x;
    const int ly = tid / (kAggTx / 8), lx = (tid % (kAggTx / 8)) * 8;
    const int y = y0 + ly, x = x0 + lx;
    const bool ok = y < p.height && x < p.width;
    float a[8], w[8];
    if (ok) load8(a, wd + (size_t)y * p.acc_stride + x, x, p.width, p.vec);
    if (p.corner_weight) {
        // the weight of a pixel is the sum of the corner plane over its 8x8
        // up-left neighbourhood: column sums, then row sums, in a fixed order.
        // All of a thread's corner loads are issued before the first store to
        // shared memory (one memory latency per tile, not one per element).
        float4 cv[kAggCIter];
#pragma unroll
        for (int j = 0; j < kAggCIter; ++j) {
            const int i = tid + j * kAggThreads;
            const int ty = i / kAggCq, q = i - ty * kAggCq;
            const int gy = y0 - 7 + ty, gx = x0 - 8 + 4 * q;
            float t[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (i < kAggCItems && gy >= 0 && gy < p.height) {
                const float *row = wt + (size_t)gy * p.acc_stride;
                if (p.vec && gx >= 0 && gx + 4 <= p.width) {
                    const float4 u = *reinterpret_cast<const float4 *>(row + gx);
                    t[0] = u.x; t[1] = u.y; t[2] = u.z; t[3] = u.w;
                } else {
#pragma unroll
                    for (int k = 0; k < 4; ++k)
                        if (gx + k >= 0 && gx + k < p.width) t[k] = row[gx + k];
                }
            }
            cv[j] = make_float4(t[0], t[1], t[2], t[3]);
        }
#pragma unroll
        for (int j = 0; j < kAggCIter; ++j) {
            const int i = tid + j * kAggThreads;
            const int ty = i / kAggCq, q = i - ty * kAggCq;
            if (i < kAggCItems) *reinterpret_cast<float4 *>(&corner[ty][4 * q]) = cv[j];
        }
        __syncthreads();
        // colsum column tx covers corner column tx + 1 (pixel x0 - 7 + tx). A
        // task is one column of 8 output rows: its 15 corner values are read
        // once and summed 8 at a time in the fixed order.
        static_assert(kAggTy % 8 == 0, "column tasks of 8 rows");
        for (int i = tid; i < (kAggTy / 8) * (kAggTx + 7); i += kAggThreads) {
            const int ty0 = 8 * (i / (kAggTx + 7)), tx = i % (kAggTx + 7);
            float c[15];
#pragma unroll
            for (int j = 0; j < 15; ++j) c[j] = corner[ty0 + j][tx + 1];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                float s = 0.0f;
#pragma unroll
                for (int d = 0; d < 8; ++d) s = __fadd_rn(s, c[t + d]);
                colsum[ty0 + t][tx] = s;
            }
        }
        __syncthreads();
        if (!ok) return;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            float s = 0.0f;
#pragma unroll
            for (int d = 0; d < 8; ++d) s = __fadd_rn(s, colsum[ly][lx + k + d]);
            w[k] = s;
        }
    } else {
        if (!ok) return;
        load8(w, wt + (size_t)y * p.acc_stride + x, x, p.width, p.vec);
    }
    float o[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) o[k] = __fdiv_rn(a[k], w[k]);
    float *dst = p.dst + pl * p.dst_plane_stride + (size_t)y * p.dst_stride + x;
    if (p.vec && x + 8 <= p.width) {
        *reinterpret_cast<float4 *>(dst) = make_float4(o[0], o[1], o[2], o[3]);
        *reinterpret_cast<float4 *>(dst + 4) = make_float4(o[4], o[5], o[6], o[7]);
    } else {
#pragma unroll
        for (int k = 0; k < 8; ++k)
            if (x + k < p.width) dst[k] = o[k];
    }
}

__global__ void __launch_bounds__(kAggThreads, 5) aggregate_kernel(AggregateParams p) {
    aggregate_tile(p, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Persistent aggregation over a batch of clips. When `remaining` is set, the
// CTA that finishes a clip's last tile stamps the clip's completion time.
__global__ void __launch_bounds__(kAggThreads) aggregate_batch_kernel(AggregateBatch b) {
    __shared__ AggregateParams ps;
    __shared__ long long item_s;
    const long long total = b.item_off[b.nclips];
    for (;;) {
        if (threadIdx.x == 0) item_s = (long long)atomicAdd(b.counter, 1ULL);
        __syncthreads();
        const long long item = item_s;
        if (item >= total) break;
        int lo = 0, hi = b.nclips;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (b.item_off[mid] <= item) lo = mid; else hi = mid;
        }
        if (threadIdx.x == 0) ps = b.clips[lo];
        __syncthreads();
        const long long j = item - b.item_off[lo];
        const int ntx = (ps.width + kAggTx - 1) / kAggTx, nty = (ps.height + kAggTy - 1) / kAggTy;
        aggregate_tile(ps, (int)(j % ntx), (int)((j / ntx) % nty), (int)(j / ((long long)ntx * nty)));
        __syncthreads();
        if (threadIdx.x == 0 && b.remaining) {
            __threadfence();
            if (atomicSub(b.remaining + lo, 1u) == 1u) b.end_ns[lo] = globaltimer_ns();
        }
    }
}

__global__ void vaggregate_kernel(VAggregateParams p) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const int k = blockIdx.z;
    if (x >= p.width) return;
    const int n = p.n0 + k;
    const int tw = 2 * p.radius + 1;
    float sw = 0.0f, sv = 0.0f;
    for (int i = 0; i < tw; ++i) {
        // replication padding at the clip ends (source/source.cpp:832-836)
        const int s = min(max(2 * p.radius - i, n - p.num_frames + 1 + p.radius), n + p.radius);
        const float *f = p.base ? p.base + (size_t)min(max(n - p.radius + i, 0), p.num_frames - 1) *
                                              p.raw_frame_floats
                                : p.vf[i];
        const float *a = f + ((size_t)s * 2 * p.height + y) * p.raw_stride + x;
        sv = __fadd_rn(sv, a[0]);
        sw = __fadd_rn(sw, a[(size_t)p.height * p.raw_stride]);
    }
    p.dst[k * p.dst_plane_stride + (size_t)y * p.dst_stride + x] = __fdiv_rn(sv, sw);
}

}  // namespace

namespace {

template <bool FINAL, bool TC, bool VAR = false>
cudaError_t launch_filter_t(const FilterParams &p, dim3 grid, cudaStream_t stream) {
    // opt in to more than 48 KB of dynamic shared memory once per device
    static int configured[64] = {};
    cudaError_t e = raise_smem_limit(configured, (const void *)filter_kernel<FINAL, TC, VAR>,
                                      filter_smem<FINAL>());
    if (e != cudaSuccess) return e;
    filter_kernel<FINAL, TC, VAR><<<grid, 128, filter_smem<FINAL>(), stream>>>(p);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_filter(const FilterParams &p, bool final_, cudaStream_t stream) {
    const long long ngroups = (long long)p.nwin * p.nblk;
    if (ngroups == 0) return cudaSuccess;
    if (p.nbx <= 0 || p.nblk % p.nbx != 0) return cudaErrorInvalidValue;
    const long long nblocks = (ngroups + kGroupsPerCta - 1) / kGroupsPerCta;
    if (nblocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    const dim3 grid((unsigned)nblocks);
    if (p.t2d < 0 || p.t2d > 3 || p.t1d < 0 || p.t1d > 3) return cudaErrorInvalidValue;
    if (p.t2d != 0 || p.t1d != 0) {
        if (p.precision != 0) return cudaErrorInvalidValue;  // variants run in FP32
        return final_ ? launch_filter_t<true, false, true>(p, grid, stream)
                      : launch_filter_t<false, false, true>(p, grid, stream);
    }
    if (p.precision == 2) return launch_filter_tc(p, final_, stream);
    if (p.precision == 1)
        return final_ ? launch_filter_t<true, true>(p, grid, stream)
                      : launch_filter_t<false, true>(p, grid, stream);
    return final_ ? launch_filter_t<true, false>(p, grid, stream)
                  : launch_filter_t<false, false>(p, grid, stream);
}

namespace {

// Resident CTAs of a persistent launch: SMs x `per_sm_want` CTAs, at most
// the occupancy limit (per_sm_want <= 0: the limit).
int persistent_grid(const void *fn, int threads, size_t smem, int per_sm_want = 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
    per_sm = std::max(1, per_sm);
    if (per_sm_want > 0) per_sm = std::min(per_sm, per_sm_want);
    return std::max(1, sms) * per_sm;
}

}  // namespace

cudaError_t launch_filter_batch(const FilterBatch &b, bool final_, cudaStream_t stream,
                                int ctas_per_sm) {
    static int configured[2][64] = {};
    cudaError_t e = final_ ? raise_smem_limit(configured[1], (const void *)filter_batch_kernel<true>,
                                              filter_smem<true>())
                           : raise_smem_limit(configured[0],
                                              (const void *)filter_batch_kernel<false>,
                                              filter_smem<false>());
    if (e != cudaSuccess) return e;
    if (final_) {
        const int grid = persistent_grid((const void *)filter_batch_kernel<true>, 128,
                                         filter_smem<true>(), ctas_per_sm);
        filter_batch_kernel<true><<<grid, 128, filter_smem<true>(), stream>>>(b);
    } else {
        const int grid = persistent_grid((const void *)filter_batch_kernel<false>, 128,
                                         filter_smem<false>(), ctas_per_sm);
        filter_batch_kernel<false><<<grid, 128, filter_smem<false>(), stream>>>(b);
    }
    return cudaGetLastError();
}

long long filter_ctas(const FilterParams &p) {
    return ((long long)p.nwin * p.nblk + kGroupsPerCta - 1) / kGroupsPerCta;
}

long long aggregate_tiles(const AggregateParams &p) {
    return (long long)((p.width + kAggTx - 1) / kAggTx) * ((p.height + kAggTy - 1) / kAggTy) *
           p.nplanes;
}

bool aggregate_vec(const AggregateParams &p) {
    const unsigned long long align = reinterpret_cast<unsigned long long>(p.wdst) |
                                     reinterpret_cast<unsigned long long>(p.dst);
    return (align % 16 == 0) && p.acc_stride % 4 == 0 && p.dst_stride % 4 == 0 &&
           p.acc_plane_stride % 4 == 0 && p.dst_plane_stride % 4 == 0 && p.weight_offset % 4 == 0;
}

cudaError_t launch_aggregate_batch(const AggregateBatch &b, cudaStream_t stream,
                                   int ctas_per_sm) {
    const int grid = persistent_grid((const void *)aggregate_batch_kernel, kAggThreads, 0,
                                     ctas_per_sm);
    aggregate_batch_kernel<<<grid, kAggThreads, 0, stream>>>(b);
    return cudaGetLastError();
}

cudaError_t launch_aggregate(const AggregateParams &p, cudaStream_t stream) {
    if (p.nplanes == 0) return cudaSuccess;
    AggregateParams q = p;
    // float4 access needs 16-byte aligned rows in every plane
    const unsigned long long align = reinterpret_cast<unsigned long long>(p.wdst) |
                                     reinterpret_cast<unsigned long long>(p.dst);
    q.vec = (align % 16 == 0) && p.acc_stride % 4 == 0 && p.dst_stride % 4 == 0 &&
            p.acc_plane_stride % 4 == 0 && p.dst_plane_stride % 4 == 0 &&
            p.weight_offset % 4 == 0;
    dim3 block(kAggThreads);
    dim3 grid((p.width + kAggTx - 1) / kAggTx, (p.height + kAggTy - 1) / kAggTy, p.nplanes);
    aggregate_kernel<<<grid, block, 0, stream>>>(q);
    return cudaGetLastError();
}

cudaError_t launch_vaggregate(const VAggregateParams &p, cudaStream_t stream) {
    if (p.nout == 0) return cudaSuccess;
    dim3 block(128), grid((p.width + 127) / 128, p.height, p.nout);
    vaggregate_kernel<<<grid, block, 0, stream>>>(p);
    return cudaGetLastError();
}

}  // namespace bm3d
