// Collaborative filtering on the 5th-generation tensor cores (precision
// BM3D_B200_PRECISION_TC_F16; no counterpart in the reference, whose 3-D
// transform is source/kernel.cu:256-363).
//
// The 2-D part of the 3-D transform of a group is one matrix per patch: the
// separable 8-point transform C along rows and columns is the Kronecker
// product T = C (x) C, T[(u,v)][(r,c)] = C[u][r] C[v][c], a 64 x 64 matrix
// (C[k][n] = 2 c_k cos(pi (2n+1) k / 16), c_0 = 1/sqrt 2, the reference's
// scaled DCT-II; its inverse is C^T, so the inverse 2-D transform is T^T).
// A CTA takes 16 groups = 128 patches, one M = 128 row each:
//
//   gather  8 lanes per patch row load the patches (one sector per row),
//           store them as FP16 into the K-major operand [128 patches][64 px]
//   MMA     D[patch][coefficient] = A . T^T: 4 tcgen05.mma kind::f16 of
//           M = 128, N = 64, K = 16, FP32 accumulators in tensor memory (the
//           Wiener filter also transforms the basic estimate's patches)
//   group   per 16-coefficient chunk: tcgen05.ld (thread = patch), a warp
//           transpose through shared memory (thread = group x 2 coefficients
//           x 8 patches), the reference's 8-point transform across the group
//           and its inverse in FP32 (packed FP32x2), the shrinkage (hard
//           threshold or Wiener) in FP32, transposed back and stored as FP16
//           into the inverse operand [128 patches][64 coefficients]
//   MMA     inverse 2-D transform: D[patch][pixel] = A . T
//   scatter tcgen05.ld, a transpose to 8 lanes per patch row, and the
//           reference's weighted scatter with the same reductions as the
//           FP32 kernel (pre-rounding, multiplicities, corner weights)
//
// The 2-D transforms see FP16 operands (11-bit significands) with FP32 sums,
// so coefficients carry relative errors of about 1e-3; thresholding, the
// Wiener coefficients, the group transform and the accumulation are FP32.
// The results are not bit-identical to the reference's arithmetic (see
// bm3d_filter.cu for that path); the tests bound their distance to it.
//
// Every wait on an mbarrier is bounded (about a second); on expiry the CTA
// records an error in *prm.err, skips its remaining work, releases its tensor
// memory and returns.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "bm3d_device.cuh"
#include "bm3d_internal.h"
#include "bm3d_umma.cuh"

namespace bm3d {

namespace {

constexpr int kTGroups = 16;                    // groups per CTA: 128 patches = M
constexpr int kTThreads = 128;
constexpr uint32_t kTSbo = 144;                 // bytes between 8-patch core-matrix groups
constexpr uint32_t kTLboA = kTGroups * kTSbo;   // bytes between 8-element K chunks (2304)
constexpr uint32_t kTABytes = 8 * kTLboA;       // one [128][64] FP16 operand (18432)
constexpr uint32_t kTLboB = 1024, kTSboB = 128;  // T operand: [64][64] FP16, unpadded
constexpr uint32_t kTBBytes = 64 * 64 * 2;
constexpr int kTPad = 33;                       // transpose pitch (words)
constexpr uint32_t kTTBytes = 4 * 16 * kTPad * 4;  // one spectrum chunk, 4 warps
constexpr int kTSGroup = 520;                   // scatter buffer words per group
constexpr int kTSPatch = 65;                    // scatter buffer words per patch
constexpr uint32_t kTSBytes = kTGroups * kTSGroup * 4;
// kind::f16 with FP16 A and B (format 0), FP32 D, both K-major, N = 64, M = 128
constexpr uint32_t kTIdesc = (1u << 4) | ((64u >> 3) << 17) | ((128u >> 4) << 24);

template <bool FINAL>
__host__ __device__ constexpr uint32_t tc_region() {
    return FINAL ? 2 * kTABytes + 2 * kTTBytes
                 : (kTABytes + kTTBytes > kTSBytes ? kTABytes + kTTBytes : kTSBytes);
}
template <bool FINAL>
__host__ __device__ constexpr size_t tc_smem() {
    return (size_t)tc_region<FINAL>() + 2 * kTBBytes + 64 * 4 + 32;
}
static_assert(tc_region<true>() >= kTSBytes, "scatter buffer fits the Wiener region");
static_assert(tc_smem<true>() < (1u << 18), "descriptor addresses fit");

__device__ __forceinline__ void umma_f16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate) {
    const uint32_t z = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
        :
        : "r"(d_tmem), "l"(adesc), "l"(bdesc), "r"(kTIdesc), "r"(accumulate), "r"(z));
}

__device__ __forceinline__ uint32_t f16x2(float lo, float hi) {
    __half2 h = __floats2half2_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&h);
}

// The 2-D transform's MMAs: D (TMEM) = A . B^T over K = 64 (4 steps of 16).
__device__ __forceinline__ void umma_k64(uint32_t d, uint32_t a_s, uint32_t b_s) {
#pragma unroll
    for (int j = 0; j < 4; ++j)
        umma_f16(d, umma_desc(a_s + 2u * j * kTLboA, kTLboA, kTSbo),
                 umma_desc(b_s + 2u * j * kTLboB, kTLboB, kTSboB), j > 0 ? 1u : 0u);
}

template <bool FINAL>
__global__ void __launch_bounds__(kTThreads, FINAL ? 3 : 4) filter_tc_kernel(FilterParams prm) {
    extern __shared__ __align__(1024) unsigned char tsm[];
    constexpr uint32_t kRegion = tc_region<FINAL>();
    unsigned char *a0 = tsm;                              // noisy patches, then inverse operand
    unsigned char *a1 = tsm + kTABytes;                   // basic-estimate patches (FINAL)
    float *tn = reinterpret_cast<float *>(tsm + (FINAL ? 2 : 1) * kTABytes);  // transposes
    float *tb = tn + 4 * 16 * kTPad;                      // (FINAL)
    float *sbuf = reinterpret_cast<float *>(tsm);        // scatter rows, after the inverse MMA
    unsigned char *bf = tsm + kRegion;                    // T^T operand (forward)
    unsigned char *bi = bf + kTBBytes;                    // T operand (inverse)
    float *ctab = reinterpret_cast<float *>(bi + kTBBytes);  // C[k][n], 64 floats
    uint64_t *bar = reinterpret_cast<uint64_t *>(ctab + 64);  // 2 mbarriers
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bar + 2);
    const uint32_t a0_s = (uint32_t)__cvta_generic_to_shared(a0);
    const uint32_t a1_s = (uint32_t)__cvta_generic_to_shared(a1);
    const uint32_t bf_s = (uint32_t)__cvta_generic_to_shared(bf);
    const uint32_t bi_s = (uint32_t)__cvta_generic_to_shared(bi);
    const uint32_t bar_s = (uint32_t)__cvta_generic_to_shared(bar);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int g = lane >> 3, me = lane & 7;
    const int G = warp * 4 + g;  // group of the CTA (0..15)

    // ---- set-up: tensor memory, barriers, the transform matrices ----------
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         (uint32_t)__cvta_generic_to_shared(tslot)),
                     "r"(FINAL ? 128u : 64u)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid < 2) mbar_init(bar_s + 8u * tid, 1u);
    if (tid < 64) {
        const int k = tid >> 3, n = tid & 7;
        const double ck = k == 0 ? 0.70710678118654752440 : 1.0;
        ctab[tid] = (float)(2.0 * ck * cos(3.14159265358979323846 * (2 * n + 1) * k / 16.0));
    }
    __syncthreads();
    // T^T for the forward MMA: B[n = (u,v)][k = (r,c)] = C[u][r] C[v][c];
    // T for the inverse: B[n = (r,c)][k = (u,v)], the same products.
    // Element (n, k) of a [64][64] K-major operand lies at byte
    // (k / 8) * 1024 + (n / 8) * 128 + (n % 8) * 16 + (k % 8) * 2.
    for (int i = tid; i < 64 * 32; i += kTThreads) {
        const int n = i >> 5, k = 2 * (i & 31);  // elements (n, k), (n, k + 1)
        const uint32_t off = (uint32_t)(k / 8) * kTLboB + (uint32_t)(n / 8) * kTSboB +
                             (uint32_t)(n % 8) * 16u + (uint32_t)(k % 8) * 2u;
        const int u = n >> 3, v = n & 7, r0 = k >> 3, c0 = k & 7;  // forward
        *reinterpret_cast<uint32_t *>(bf + off) =
            f16x2(ctab[u * 8 + r0] * ctab[v * 8 + c0], ctab[u * 8 + r0] * ctab[v * 8 + c0 + 1]);
        const int r = n >> 3, c = n & 7, u0 = k >> 3, v0 = k & 7;  // inverse
        *reinterpret_cast<uint32_t *>(bi + off) =
            f16x2(ctab[u0 * 8 + r] * ctab[v0 * 8 + c], ctab[u0 * 8 + r] * ctab[(v0 + 1) * 8 + c]);
    }

    // ---- groups of this CTA (block rows across windows, as the FP32 kernel)
    const long long row_groups = (long long)prm.nwin * prm.nbx;
    const long long ngroups = row_groups * (prm.nblk / prm.nbx);
    const long long gid = (long long)blockIdx.x * kTGroups + G;
    const bool active = gid < ngroups;
    const long long gidc = active ? gid : 0;
    const int brow = (int)(gidc / row_groups);
    const long long rem = gidc - (long long)brow * row_groups;
    const int wrel = (int)(rem / prm.nbx);
    const int blk = brow * prm.nbx + (int)(rem - (long long)wrel * prm.nbx);
    const int win = prm.win0 + wrel;
    const int tw = 2 * prm.radius + 1;
    int pos[8];
    {
        const int4 *m = reinterpret_cast<const int4 *>(prm.matches +
                                                       ((size_t)win * prm.nblk + blk) * 8);
        const int4 a = __ldg(m), b = __ldg(m + 1);
        pos[0] = a.x; pos[1] = a.y; pos[2] = a.z; pos[3] = a.w;
        pos[4] = b.x; pos[5] = b.y; pos[6] = b.z; pos[7] = b.w;
    }

    // ---- gather: lane `me` = column, FP16 pairs (me, me + 1) from even lanes.
    // Element (m = 8G + p, k = 8r + me) at r * kTLboA + G * kTSbo + p * 16 + me * 2.
#pragma unroll 1
    for (int it = 0; it < (FINAL ? 2 : 1); ++it) {
        const float *const *planes = (it == 0 ? prm.src : prm.ref) + (size_t)win * tw;
        unsigned char *a = it == 0 ? a0 : a1;
        float v[8][8];
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            const float *b = planes[pos_z(pos[p])] + (size_t)pos_y(pos[p]) * prm.stride +
                             pos_x(pos[p]) + me;
#pragma unroll
            for (int r = 0; r < 8; ++r) v[p][r] = __ldg(b + (size_t)r * prm.stride);
        }
#pragma unroll
        for (int p = 0; p < 8; ++p)
#pragma unroll
            for (int r = 0; r < 8; ++r) {
                const float nb = __shfl_down_sync(0xffffffffu, v[p][r], 1, 8);
                if ((me & 1) == 0)
                    *reinterpret_cast<uint32_t *>(a + (uint32_t)r * kTLboA + (uint32_t)G * kTSbo +
                                                  (uint32_t)p * 16u + (uint32_t)me * 2u) =
                        f16x2(v[p][r], nb);
            }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    bool ok = true;

    // ---- forward 2-D transform(s) ------------------------------------------
    if (tid == 0) {
        umma_k64(tmem, a0_s, bf_s);
        if (FINAL) umma_k64(tmem + 64u, a1_s, bf_s);
        umma_commit(bar_s);
    }
    ok = __syncthreads_and(mbar_wait_bounded(bar_s, 0)) != 0;
    tc_fence_after();

    // ---- group transform, shrinkage, inverse group transform ---------------
    // Chunk j: coefficients 16j .. 16j + 15 of every patch. In the transpose
    // buffer row c holds coefficient c of the warp's 32 patches; thread
    // (g, q = me) takes coefficients q and q + 8 of group g's 8 patches.
    const uint32_t tq = tmem + ((uint32_t)(32 * warp) << 16);
    float *tw_n = tn + warp * 16 * kTPad;
    float *tw_b = tb + warp * 16 * kTPad;
    const float inv4096 = 1.0f / 4096.0f;
    const float sigma = prm.sigma;
    int nnz = 0;
    float norm = 0.0f;
    const int q = me;
#pragma unroll 1
    for (int j = 0; j < 4 && ok; ++j) {
        float cn[16], cb[16];
        tmem_ld16(tq + 16u * j, cn);
        if (FINAL) tmem_ld16(tq + 64u + 16u * j, cb);
#pragma unroll
        for (int c = 0; c < 16; ++c) {
            tw_n[c * kTPad + lane] = cn[c];
            if (FINAL) tw_b[c * kTPad + lane] = cb[c];
        }
        __syncwarp();
        f32x2 x[8], y[8];
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            x[p] = pack2(tw_n[q * kTPad + 8 * g + p], tw_n[(q + 8) * kTPad + 8 * g + p]);
            if (FINAL) y[p] = pack2(tw_b[q * kTPad + 8 * g + p], tw_b[(q + 8) * kTPad + 8 * g + p]);
        }
        __syncwarp();
        dct8_fwd2(x);
        if (FINAL) dct8_fwd2(y);
#pragma unroll
        for (int f = 0; f < 8; ++f) {
            float x0, x1;
            unpack2(x[f], x0, x1);
            const bool dc = j == 0 && q == 0 && f == 0;  // coefficient (0, 0), group frequency 0
            if (FINAL) {
                float y0, y1;
                unpack2(y[f], y0, y1);
                const float s0 = y0 * y0, s1 = y1 * y1, ss = sigma * sigma;
                const float w0 = dc ? 1.0f : s0 / (s0 + ss), w1 = s1 / (s1 + ss);
                norm += w0 * w0 + w1 * w1;
                x0 *= w0 * inv4096;
                x1 *= w1 * inv4096;
            } else {
                const bool k0 = dc || fabsf(x0) >= sigma, k1 = fabsf(x1) >= sigma;
                nnz += (k0 ? 1 : 0) + (k1 ? 1 : 0);
                x0 = k0 ? x0 * inv4096 : 0.0f;
                x1 = k1 ? x1 * inv4096 : 0.0f;
            }
            x[f] = pack2(x0, x1);
        }
        dct8_inv2(x);
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            float z0, z1;
            unpack2(x[p], z0, z1);
            tw_n[q * kTPad + 8 * g + p] = z0;
            tw_n[(q + 8) * kTPad + 8 * g + p] = z1;
        }
        __syncwarp();
        // thread = patch m = 32 warp + lane: its 16 coefficients, as FP16,
        // into K chunks 2j and 2j + 1 of the inverse operand (over a0)
        uint32_t h[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) h[c] = f16x2(tw_n[(2 * c) * kTPad + lane],
                                                 tw_n[(2 * c + 1) * kTPad + lane]);
        __syncwarp();
        const int m = 32 * warp + lane;
        unsigned char *dst = a0 + (uint32_t)(m >> 3) * kTSbo + (uint32_t)(m & 7) * 16u;
        *reinterpret_cast<uint4 *>(dst + (2u * j) * kTLboA) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(dst + (2u * j + 1u) * kTLboA) =
            make_uint4(h[4], h[5], h[6], h[7]);
    }
    // group weight: 1 / kept coefficients (hard threshold), 1 / sum of squared
    // Wiener coefficients; the 8 lanes of a group hold all 512 coefficients
    float weight;
    if (FINAL) {
        norm += __shfl_xor_sync(0xffffffffu, norm, 1);
        norm += __shfl_xor_sync(0xffffffffu, norm, 2);
        norm += __shfl_xor_sync(0xffffffffu, norm, 4);
        weight = 1.0f / norm;
    } else {
        nnz += __shfl_xor_sync(0xffffffffu, nnz, 1);
        nnz += __shfl_xor_sync(0xffffffffu, nnz, 2);
        nnz += __shfl_xor_sync(0xffffffffu, nnz, 4);
        weight = 1.0f / (float)max(nnz, 1);
    }
    fence_async_smem();
    tc_fence_before();
    ok = __syncthreads_and(ok) != 0;
    tc_fence_after();

    // ---- inverse 2-D transform ---------------------------------------------
    if (ok && tid == 0) {
        umma_k64(tmem, a0_s, bi_s);
        umma_commit(bar_s + 8u);
    }
    if (ok) ok = mbar_wait_bounded(bar_s + 8u, 0);
    ok = __syncthreads_and(ok) != 0;
    tc_fence_after();

    // ---- pixels to the scatter layout: word G * 520 + p * 65 + r * 8 + c
    if (ok) {
        const int m = 32 * warp + lane, mg = m >> 3, mp = m & 7;
        float *srow = sbuf + mg * kTSGroup + mp * kTSPatch;
#pragma unroll 1
        for (int j = 0; j < 4; ++j) {
            float px[16];
            tmem_ld16(tq + 16u * j, px);
#pragma unroll
            for (int k = 0; k < 16; ++k) srow[16 * j + k] = px[k];  // pixel (r, c) = 8 r + c
        }
    }
    tc_fence_before();
    ok = __syncthreads_and(ok) != 0;
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(FINAL ? 128u : 64u)
                     : "memory");
    }
    if (!ok) {
        if (tid == 0 && prm.err) atomicOr(prm.err, 1u);
        return;
    }

    // ---- weighted scatter (as the FP32 kernel: source/kernel.cu:717-756) ---
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
    const float *sg = sbuf + G * kTSGroup;
#pragma unroll 1
    for (int p = 0; p < 8; ++p) {
        float *wd = reinterpret_cast<float *>(__shfl_sync(0xffffffffu, dst_me, p, 8));
        const float mul = __shfl_sync(0xffffffffu, mul_me, p, 8);
        if (!active || wd == nullptr) continue;
        const float wm = __fmul_rn(wq, mul);
        float *wt = wd + prm.weight_offset;
        const float *sp = sg + p * kTSPatch + me;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
            float val = __fmul_rn(weight, sp[r * 8]);
            val = __fsub_rn(__fadd_rn(val, ext), ext);
            atomicAdd(wd + (size_t)r * prm.acc_stride + me, __fmul_rn(val, mul));
            if (!prm.corner_weight) atomicAdd(wt + (size_t)r * prm.acc_stride + me, wm);
        }
        if (prm.corner_weight && me == 0) atomicAdd(wt, wm);
    }
}

template <bool FINAL>
cudaError_t launch_tc(const FilterParams &p, unsigned grid, cudaStream_t stream) {
    static int configured[64] = {};
    cudaError_t e = raise_smem_limit(configured, (const void *)filter_tc_kernel<FINAL>,
                                     tc_smem<FINAL>());
    if (e != cudaSuccess) return e;
    filter_tc_kernel<FINAL><<<grid, kTThreads, tc_smem<FINAL>(), stream>>>(p);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_filter_tc(const FilterParams &p, bool final_, cudaStream_t stream) {
    const long long ngroups = (long long)p.nwin * p.nblk;
    if (ngroups == 0) return cudaSuccess;
    if (p.nbx <= 0 || p.nblk % p.nbx != 0) return cudaErrorInvalidValue;
    const long long nblocks = (ngroups + kTGroups - 1) / kTGroups;
    if (nblocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    return final_ ? launch_tc<true>(p, (unsigned)nblocks, stream)
                  : launch_tc<false>(p, (unsigned)nblocks, stream);
}

}  // namespace bm3d
