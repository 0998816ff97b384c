// Test infrastructure only: a harness around the reference's own CPU BM3D
// implementation (bm3dcpu, cpu_source/source.cpp), compiled unchanged from the
// reference tree by oracle/Makefile into oracle/_ref/. Nothing in the product
// links this file.
//
// The reference file is #included as one translation unit, so its `static`
// templates (bm3d<temporal,chroma,final_>, block_matching*, insert_if_not_in*)
// are callable here. With BM3D_EXACT_RCP defined, every `_mm256_rcp_ps` (the
// ~12-bit reciprocal estimate at cpu_source/source.cpp:593, 628, 749) becomes an
// IEEE division, which is the parity build; without it the stock estimate runs.
//
// Entry points:
//   ref_bm3d          - one BM3D call over one frame window, exactly as
//                       BM3DGetFrame does it (cpu_source/source.cpp:1009-1227):
//                       sigma scaling, zeroed accumulators, bm3d<> template.
//   ref_match_lists   - the block-matching result per reference block,
//                       before and after the centre insertion
//                       (cpu_source/source.cpp:787-844).

#include <immintrin.h>

#ifdef BM3D_EXACT_RCP
#define _mm256_rcp_ps(x) _mm256_div_ps(_mm256_set1_ps(1.0f), (x))
#endif

#include BM3D_REF_SOURCE

#include <cstdint>

namespace {

// Same expression as cpu_source/source.cpp:1323-1326.
float scale_sigma(float s, bool final_) {
    s *= (3.f / 4.f) / 255.f * 64.f * (final_ ? 1.0f : 2.7f);
    return s;
}

template <bool temporal, bool chroma, bool final_>
void run_one(float *const *dstps_in, const float *const *srcps, const float *const *refps,
             int width, int height, int stride, const float *sigma_user,
             int block_step, int bm_range, int radius, int ps_num, int ps_range) {
    constexpr int np = chroma ? 3 : 1;
    std::array<float *VS_RESTRICT, np> dstps;
    std::array<float, np> sigma;
    for (int p = 0; p < np; ++p) {
        dstps[p] = dstps_in[p];
        sigma[p] = scale_sigma(sigma_user[p], final_);
    }
    const int temporal_width = 2 * radius + 1;
    float *buffer = nullptr;
    if (!temporal) {
        buffer = vs_aligned_malloc<float>(sizeof(float) * stride * height * 2 * np, 32);
        memset(buffer, 0, sizeof(float) * stride * height * 2 * np);
    } else {
        for (int p = 0; p < np; ++p)
            memset(dstps[p], 0, sizeof(float) * stride * height * 2 * temporal_width);
    }
    using refs_t = std::conditional_t<final_, const float *VS_RESTRICT *, std::nullptr_t>;
    refs_t r{};
    if constexpr (final_) r = const_cast<const float *VS_RESTRICT *>(refps);
    std::conditional_t<temporal, std::nullptr_t, float *VS_RESTRICT> buf{};
    if constexpr (!temporal) buf = buffer;
    bm3d<temporal, chroma, final_>(
        dstps, stride, const_cast<const float *VS_RESTRICT *>(srcps), r,
        width, height, sigma, block_step, bm_range, radius, ps_num, ps_range, buf);
    if (buffer) vs_aligned_free(buffer);
}

}  // namespace

extern "C" {

// dstps: one pointer per processed plane (3 when chroma, else 1).
//   radius == 0: [height][stride] denoised plane.
//   radius  > 0: [2r+1][2][height][stride] raw V-BM3D accumulators.
// srcps/refps: (chroma ? 3 : 1) * (2r+1) plane pointers, plane-major.
// sigma_user: the user-level sigma per processed plane (unscaled).
// stride must be a multiple of 8 floats and dstps 32-byte aligned.
int ref_bm3d(float *const *dstps, const float *const *srcps, const float *const *refps,
             int width, int height, int stride, const float *sigma_user,
             int block_step, int bm_range, int radius, int ps_num, int ps_range, int chroma) {
    if (stride % 8 != 0 || width < 8 || height < 8 || stride < width) return -1;
    const bool final_ = refps != nullptr;
    const bool temporal = radius > 0;
#define BM3D_RUN(T, C, F) run_one<T, C, F>(dstps, srcps, refps, width, height, stride, sigma_user, \
                                           block_step, bm_range, radius, ps_num, ps_range)
    if (temporal) {
        if (chroma) { if (final_) BM3D_RUN(true, true, true); else BM3D_RUN(true, true, false); }
        else        { if (final_) BM3D_RUN(true, false, true); else BM3D_RUN(true, false, false); }
    } else {
        if (chroma) { if (final_) BM3D_RUN(false, true, true); else BM3D_RUN(false, true, false); }
        else        { if (final_) BM3D_RUN(false, false, true); else BM3D_RUN(false, false, false); }
    }
#undef BM3D_RUN
    return 0;
}

// Block-matching lists for every reference block of the frame, in the
// reference's scan order (rows of blocks outer, columns inner).
// mplanes: (2r+1) plane pointers of the matching input (src, or ref for final).
// pre:  [nblocks][8] {x, y, z} before the centre insertion; pre_err: [nblocks][8]
// post: [nblocks][8] {x, y, z} after it. Returns the number of blocks.
int ref_match_lists(int *pre, float *pre_err, int *post, const float *const *mplanes,
                    int width, int height, int stride, int block_step, int bm_range,
                    int radius, int ps_num, int ps_range) {
    int nb = 0;
    const int center = radius;
    for (int _y = 0; _y < height - 8 + block_step; _y += block_step) {
        int y = std::min(_y, height - 8);
        for (int _x = 0; _x < width - 8 + block_step; _x += block_step) {
            int x = std::min(_x, width - 8);
            __m256 reference_block[8];
            load_block(reference_block, &mplanes[center][y * stride + x], stride);
            std::array<float, 8> errors;
            errors.fill(std::numeric_limits<float>::max());
            std::array<int, 8> ix, iy, iz;
            ix.fill(x);
            iy.fill(y);
            iz.fill(center);
            if (radius > 0) {
                block_matching_temporal(errors, ix, iy, iz, reference_block,
                                        const_cast<const float *VS_RESTRICT *>(mplanes), stride,
                                        width, height, bm_range, x, y, radius, ps_num, ps_range);
            } else {
                block_matching(errors, ix, iy, reference_block, mplanes[0], stride,
                               width, height, bm_range, x, y);
            }
            for (int k = 0; k < 8; ++k) {
                if (pre) {
                    pre[(nb * 8 + k) * 3 + 0] = ix[k];
                    pre[(nb * 8 + k) * 3 + 1] = iy[k];
                    pre[(nb * 8 + k) * 3 + 2] = iz[k];
                }
                if (pre_err) pre_err[nb * 8 + k] = errors[k];
            }
            if (radius > 0) insert_if_not_in_temporal(ix, iy, iz, x, y, center);
            else insert_if_not_in(ix, iy, x, y);
            for (int k = 0; k < 8; ++k) {
                if (post) {
                    post[(nb * 8 + k) * 3 + 0] = ix[k];
                    post[(nb * 8 + k) * 3 + 1] = iy[k];
                    post[(nb * 8 + k) * 3 + 2] = iz[k];
                }
            }
            ++nb;
        }
    }
    return nb;
}

}  // extern "C"
