/*
 * Minimal, project-written helpers with the names the bm3d filter code uses
 * from the VapourSynth SDK's VSHelper.h (format check, int narrowing, aligned
 * allocation, plane blit). Implementations are this project's own.
 */
#ifndef BM3D_B200_VSHELPER_MIN_H
#define BM3D_B200_VSHELPER_MIN_H

#include <limits.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "VapourSynth.h"

#ifndef VS_RESTRICT
#define VS_RESTRICT __restrict
#endif

static inline int isConstantFormat(const VSVideoInfo *vi) {
    return vi->height > 0 && vi->width > 0 && vi->format != 0;
}

static inline int int64ToIntS(int64_t i) {
    if (i > INT_MAX) return INT_MAX;
    if (i < INT_MIN) return INT_MIN;
    return (int)i;
}

static inline void vs_bitblt(void *dstp, int dst_stride, const void *srcp, int src_stride,
                             size_t row_size, size_t height) {
    if (!height) return;
    if (src_stride == dst_stride && (size_t)src_stride == row_size) {
        memcpy(dstp, srcp, row_size * height);
        return;
    }
    const uint8_t *s = (const uint8_t *)srcp;
    uint8_t *d = (uint8_t *)dstp;
    for (size_t i = 0; i < height; ++i) {
        memcpy(d, s, row_size);
        s += src_stride;
        d += dst_stride;
    }
}

#ifdef __cplusplus
template <typename T>
static inline T *vs_aligned_malloc(size_t size, size_t alignment) {
    void *p = nullptr;
    if (posix_memalign(&p, alignment, size) != 0) return nullptr;
    return static_cast<T *>(p);
}
static inline void vs_aligned_free(void *ptr) { free(ptr); }
#endif

#endif /* BM3D_B200_VSHELPER_MIN_H */
