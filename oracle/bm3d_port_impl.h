/*
 * Test infrastructure only (the oracle): scalar C restatement of the BM3D /
 * V-BM3D algorithm of the reference CPU implementation, cpu_source/source.cpp.
 * Included twice by bm3d_port.c: once with REAL=float (arithmetic step for step
 * like bm3dcpu built with an exact reciprocal, so results are bit-identical to
 * it) and once with REAL=double (the FP64 oracle, exact division everywhere).
 *
 * Layout conventions follow the reference:
 *   a plane is [height][stride] floats; a group is g[64][8] where row index
 *   i = patch * 8 + row-within-patch and the 8 lanes are the patch columns
 *   (cpu_source/source.cpp:393-421, one __m256 per patch row).
 *   radius > 0 output: [2r+1][2][height][stride] (wdst slab, then weight slab)
 *   (cpu_source/source.cpp:705-735).
 */

#define PCAT_(a, b) a##b
#define PCAT(a, b) PCAT_(a, b)
#define FN(name) PCAT(name, SFX)

/* ---- 8-point scaled DCT-II / DCT-III (cpu_source/source.cpp:441-536) ----
 * Same FFTW-derived factorisation and the same fused multiply-add placement as
 * the reference, so the float instantiation rounds identically. */
static void FN(dct8_fwd)(REAL v[8]) {
    const REAL KP414213562 = (REAL)0.414213562373095048801688724209698078569671875;
    const REAL KP1_847759065 = (REAL)1.847759065022573512256366378793576573644833252;
    const REAL KP198912367 = (REAL)0.198912367379658006911597622644676228597850501;
    const REAL KP1_961570560 = (REAL)1.961570560806460898252364472268478073947867462;
    const REAL KP1_414213562 = (REAL)1.414213562373095048801688724209698078569671875;
    const REAL KP668178637 = (REAL)0.668178637919298919997757686523080761552472251;
    const REAL KP1_662939224 = (REAL)1.662939224605090474157576755235811513477121624;
    const REAL KP707106781 = (REAL)0.707106781186547524400844362104849039284835938;
    REAL T1 = v[0], T2 = v[7];
    REAL T3 = T1 - T2, Tj = T1 + T2;
    REAL Tc = v[4], Td = v[3];
    REAL Te = Tc - Td, Tk = Tc + Td;
    REAL T4 = v[2], T5 = v[5];
    REAL T6 = T4 - T5;
    REAL T7 = v[1], T8 = v[6];
    REAL T9 = T7 - T8;
    REAL Ta = T6 + T9, Tn = T7 + T8, Tf = T6 - T9, Tm = T4 + T5;
    REAL Tb = RFMA(-KP707106781, Ta, T3);
    REAL Tg = RFMA(-KP707106781, Tf, Te);
    v[3] = KP1_662939224 * RFMA(KP668178637, Tg, Tb);
    v[5] = -(KP1_662939224 * RFMA(-KP668178637, Tb, Tg));
    REAL Tp = Tj + Tk, Tq = Tm + Tn;
    v[4] = KP1_414213562 * (Tp - Tq);
    v[0] = KP1_414213562 * (Tp + Tq);
    REAL Th = RFMA(KP707106781, Ta, T3);
    REAL Ti = RFMA(KP707106781, Tf, Te);
    v[1] = KP1_961570560 * RFMA(-KP198912367, Ti, Th);
    v[7] = KP1_961570560 * RFMA(KP198912367, Th, Ti);
    REAL Tl = Tj - Tk, To = Tm - Tn;
    v[2] = KP1_847759065 * RFMA(-KP414213562, To, Tl);
    v[6] = KP1_847759065 * RFMA(KP414213562, Tl, To);
}

static void FN(dct8_inv)(REAL v[8]) {
    const REAL KP1_662939224 = (REAL)1.662939224605090474157576755235811513477121624;
    const REAL KP668178637 = (REAL)0.668178637919298919997757686523080761552472251;
    const REAL KP1_961570560 = (REAL)1.961570560806460898252364472268478073947867462;
    const REAL KP198912367 = (REAL)0.198912367379658006911597622644676228597850501;
    const REAL KP1_847759065 = (REAL)1.847759065022573512256366378793576573644833252;
    const REAL KP707106781 = (REAL)0.707106781186547524400844362104849039284835938;
    const REAL KP414213562 = (REAL)0.414213562373095048801688724209698078569671875;
    const REAL KP1_414213562 = (REAL)1.414213562373095048801688724209698078569671875;
    REAL T1 = KP1_414213562 * v[0];
    REAL T2 = v[4];
    REAL T3 = RFMA(KP1_414213562, T2, T1);
    REAL Tj = RFMA(-KP1_414213562, T2, T1);
    REAL T4 = v[2], T5 = v[6];
    REAL T6 = RFMA(KP414213562, T5, T4);
    REAL Tk = RFMA(KP414213562, T4, -T5);
    REAL T8 = v[1], Td = v[7], T9 = v[5], Ta = v[3];
    REAL Tb = T9 + Ta, Te = Ta - T9;
    REAL Tc = RFMA(KP707106781, Tb, T8);
    REAL Tn = RFMA(-KP707106781, Te, Td);
    REAL Tf = RFMA(KP707106781, Te, Td);
    REAL Tm = RFMA(-KP707106781, Tb, T8);
    REAL T7 = RFMA(KP1_847759065, T6, T3);
    REAL Tg = RFMA(KP198912367, Tf, Tc);
    v[7] = RFMA(-KP1_961570560, Tg, T7);
    v[0] = RFMA(KP1_961570560, Tg, T7);
    REAL Tp = RFMA(-KP1_847759065, Tk, Tj);
    REAL Tq = RFMA(KP668178637, Tm, Tn);
    v[5] = RFMA(-KP1_662939224, Tq, Tp);
    v[2] = RFMA(KP1_662939224, Tq, Tp);
    REAL Th = RFMA(-KP1_847759065, T6, T3);
    REAL Ti = RFMA(-KP198912367, Tc, Tf);
    v[3] = RFMA(-KP1_961570560, Ti, Th);
    v[4] = RFMA(KP1_961570560, Ti, Th);
    REAL Tl = RFMA(KP1_847759065, Tk, Tj);
    REAL To = RFMA(-KP668178637, Tn, Tm);
    v[6] = RFMA(-KP1_662939224, To, Tl);
    v[1] = RFMA(KP1_662939224, To, Tl);
}

/*
 * Transforms of the run-time-compiled plugin variant (bm3dcuda_rtc,
 * rtc_source/kernel.hpp:200-380): Haar, Walsh-Hadamard and biorthogonal
 * spline 1.5, "normalized, scaled" like the DCT. Coefficients are the
 * reference's; every product is rounded on its own (no fusion) and sums run
 * left to right, the rounding sequence the engine's kernels use too. The
 * reference's inverse Haar combines only coefficients 0, 1, 2 and 4
 * (rtc_source/kernel.hpp:226-252); it is restated as it is.
 */
static void FN(haar8)(REAL v[8], int forward) {
    const REAL S = (REAL)1.414213562373095048801688724209698078569671875;
    const REAL S2 = S * (REAL)2;
    if (forward) {
        REAL T1 = v[0] + v[1], T2 = v[0] - v[1], T3 = v[2] + v[3], T4 = v[2] - v[3];
        REAL T5 = v[4] + v[5], T6 = v[4] - v[5], T7 = v[6] + v[7], T8 = v[6] - v[7];
        REAL T9 = T1 + T3, T10 = S * (T1 - T3), T11 = T5 + T7, T12 = S * (T5 - T7);
        v[0] = S * (T9 + T11); v[1] = S * (T9 - T11); v[2] = S * T10; v[3] = S * T12;
        v[4] = S2 * T2; v[5] = S2 * T4; v[6] = S2 * T6; v[7] = S2 * T8;
    } else {
        REAL T1 = v[0] + v[1], T2 = v[0] - v[1];
        REAL a = S * v[2], b = (REAL)2 * v[4];
        REAL P = a + b, Q = a - b, R = -a + b, U = -a - b;
        v[0] = S * (T1 + P); v[1] = S * (T1 + Q); v[2] = S * (T1 + R); v[3] = S * (T1 + U);
        v[4] = S * (T2 + P); v[5] = S * (T2 + Q); v[6] = S * (T2 + R); v[7] = S * (T2 + U);
    }
}

static void FN(wht8)(REAL v[8]) {
    const REAL S = (REAL)1.414213562373095048801688724209698078569671875;
    REAL T1 = v[0] + v[1], T2 = v[0] - v[1], T3 = v[2] + v[3], T4 = v[2] - v[3];
    REAL T5 = v[4] + v[5], T6 = v[4] - v[5], T7 = v[6] + v[7], T8 = v[6] - v[7];
    REAL T9 = T1 + T3, T10 = T1 - T3, T11 = T2 + T4, T12 = T2 - T4;
    REAL T13 = T5 + T7, T14 = T5 - T7, T15 = T6 + T8, T16 = T6 - T8;
    v[0] = S * (T9 + T13); v[1] = S * (T9 - T13); v[2] = S * (T10 - T14); v[3] = S * (T10 + T14);
    v[4] = S * (T12 + T16); v[5] = S * (T12 - T16); v[6] = S * (T11 - T15); v[7] = S * (T11 + T15);
}

static void FN(bior8)(REAL v[8], int forward) {
    const REAL S = (REAL)1.414213562373095048801688724209698078569671875;
    const REAL C2828 = (REAL)2.828427124746190097603377448419396157139343751;
    if (forward) {
        const REAL C877 = (REAL)0.877670597010003062405456290501163901200537360;
        const REAL C1797 = (REAL)1.797135031972863413496886690073811797696338403;
        const REAL C2277 = (REAL)2.277437593371384746027611934034934695963515886;
        const REAL C1609 = (REAL)1.609389232649111887192845766718020518480884560;
        const REAL C334 = (REAL)0.334024180361136429417383083658457088741315663;
        REAL T1 = v[0] + v[3], T2 = v[0] - v[3], T3 = v[1] + v[2], T4 = v[1] - v[2];
        REAL T5 = v[4] + v[7], T6 = v[4] - v[7], T7 = v[5] + v[6], T8 = v[5] - v[6];
        REAL T9 = v[0] - v[1], T10 = v[2] - v[3], T11 = v[4] - v[5], T12 = v[6] - v[7];
        v[0] = S * (((T1 + T5) + T3) + T7);
        v[1] = C877 * (T1 - T5) + C1797 * (T3 - T7);
        v[2] = (C2277 * T2 + C1609 * T4) + C334 * (T8 - T6);
        v[3] = (C2277 * T6 + C1609 * T8) + C334 * (T4 - T2);
        v[4] = C2828 * T9; v[5] = C2828 * T10; v[6] = C2828 * T11; v[7] = C2828 * T12;
    } else {
        const REAL C1495 = (REAL)1.495435764250674860795011090214036706658653686;
        const REAL C2058 = (REAL)2.058234225009388964222454285384072231477027482;
        const REAL C486 = (REAL)0.486135912065751423025580498947083714508324707;
        REAL T1 = S * v[0], T2 = C1495 * v[1], T3 = C2058 * v[2], T4 = C2058 * v[3];
        REAL T5 = C2828 * v[4], T6 = C486 * v[4], T7 = C2828 * v[5], T8 = C486 * v[5];
        REAL T9 = C2828 * v[6], T10 = C486 * v[6], T11 = C2828 * v[7], T12 = C486 * v[7];
        REAL T13 = T1 + T2, T14 = T1 - T2, T15 = T8 - T12, T16 = T6 - T10;
        v[0] = (T13 + T3) + (T5 - T15); v[1] = (T13 + T3) - (T5 + T15);
        v[2] = (T13 - T3) + (T16 + T7); v[3] = (T13 - T3) + (T16 - T7);
        v[4] = (T14 + T4) + (T15 + T9); v[5] = (T14 + T4) + (T15 - T9);
        v[6] = (T14 - T4) - (T16 - T11); v[7] = (T14 - T4) - (T16 + T11);
    }
}

/* kind: 0 DCT, 1 Haar, 2 Walsh-Hadamard, 3 biorthogonal 1.5 */
static void FN(tx8)(REAL v[8], int kind, int forward) {
    switch (kind) {
    case 1: FN(haar8)(v, forward); break;
    case 2: FN(wht8)(v); break;
    case 3: FN(bior8)(v, forward); break;
    default: if (forward) FN(dct8_fwd)(v); else FN(dct8_inv)(v);
    }
}

/* One 1-D pass over the group, lane-wise (transform_pack8,
 * cpu_source/source.cpp:423-439). stride 1: along rows within each patch;
 * stride 8: along the patch (group) axis. */
static void FN(pass)(REAL g[64][8], int along_group, int forward, int kind) {
    for (int it = 0; it < 8; ++it) {
        for (int c = 0; c < 8; ++c) {
            REAL v[8];
            for (int k = 0; k < 8; ++k) v[k] = along_group ? g[it + 8 * k][c] : g[it * 8 + k][c];
            FN(tx8)(v, kind, forward);
            for (int k = 0; k < 8; ++k) {
                if (along_group) g[it + 8 * k][c] = v[k]; else g[it * 8 + k][c] = v[k];
            }
        }
    }
}

/* Transpose each 8x8 patch (cpu_source/source.cpp:538-560). */
static void FN(transpose)(REAL g[64][8]) {
    for (int it = 0; it < 8; ++it) {
        for (int a = 0; a < 8; ++a) {
            for (int b = a + 1; b < 8; ++b) {
                REAL t = g[it * 8 + a][b];
                g[it * 8 + a][b] = g[it * 8 + b][a];
                g[it * 8 + b][a] = t;
            }
        }
    }
}

/* 3-D forward / inverse transform in the reference's pass order
 * (cpu_source/source.cpp:596-615, rtc_source/kernel.hpp:664-683): rows,
 * transpose, rows, transpose (transform t2d), then the group (transform t1d). */
static void FN(transform3d)(REAL g[64][8], int forward, int t2d, int t1d) {
    for (int nd = 0; nd < 2; ++nd) {
        FN(pass)(g, 0, forward, t2d);
        FN(transpose)(g);
    }
    FN(pass)(g, 1, forward, t1d);
}

/* Cross-lane sum with the reference's butterfly (reduce_add,
 * cpu_source/source.cpp:97-103): pairs, then quads, then halves. */
static REAL FN(lane_sum)(const REAL x[8]) {
    return ((x[0] + x[1]) + (x[2] + x[3])) + ((x[4] + x[5]) + (x[6] + x[7]));
}

/* SSD of an 8x8 reference block against a candidate block
 * (compute_distance, cpu_source/source.cpp:122-136): per column, two FMA
 * chains over even and odd rows, then the butterfly across columns. */
static REAL FN(ssd)(const REAL ref[8][8], const float *cand, int stride) {
    REAL col[8];
    for (int c = 0; c < 8; ++c) {
        REAL e0 = 0, e1 = 0;
        for (int r = 0; r < 8; ++r) {
            REAL d = ref[r][c] - (REAL)cand[r * stride + c];
            if (r % 2 == 0) e0 = RFMA(d, d, e0); else e1 = RFMA(d, d, e1);
        }
        col[c] = e0 + e1;
    }
    return FN(lane_sum)(col);
}

/* Final-stage lists from the basic stage's (the engine's BASIC_LISTS final
 * matching, no counterpart in the reference): every block's 8 positions
 * [x, y, slot] scored with the reference's block distance against the block
 * at its own origin in the centre plane (planes[radius]) and sorted
 * ascending, ties keeping the basic order (a strict-< insertion, as the
 * reference's list insertion). */
static void FN(rescore)(int *xyz, const float *const *planes, int width, int height,
                        int stride, int block_step, int radius) {
    const int nbx = (width - 8 + block_step - 1) / block_step + 1;
    const int nby = (height - 8 + block_step - 1) / block_step + 1;
    for (int by = 0; by < nby; ++by)
        for (int bx = 0; bx < nbx; ++bx) {
            const int x = bx * block_step < width - 8 ? bx * block_step : width - 8;
            const int y = by * block_step < height - 8 ? by * block_step : height - 8;
            REAL ref[8][8];
            for (int r = 0; r < 8; ++r)
                for (int c = 0; c < 8; ++c)
                    ref[r][c] = (REAL)planes[radius][(size_t)(y + r) * stride + x + c];
            int *l = xyz + ((size_t)by * nbx + bx) * 24;
            REAL d[8];
            int e[8][3], n = 0;
            for (int i = 0; i < 8; ++i) {
                const int *q = l + 3 * i;
                const REAL di = FN(ssd)(ref, planes[q[2]] + (size_t)q[1] * stride + q[0], stride);
                int j = n++;
                for (; j > 0 && di < d[j - 1]; --j) {
                    d[j] = d[j - 1];
                    e[j][0] = e[j - 1][0]; e[j][1] = e[j - 1][1]; e[j][2] = e[j - 1][2];
                }
                d[j] = di;
                e[j][0] = q[0]; e[j][1] = q[1]; e[j][2] = q[2];
            }
            for (int i = 0; i < 8; ++i)
                for (int k = 0; k < 3; ++k) l[3 * i + k] = e[i][k];
        }
}

/* Block distances of the run-time-compiled variant (rtc_source/kernel.hpp:
 * 392-504), lane = column c: metric 1 SAD, 2 ZSSD, 3 ZSAD, 4 SSD/NORM (0 is
 * the SSD above). Per column two accumulators over even and odd rows, then
 * the butterfly across columns; means are the butterfly of the per-column
 * pairwise sums times 1/64. */
static REAL FN(col_tree)(const REAL c[8]) {
    return ((c[0] + c[1]) + (c[2] + c[3])) + ((c[4] + c[5]) + (c[6] + c[7]));
}

static REAL FN(block_error)(int metric, const REAL ref[8][8], const float *cand, int stride) {
    if (metric == 0) return FN(ssd)(ref, cand, stride);
    REAL n[8][8];
    for (int r = 0; r < 8; ++r)
        for (int c = 0; c < 8; ++c) n[r][c] = (REAL)cand[r * stride + c];
    REAL col[8];
    if (metric == 1) {
        for (int c = 0; c < 8; ++c) {
            REAL e0 = 0, e1 = 0;
            for (int r = 0; r < 8; ++r) {
                REAL d = RABS(ref[r][c] - n[r][c]);
                if (r % 2 == 0) e0 = e0 + d; else e1 = e1 + d;
            }
            col[c] = e0 + e1;
        }
        return FN(lane_sum)(col);
    }
    if (metric == 2 || metric == 3) {
        REAL cs[8], ns[8];
        for (int c = 0; c < 8; ++c) {
            REAL a[8], b[8];
            for (int r = 0; r < 8; ++r) { a[r] = ref[r][c]; b[r] = n[r][c]; }
            cs[c] = FN(col_tree)(a);
            ns[c] = FN(col_tree)(b);
        }
        const REAL inv64 = (REAL)(1.0 / 64.0);
        const REAL dm = FN(lane_sum)(cs) * inv64 - FN(lane_sum)(ns) * inv64;
        for (int c = 0; c < 8; ++c) {
            REAL e0 = 0, e1 = 0;
            for (int r = 0; r < 8; ++r) {
                REAL d = (ref[r][c] - n[r][c]) - dm;
                REAL t = metric == 2 ? RFMA(d, d, r % 2 == 0 ? e0 : e1)
                                     : (r % 2 == 0 ? e0 : e1) + RABS(d);
                if (r % 2 == 0) e0 = t; else e1 = t;
            }
            col[c] = e0 + e1;
        }
        return FN(lane_sum)(col);
    }
    /* SSD/NORM: 2 - 2 <a, b> / (|a| |b| + FLT_EPSILON) */
    REAL ca[8], cb[8];
    for (int c = 0; c < 8; ++c) {
        REAL a0 = 0, a1 = 0, b0 = 0, b1 = 0, d0 = 0, d1 = 0;
        for (int r = 0; r < 8; ++r) {
            if (r % 2 == 0) {
                a0 = RFMA(ref[r][c], ref[r][c], a0);
                b0 = RFMA(n[r][c], n[r][c], b0);
                d0 = RFMA(ref[r][c], n[r][c], d0);
            } else {
                a1 = RFMA(ref[r][c], ref[r][c], a1);
                b1 = RFMA(n[r][c], n[r][c], b1);
                d1 = RFMA(ref[r][c], n[r][c], d1);
            }
        }
        ca[c] = a0 + a1;
        cb[c] = b0 + b1;
        col[c] = d0 + d1;
    }
    const REAL na = RSQRT(FN(lane_sum)(ca)), nb = RSQRT(FN(lane_sum)(cb));
    const REAL den = RFMA(na, nb, (REAL)FLT_EPSILON);
    return (REAL)2 - ((REAL)2 * FN(lane_sum)(col)) / den;
}

/* Sorted-list insertion with the reference's lane logic
 * (cpu_source/source.cpp:179-204): lanes whose error exceeds the candidate's
 * take their left neighbour, the new entry lands at lane 8 - count. */
static void FN(list_insert)(REAL err8[8], int ix[8], int iy[8], int iz[8],
                            REAL err, int x, int y, int z) {
    int flag[8], count = 0;
    for (int i = 0; i < 8; ++i) {
        flag[i] = err < err8[i];
        count += flag[i];
    }
    if (!count) return;
    REAL ne[8];
    int nx[8], ny[8], nz[8];
    for (int i = 0; i < 8; ++i) {
        int src = flag[i] ? ((i - 1) & 7) : i;
        ne[i] = err8[src];
        nx[i] = ix[src];
        ny[i] = iy[src];
        nz[i] = iz[src];
    }
    ne[8 - count] = err;
    nx[8 - count] = x;
    ny[8 - count] = y;
    nz[8 - count] = z;
    for (int i = 0; i < 8; ++i) {
        err8[i] = ne[i];
        ix[i] = nx[i];
        iy[i] = ny[i];
        iz[i] = nz[i];
    }
}

/* Exhaustive window search (block_matching, cpu_source/source.cpp:143-215). */
static void FN(block_matching)(REAL err8[8], int ix[8], int iy[8], int iz[8], int z,
                               const REAL ref[8][8], const float *srcp, int stride,
                               int width, int height, int range, int x, int y, int metric) {
    int left = x - range > 0 ? x - range : 0;
    int right = x + range < width - 8 ? x + range : width - 8;
    int top = y - range > 0 ? y - range : 0;
    int bottom = y + range < height - 8 ? y + range : height - 8;
    for (int row = top; row <= bottom; ++row) {
        for (int col = left; col <= right; ++col) {
            REAL e = FN(block_error)(metric, ref, &srcp[row * stride + col], stride);
            FN(list_insert)(err8, ix, iy, iz, e, col, row, z);
        }
    }
}

/* Spatial search in the centre frame followed by the predictive temporal
 * search (block_matching_temporal, cpu_source/source.cpp:220-321). The
 * per-frame list indices start at (0, 0), where the reference leaves them
 * unset; they are only ever read in windows with fewer than ps_num candidates. */
static void FN(block_matching_temporal)(REAL err8[8], int ix[8], int iy[8], int iz[8],
                                        const REAL ref[8][8], const float *const *frames,
                                        int stride, int width, int height, int bm_range,
                                        int x, int y, int radius, int ps_num, int ps_range,
                                        int metric) {
    int center = radius;
    FN(block_matching)(err8, ix, iy, iz, center, ref, frames[center], stride, width, height,
                       bm_range, x, y, metric);
    for (int i = 0; i < 8; ++i) iz[i] = center;
    int cx[8], cy[8];
    for (int i = 0; i < 8; ++i) { cx[i] = ix[i]; cy[i] = iy[i]; }
    for (int dir = -1; dir <= 1; dir += 2) {
        int lx[8], ly[8];
        for (int i = 0; i < 8; ++i) { lx[i] = cx[i]; ly[i] = cy[i]; }
        for (int t = 1; t <= radius; ++t) {
            int z = center + dir * t;
            REAL fe[8];
            int fx[8], fy[8], fz[8];
            for (int i = 0; i < 8; ++i) { fe[i] = (REAL)FLT_MAX; fx[i] = 0; fy[i] = 0; fz[i] = z; }
            for (int i = 0; i < ps_num; ++i)
                FN(block_matching)(fe, fx, fy, fz, z, ref, frames[z], stride, width, height,
                                   ps_range, lx[i], ly[i], metric);
            for (int i = 0; i < ps_num; ++i)
                FN(list_insert)(err8, ix, iy, iz, fe[i], fx[i], fy[i], z);
            for (int i = 0; i < 8; ++i) { lx[i] = fx[i]; ly[i] = fy[i]; }
        }
    }
}

/* Centre insertion (insert_if_not_in[_temporal], cpu_source/source.cpp:325-391). */
static void FN(insert_center)(int ix[8], int iy[8], int iz[8], int x, int y, int z) {
    for (int i = 0; i < 8; ++i)
        if (ix[i] == x && iy[i] == y && iz[i] == z) return;
    for (int i = 7; i > 0; --i) { ix[i] = ix[i - 1]; iy[i] = iy[i - 1]; iz[i] = iz[i - 1]; }
    ix[0] = x; iy[0] = y; iz[0] = z;
}

/* Hard thresholding (cpu_source/source.cpp:562-594). Returns the group weight
 * 1 / (number of kept coefficients); the DC (row 0, lane 0) is always kept. */
static REAL FN(hard_threshold)(REAL g[64][8], REAL sigma) {
    int nnz = 0;
    const REAL scaler = (REAL)(1.0 / 4096.0);
    for (int i = 0; i < 64; ++i) {
        for (int c = 0; c < 8; ++c) {
            REAL thr = (i == 0) ? sigma * (c == 0 ? (REAL)0 : (REAL)1) : sigma;
            REAL v = g[i][c];
            int keep = RABS(v) >= thr;
            nnz += keep;
            g[i][c] = keep ? v * scaler : (REAL)0;
        }
    }
    return (REAL)1 / (REAL)nnz;
}

/* Empirical Wiener shrinkage (cpu_source/source.cpp:617-643). Returns
 * 1 / sum(coeff^2); the DC coefficient is forced to 1. */
static REAL FN(wiener)(REAL g[64][8], const REAL r[64][8], REAL sigma) {
    REAL norm[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    const REAL sqr_sigma = sigma * sigma;
    const REAL scaler = (REAL)(1.0 / 4096.0);
    for (int i = 0; i < 64; ++i) {
        for (int c = 0; c < 8; ++c) {
            REAL sqr_ref = r[i][c] * r[i][c];
            REAL coeff = sqr_ref * ((REAL)1 / (sqr_ref + sqr_sigma));
            if (i == 0 && c == 0) coeff = (REAL)1;
            norm[c] = RFMA(coeff, coeff, norm[c]);
            g[i][c] = (g[i][c] * scaler) * coeff;
        }
    }
    return (REAL)1 / FN(lane_sum)(norm);
}

static void FN(load_group)(REAL g[64][8], const float *const *planes, int stride,
                           const int ix[8], const int iy[8], const int iz[8]) {
    for (int p = 0; p < 8; ++p) {
        const float *src = planes[iz[p]] + (size_t)iy[p] * stride + ix[p];
        for (int r = 0; r < 8; ++r)
            for (int c = 0; c < 8; ++c) g[p * 8 + r][c] = (REAL)src[r * stride + c];
    }
}

/* Accumulation (local_accumulation[_temporal], cpu_source/source.cpp:674-735).
 * extractor == 0: wdst = fma(w, value, wdst), weight += w, as bm3dcpu does.
 * extractor  > 0: each term is pre-rounded as (v + e) - e before a plain add,
 * as the CUDA kernel does for deterministic output (source/kernel.cu:737-750). */
static void FN(accumulate)(REAL *acc, int stride, int height, const REAL g[64][8],
                           const int ix[8], const int iy[8], const int iz[8], REAL w,
                           REAL extractor) {
    for (int p = 0; p < 8; ++p) {
        REAL *wd = acc + (size_t)iz[p] * 2 * height * stride + (size_t)iy[p] * stride + ix[p];
        REAL *wt = wd + (size_t)height * stride;
        for (int r = 0; r < 8; ++r) {
            for (int c = 0; c < 8; ++c) {
                if (extractor > 0) {
                    REAL v = w * g[p * 8 + r][c];
                    v = (v + extractor) - extractor;
                    REAL u = (w + extractor) - extractor;
                    wd[r * stride + c] = wd[r * stride + c] + v;
                    wt[r * stride + c] = wt[r * stride + c] + u;
                } else {
                    wd[r * stride + c] = RFMA(w, g[p * 8 + r][c], wd[r * stride + c]);
                    wt[r * stride + c] = wt[r * stride + c] + w;
                }
            }
        }
    }
}

/*
 * One BM3D call over one temporal window (bm3d<temporal,chroma,final_>,
 * cpu_source/source.cpp:769-911, driven as BM3DGetFrame does,
 * cpu_source/source.cpp:1009-1227).
 *
 * acc: per processed plane (np = chroma ? 3 : 1), [2r+1][2][height][stride]
 *      accumulators, zeroed here. For radius == 0 the slab count is 1.
 * out: radius == 0 only, per plane [height][stride] = wdst * (1 / weight)
 *      (aggregation, cpu_source/source.cpp:738-757); may be NULL.
 * srcps/refps: np * (2r+1) plane pointers, plane-major; refps NULL for basic.
 * sigma: effective (already scaled) sigma per plane.
 * match_in: optional [nblocks][8][3] lists used instead of searching.
 * match_out: optional [nblocks][8][3] lists actually used.
 */
static int FN(bm3d_window)(REAL *const *acc, REAL *const *out, const float *const *srcps,
                           const float *const *refps, int width, int height, int stride,
                           const REAL *sigma, int block_step, int bm_range, int radius,
                           int ps_num, int ps_range, int chroma, REAL extractor,
                           const int *match_in, int *match_out, int metric, int t2d,
                           int t1d) {
    const int np = chroma ? 3 : 1;
    const int tw = 2 * radius + 1;
    const int center = radius;
    const int final_ = refps != NULL;
    const float *const *mplanes = final_ ? refps : srcps;
    for (int p = 0; p < np; ++p)
        memset(acc[p], 0, sizeof(REAL) * (size_t)stride * height * 2 * tw);
    int nb = 0;
    for (int _y = 0; _y < height - 8 + block_step; _y += block_step) {
        int y = _y < height - 8 ? _y : height - 8;
        for (int _x = 0; _x < width - 8 + block_step; _x += block_step, ++nb) {
            int x = _x < width - 8 ? _x : width - 8;
            int ix[8], iy[8], iz[8];
            if (match_in) {
                for (int k = 0; k < 8; ++k) {
                    ix[k] = match_in[(nb * 8 + k) * 3 + 0];
                    iy[k] = match_in[(nb * 8 + k) * 3 + 1];
                    iz[k] = match_in[(nb * 8 + k) * 3 + 2];
                }
            } else {
                REAL ref[8][8];
                const float *rp = mplanes[center] + (size_t)y * stride + x;
                for (int r = 0; r < 8; ++r)
                    for (int c = 0; c < 8; ++c) ref[r][c] = (REAL)rp[r * stride + c];
                REAL err8[8];
                for (int k = 0; k < 8; ++k) { err8[k] = (REAL)FLT_MAX; ix[k] = x; iy[k] = y; iz[k] = center; }
                if (radius > 0)
                    FN(block_matching_temporal)(err8, ix, iy, iz, ref, mplanes, stride, width,
                                                height, bm_range, x, y, radius, ps_num, ps_range,
                                                metric);
                else
                    FN(block_matching)(err8, ix, iy, iz, center, ref, mplanes[0], stride, width,
                                       height, bm_range, x, y, metric);
                FN(insert_center)(ix, iy, iz, x, y, center);
            }
            if (match_out) {
                for (int k = 0; k < 8; ++k) {
                    match_out[(nb * 8 + k) * 3 + 0] = ix[k];
                    match_out[(nb * 8 + k) * 3 + 1] = iy[k];
                    match_out[(nb * 8 + k) * 3 + 2] = iz[k];
                }
            }
            for (int p = 0; p < np; ++p) {
                if (chroma && sigma[p] < (REAL)FLT_EPSILON) continue;
                REAL g[64][8];
                REAL w;
                FN(load_group)(g, srcps + p * tw, stride, ix, iy, iz);
                FN(transform3d)(g, 1, t2d, t1d);
                if (final_) {
                    REAL rg[64][8];
                    FN(load_group)(rg, refps + p * tw, stride, ix, iy, iz);
                    FN(transform3d)(rg, 1, t2d, t1d);
                    w = FN(wiener)(g, (const REAL(*)[8])rg, sigma[p]);
                } else {
                    w = FN(hard_threshold)(g, sigma[p]);
                }
                FN(transform3d)(g, 0, t2d, t1d);
                FN(accumulate)(acc[p], stride, height, (const REAL(*)[8])g, ix, iy, iz, w,
                               extractor);
            }
        }
    }
    if (radius == 0 && out) {
        for (int p = 0; p < np; ++p) {
            if (chroma && sigma[p] < (REAL)FLT_EPSILON) continue;
            const REAL *wd = acc[p];
            const REAL *wt = acc[p] + (size_t)height * stride;
            for (int yy = 0; yy < height; ++yy)
                for (int xx = 0; xx < width; ++xx) {
                    size_t o = (size_t)yy * stride + xx;
                    out[p][o] = AGG_DIVIDE(wd[o], wt[o]);
                }
        }
    }
    return nb;
}

/* VAggregate for output frame n (cpu_source/source.cpp:1507-1544): sums the
 * slabs that frames clamp(n-r .. n+r) hold for frame n, with replication at the
 * clip ends, then divides. vframes: (2r+1) raw outputs [2r+1][2][height][stride]. */
static void FN(vaggregate)(REAL *dst, const REAL *const *vframes, int width, int height,
                           int stride, int radius, int n, int num_frames) {
    REAL *buf = (REAL *)malloc(sizeof(REAL) * 2 * width);
    for (int y = 0; y < height; ++y) {
        for (int x = 0; x < 2 * width; ++x) buf[x] = 0;
        for (int i = 0; i < 2 * radius + 1; ++i) {
            int lo = n - num_frames + 1 + radius, hi = n + radius, s = 2 * radius - i;
            s = s < lo ? lo : (s > hi ? hi : s);
            const REAL *a = vframes[i] + ((size_t)s * 2 * height + y) * stride;
            for (int x = 0; x < width; ++x) buf[x] = buf[x] + a[x];
            a += (size_t)height * stride;
            for (int x = 0; x < width; ++x) buf[width + x] = buf[width + x] + a[x];
        }
        for (int x = 0; x < width; ++x) dst[(size_t)y * stride + x] = buf[x] / buf[width + x];
    }
    free(buf);
}

#undef FN
