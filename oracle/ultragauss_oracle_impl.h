/*
 * TEST INFRASTRUCTURE ONLY — never part of the product path.
 *
 * CPU restatement of the reference UltraGauss renderer (KevinWCCC/ultrasound-3d-
 * reconstruction, ops/ultragauss_renderer), used by the tests as the checker and by the
 * benchmark as the timed CPU baseline. Included twice by ultragauss_oracle.c with
 * REAL = float (suffix _f32, the reference's precision) and REAL = double (suffix _f64,
 * the FP64 oracle). Each function names the reference lines it follows.
 *
 * Differences from the GPU build of the reference that are inherent to a CPU restatement:
 * IEEE division/sqrt/exp instead of the --use_fast_math approximations, and no FMA
 * contraction. Decisions that sit within rounding of a threshold can therefore differ; the
 * window test reports such "ambiguous" pairs so tests can account for them.
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUFFIX)

/* ops/ultragauss_renderer/src/mapper/core.cu:9-44 (compute_probe_bbox_radii). */
static void FN(radii)(const REAL* t, REAL chi2, REAL beta, const REAL* lat, const REAL* ax, const REAL* ele,
                      REAL* r_lat, REAL* r_ax, REAL* r_ele) {
    const REAL l11 = t[0] * t[0] + beta, l12 = t[1], l13 = t[2];
    const REAL l22 = t[3] * t[3] + beta, l23 = t[4], l33 = t[5] * t[5] + beta;
    const REAL d1 = FMAX(l11, (REAL)1e-10), d2 = FMAX(l22, (REAL)1e-10), d3 = FMAX(l33, (REAL)1e-10);
    const REAL* axes[3] = {lat, ax, ele};
    REAL var[3];
    for (int k = 0; k < 3; ++k) {
        const REAL* a = axes[k];
        const REAL y0 = a[0] / d1;
        const REAL y1 = (a[1] - l12 * y0) / d2;
        const REAL y2 = (a[2] - l13 * y0 - l23 * y1) / d3;
        var[k] = FMAX(y0 * y0 + y1 * y1 + y2 * y2, (REAL)1e-12);
    }
    const REAL kk = SQRT(chi2);
    *r_lat = FMAX((REAL)1e-3, kk * SQRT(var[0]));
    *r_ax = FMAX((REAL)1e-3, kk * SQRT(var[1]));
    *r_ele = FMAX((REAL)1e-3, kk * SQRT(var[2]));
}

static inline REAL FN(dot3)(const REAL* a, const REAL* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/*
 * Projection, elevational cull and 16x16 tile rectangles
 * (ops/ultragauss_renderer/src/mapper/core.cu:46-116).
 * geo = origin(3) lat(3) ax(3) ele(3) dlat dax near coloff.
 */
void FN(ugo_project)(int64_t G, const REAL* means, const REAL* tril, const REAL* geo, int H, int W, REAL chi2,
                     REAL beta, int32_t* touched, int32_t* rects, REAL* depths) {
    const REAL *o = geo, *lat = geo + 3, *ax = geo + 6, *ele = geo + 9;
    const REAL dlat = geo[12], dax = geo[13], nearmm = geo[14], coloff = geo[15];
    const int tiles_x = (W + UGO_TILE - 1) / UGO_TILE, tiles_y = (H + UGO_TILE - 1) / UGO_TILE;
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < G; ++g) {
        const REAL* m = means + 3 * g;
        const REAL v[3] = {m[0] - o[0], m[1] - o[1], m[2] - o[2]};
        const REAL l = FN(dot3)(v, lat), e = FN(dot3)(v, ele), a = FN(dot3)(v, ax);
        REAL r_lat, r_ax, r_ele;
        FN(radii)(tril + 6 * g, chi2, beta, lat, ax, ele, &r_lat, &r_ax, &r_ele);
        touched[g] = 0;
        rects[4 * g + 0] = rects[4 * g + 1] = rects[4 * g + 2] = rects[4 * g + 3] = 0;
        depths[g] = 0;
        if (FABS(e) > r_ele) continue;
        const REAL u_pix = l / dlat + coloff;
        const REAL v_pix = (a - nearmm) / dax;
        const REAL r_u = FMAX((REAL)1.0, r_lat / dlat);
        const REAL r_v = FMAX((REAL)1.0, r_ax / dax);
        int x0 = ugo_to_i32_sat((double)FLOOR((u_pix - r_u) / (REAL)UGO_TILE));
        int y0 = ugo_to_i32_sat((double)FLOOR((v_pix - r_v) / (REAL)UGO_TILE));
        int x1 = ugo_to_i32_sat((double)CEIL((u_pix + r_u) / (REAL)UGO_TILE));
        int y1 = ugo_to_i32_sat((double)CEIL((v_pix + r_v) / (REAL)UGO_TILE));
        x0 = x0 > 0 ? x0 : 0;
        y0 = y0 > 0 ? y0 : 0;
        x1 = x1 < tiles_x ? x1 : tiles_x;
        y1 = y1 < tiles_y ? y1 : tiles_y;
        if (x0 >= x1 || y0 >= y1) continue;
        rects[4 * g + 0] = x0;
        rects[4 * g + 1] = y0;
        rects[4 * g + 2] = x1;
        rects[4 * g + 3] = y1;
        depths[g] = v_pix;
        touched[g] = (x1 - x0) * (y1 - y0);
    }
}

/* Keys (tile << 32) | u32((v + 500) * 1000) and values = Gaussian index, emitted Gaussian
 * by Gaussian, tiles row-major (ops/ultragauss_renderer/src/mapper/core.cu:118-143).
 * offsets = exclusive scan of touched (G + 1 entries). */
void FN(ugo_keys)(int64_t G, int tiles_x, int sort_by_depth, const int32_t* rects, const REAL* depths,
                  const int64_t* offsets, uint64_t* keys, int32_t* vals) {
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < G; ++g) {
        int64_t off = offsets[g];
        if (offsets[g + 1] - off <= 0) continue;
        const int32_t* r = rects + 4 * g;
        const uint32_t dk = sort_by_depth ? ugo_to_u32_sat((double)((depths[g] + (REAL)500.0) * (REAL)1000.0)) : 0u;
        for (int y = r[1]; y < r[3]; ++y)
            for (int x = r[0]; x < r[2]; ++x) {
                const uint64_t tile = (uint64_t)(y * tiles_x + x);
                keys[off] = (tile << 32) | dk;
                vals[off] = (int32_t)g;
                ++off;
            }
    }
}

/* Window test of one (pixel, Gaussian) pair (ops/ultragauss_renderer/src/mapper/core.cu:
 * 166-182). *ambiguous is set when a comparison is within 1e-5 relative of its threshold. */
static inline int FN(window_hit)(const REAL* p, const REAL* m, const REAL* t, REAL chi2, REAL beta,
                                 const REAL* lat, const REAL* ax, const REAL* ele, int* ambiguous) {
    REAL r_lat, r_ax, r_ele;
    FN(radii)(t, chi2, beta, lat, ax, ele, &r_lat, &r_ax, &r_ele);
    const REAL d[3] = {p[0] - m[0], p[1] - m[1], p[2] - m[2]};
    const REAL dl = FABS(FN(dot3)(d, lat));
    const REAL da = FABS(FN(dot3)(d, ax));
    const int hit = dl <= r_lat && da <= r_ax;
    if (ambiguous) {
        const double el = fabs((double)dl - (double)r_lat) / ((double)r_lat + 1e-30);
        const double ea = fabs((double)da - (double)r_ax) / ((double)r_ax + 1e-30);
        /* a flip needs one comparison at its threshold and the other one passing */
        *ambiguous = (el < 1e-5 && da <= r_ax * (1 + 1e-5)) || (ea < 1e-5 && dl <= r_lat * (1 + 1e-5));
    }
    return hit;
}

/* Per-pixel candidate counts (core.cu:184-235) and, if out_indices is not NULL, the
 * candidate lists (core.cu:237-287). Pixel p sits in tile (x/16, y/16) of a 16x16 grid;
 * sorted_vals / range_start / range_end are the mapper outputs. ambiguous (optional)
 * receives the number of near-threshold window tests per pixel. */
void FN(ugo_pixel_candidates)(int H, int W, const REAL* pixels, const REAL* means, const REAL* tril,
                              const int32_t* sorted_vals, const int32_t* range_start, const int32_t* range_end,
                              const REAL* geo, REAL chi2, REAL beta, int32_t* counts, const int64_t* offsets,
                              int32_t* out_indices, int32_t* ambiguous) {
    const REAL *lat = geo + 3, *ax = geo + 6, *ele = geo + 9;
    const int grid_w = (W + UGO_TILE - 1) / UGO_TILE;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t p = 0; p < (int64_t)H * W; ++p) {
        const int px = (int)(p % W), py = (int)(p / W);
        const int tile = (py / UGO_TILE) * grid_w + (px / UGO_TILE);
        const int s = range_start[tile], e = range_end[tile];
        int c = 0, amb = 0;
        int64_t wp = offsets ? offsets[p] : 0;
        if (!(s == -1 || s >= e)) {
            for (int i = s; i < e; ++i) {
                const int g = sorted_vals[i];
                int a = 0;
                if (FN(window_hit)(pixels + 3 * p, means + 3 * (int64_t)g, tril + 6 * (int64_t)g, chi2, beta, lat, ax,
                                   ele, ambiguous ? &a : NULL)) {
                    ++c;
                    if (out_indices) out_indices[wp++] = g;
                }
                amb += a;
            }
        }
        if (counts) counts[p] = c;
        if (ambiguous) ambiguous[p] = amb;
    }
}

/* Precision Lambda = L L^T from the raw factor (include/shader/shared.cuh:4-25). */
static inline void FN(precision)(const REAL* t, REAL beta, REAL* S) {
    const REAL l11 = t[0] * t[0] + beta, l12 = t[1], l13 = t[2];
    const REAL l22 = t[3] * t[3] + beta, l23 = t[4], l33 = t[5] * t[5] + beta;
    S[0] = l11 * l11;
    S[1] = l11 * l12;
    S[2] = l11 * l13;
    S[3] = S[1];
    S[4] = l12 * l12 + l22 * l22;
    S[5] = l12 * l13 + l22 * l23;
    S[6] = S[2];
    S[7] = S[5];
    S[8] = l13 * l13 + l23 * l23 + l33 * l33;
}

static inline REAL FN(quad)(const REAL* d, const REAL* S) {
    return (S[0] * d[0] + S[1] * d[1] + S[2] * d[2]) * d[0] + (S[3] * d[0] + S[4] * d[1] + S[5] * d[2]) * d[1] +
           (S[6] * d[0] + S[7] * d[1] + S[8] * d[2]) * d[2];
}

/* Forward shading over the per-pixel CSR (ops/ultragauss_renderer/src/shader/forward.cu:
 * 17-76). attr = (opacity, intensity) per Gaussian (G,2). */
void FN(ugo_forward)(int64_t P, int64_t G, const REAL* attr, const REAL* means, const REAL* tril,
                     const REAL* pixels, const REAL* origin, const REAL* ele, const int64_t* offsets,
                     const int32_t* counts, const int32_t* indices, REAL bg_alpha, REAL bg_intensity, REAL chi2,
                     REAL beta, REAL* image, REAL* alpha, REAL* depth) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t p = 0; p < P; ++p) {
        const REAL* pp = pixels + 3 * p;
        REAL sa = 0, sc = 0, sd = 0;
        for (int k = 0; k < counts[p]; ++k) {
            const int g = indices[offsets[p] + k];
            if (g < 0 || g >= G) continue;
            REAL S[9];
            FN(precision)(tril + 6 * (int64_t)g, beta, S);
            const REAL* m = means + 3 * (int64_t)g;
            const REAL d[3] = {pp[0] - m[0], pp[1] - m[1], pp[2] - m[2]};
            const REAL q = FN(quad)(d, S);
            if (q > chi2) continue;
            const REAL w = EXP((REAL)-0.5 * q);
            const REAL ah = attr[2 * (int64_t)g] * w;
            if (ah <= (REAL)1e-8) continue;
            const REAL mo[3] = {m[0] - origin[0], m[1] - origin[1], m[2] - origin[2]};
            sa += ah;
            sc += ah * attr[2 * (int64_t)g + 1];
            sd += ah * FN(dot3)(mo, ele);
        }
        const REAL at = sa + bg_alpha;
        const REAL num = sc + bg_alpha * bg_intensity;
        REAL im = num / FMAX(at, (REAL)1e-8);
        im = im < 0 ? 0 : (im > 1 ? 1 : im);
        alpha[p] = at;
        image[p] = im;
        depth[p] = sd / FMAX(sa, (REAL)1e-8);
    }
}

/* Backward (ops/ultragauss_renderer/src/shader/backward.cu:17-131). Gradients are
 * accumulated per thread and summed (d_means (G,4) as in the reference, d_tril (G,6),
 * d_attr (G,2)); outputs are overwritten. */
void FN(ugo_backward)(int64_t P, int64_t G, const REAL* dI, const REAL* dA, const REAL* dD, const REAL* attr,
                      const REAL* means, const REAL* tril, const REAL* pixels, const REAL* origin, const REAL* ele,
                      const int64_t* offsets, const int32_t* counts, const int32_t* indices, const REAL* pix_alpha,
                      REAL bg_alpha, REAL bg_intensity, REAL chi2, REAL beta, REAL* d_means, REAL* d_tril,
                      REAL* d_attr) {
    int nt = ugo_max_threads();
    /* per-thread gradient buffers, capped at ~8 GB in total */
    const double per_thread = 12.0 * (double)G * sizeof(REAL);
    if (per_thread * nt > 8e9) nt = (int)(8e9 / per_thread) > 1 ? (int)(8e9 / per_thread) : 1;
    REAL** locals = (REAL**)calloc((size_t)nt, sizeof(REAL*));
#pragma omp parallel num_threads(nt)
    {
        const int tid = ugo_thread_id();
        REAL* lm = (REAL*)calloc((size_t)(12 * G + 1), sizeof(REAL));
        locals[tid] = lm;
        REAL* lt = lm + 4 * G;
        REAL* la = lt + 6 * G;
#pragma omp for schedule(dynamic, 64)
        for (int64_t p = 0; p < P; ++p) {
            const REAL* pp = pixels + 3 * p;
            const int64_t st = offsets[p];
            const int cnt = counts[p];
            const REAL sum_alpha = pix_alpha[p] - bg_alpha;
            REAL sum_c = 0, sum_d = 0;
            for (int k = 0; k < cnt; ++k) {
                const int g = indices[st + k];
                if (g < 0 || g >= G) continue;
                REAL S[9];
                FN(precision)(tril + 6 * (int64_t)g, beta, S);
                const REAL* m = means + 3 * (int64_t)g;
                const REAL d[3] = {pp[0] - m[0], pp[1] - m[1], pp[2] - m[2]};
                const REAL q = FN(quad)(d, S);
                if (q > chi2) continue;
                const REAL w = EXP((REAL)-0.5 * q);
                const REAL ah = attr[2 * (int64_t)g] * w;
                const REAL mo[3] = {m[0] - origin[0], m[1] - origin[1], m[2] - origin[2]};
                sum_c += ah * attr[2 * (int64_t)g + 1];
                sum_d += ah * FN(dot3)(mo, ele);
            }
            const REAL at = sum_alpha + bg_alpha;
            const REAL inv_a = (REAL)1 / FMAX(at, (REAL)1e-8);
            const REAL num = sum_c + bg_alpha * bg_intensity;
            const REAL dnum = dI[p] * inv_a;
            const REAL dat = dA[p] - dI[p] * num * inv_a * inv_a;
            const REAL inv_sa = (REAL)1 / FMAX(sum_alpha, (REAL)1e-8);
            const REAL ddw = dD[p] * inv_sa;
            const REAL dsad = -dD[p] * sum_d * inv_sa * inv_sa;
            for (int k = 0; k < cnt; ++k) {
                const int g = indices[st + k];
                if (g < 0 || g >= G) continue;
                REAL S[9];
                FN(precision)(tril + 6 * (int64_t)g, beta, S);
                const REAL* m = means + 3 * (int64_t)g;
                const REAL o = attr[2 * (int64_t)g], c = attr[2 * (int64_t)g + 1];
                const REAL d[3] = {pp[0] - m[0], pp[1] - m[1], pp[2] - m[2]};
                const REAL q = FN(quad)(d, S);
                if (q > chi2) continue;
                const REAL w = EXP((REAL)-0.5 * q);
                const REAL ah = o * w;
                const REAL mo[3] = {m[0] - origin[0], m[1] - origin[1], m[2] - origin[2]};
                const REAL dterm = FN(dot3)(mo, ele);
                const REAL dah = dnum * c + dat + dsad + ddw * dterm;
                la[2 * g + 1] += dnum * ah;
                la[2 * g + 0] += dah * w;
                const REAL dq = dah * o * w * (REAL)-0.5;
                const REAL v0 = S[0] * d[0] + S[1] * d[1] + S[2] * d[2];
                const REAL v1 = S[3] * d[0] + S[4] * d[1] + S[5] * d[2];
                const REAL v2 = S[6] * d[0] + S[7] * d[1] + S[8] * d[2];
                lm[4 * g + 0] += dq * (-2 * v0) + ddw * ah * ele[0];
                lm[4 * g + 1] += dq * (-2 * v1) + ddw * ah * ele[1];
                lm[4 * g + 2] += dq * (-2 * v2) + ddw * ah * ele[2];
                REAL dS[9];
                for (int i = 0; i < 3; ++i)
                    for (int j = 0; j < 3; ++j) dS[3 * i + j] = dq * d[i] * d[j];
                const REAL* t = tril + 6 * (int64_t)g;
                const REAL l11 = t[0] * t[0] + beta, l12 = t[1], l13 = t[2];
                const REAL l22 = t[3] * t[3] + beta, l23 = t[4], l33 = t[5] * t[5] + beta;
                const REAL dl11 = dS[0] * (2 * l11) + (dS[1] + dS[3]) * l12 + (dS[2] + dS[6]) * l13;
                const REAL dl12 = (dS[1] + dS[3]) * l11 + dS[4] * (2 * l12) + (dS[5] + dS[7]) * l13;
                const REAL dl13 = (dS[2] + dS[6]) * l11 + (dS[5] + dS[7]) * l12 + dS[8] * (2 * l13);
                const REAL dl22 = dS[4] * (2 * l22) + (dS[5] + dS[7]) * l23;
                const REAL dl23 = (dS[5] + dS[7]) * l22 + dS[8] * (2 * l23);
                const REAL dl33 = dS[8] * (2 * l33);
                lt[6 * g + 0] += dl11 * (2 * t[0]);
                lt[6 * g + 1] += dl12;
                lt[6 * g + 2] += dl13;
                lt[6 * g + 3] += dl22 * (2 * t[3]);
                lt[6 * g + 4] += dl23;
                lt[6 * g + 5] += dl33 * (2 * t[5]);
            }
        }
    }
    /* fixed-order reduction over threads */
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < 12 * G; ++i) {
        REAL s = 0;
        for (int t = 0; t < nt; ++t) s += locals[t][i];
        if (i < 4 * G) d_means[i] = s;
        else if (i < 10 * G) d_tril[i - 4 * G] = s;
        else d_attr[i - 10 * G] = s;
    }
    for (int t = 0; t < nt; ++t) free(locals[t]);
    free(locals);
}

#undef FN
#undef CAT
#undef CAT2
