/*
 * TEST INFRASTRUCTURE ONLY — never part of the product path.
 *
 * CPU restatement of the reference GaussianPile projected-slice renderer
 * (KevinWCCC/ultrasound-3d-reconstruction, ops/gaussianplie_renderer) for the configuration
 * its adapter uses: us_focus shader weights, 16x16 tile mapper, additive compositing, no
 * depth order inside a tile. Included twice by gaussianpile_oracle.c with REAL = float
 * (suffix _f32) and REAL = double (suffix _f64).
 */

#define GCAT2(a, b) a##b
#define GCAT(a, b) GCAT2(a, b)
#define GFN(name) GCAT(name, SUFFIX)

typedef struct {
    REAL mu2_lat, mu2_ax, s2_00, s2_01, s2_11, inv00, inv01, inv11, det2;
    REAL sigma_ele, sigma_lat, mu_lat, mu_ax, mu_ele, sc22;
    REAL Lc[9], Se[9];
    REAL r_lat, r_ax;
} GFN(gpo_fp);

typedef struct {
    REAL lat[3], ax[3], ele[3], raw_lat[3], raw_ax[3], raw_ele[3], o[3];
} GFN(gpo_axes);

static inline REAL GFN(gd3)(const REAL* a, const REAL* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* Normalised pose columns 0..2 and translation column 3 (core_tile.cu:51-57). */
static void GFN(gpo_axes_from_pose)(const REAL* P, GFN(gpo_axes) * A) {
    const REAL raw[3][3] = {{P[0], P[4], P[8]}, {P[1], P[5], P[9]}, {P[2], P[6], P[10]}};
    REAL* outs[3] = {A->lat, A->ax, A->ele};
    REAL* raws[3] = {A->raw_lat, A->raw_ax, A->raw_ele};
    for (int k = 0; k < 3; ++k) {
        REAL n = GSQRT(GMAX((REAL)1e-12, GFN(gd3)(raw[k], raw[k])));
        for (int i = 0; i < 3; ++i) {
            raws[k][i] = raw[k][i];
            outs[k][i] = raw[k][i] / n;
        }
    }
    A->o[0] = P[3];
    A->o[1] = P[7];
    A->o[2] = P[11];
}

/* shared.cuh:16-34 (quaternion (w,x,y,z) -> R, normalised) */
static void GFN(gpo_quat)(const REAL* q, REAL* R) {
    const REAL nq = (REAL)1 / GSQRT(GMAX((REAL)1e-12, q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]));
    const REAL w = q[0] * nq, x = q[1] * nq, y = q[2] * nq, z = q[3] * nq;
    R[0] = 1 - 2 * (y * y + z * z);
    R[1] = 2 * (x * y - w * z);
    R[2] = 2 * (x * z + w * y);
    R[3] = 2 * (x * y + w * z);
    R[4] = 1 - 2 * (x * x + z * z);
    R[5] = 2 * (y * z - w * x);
    R[6] = 2 * (x * z - w * y);
    R[7] = 2 * (y * z + w * x);
    R[8] = 1 - 2 * (x * x + y * y);
}

/* us_focus_device.cuh:115-151 */
static int GFN(gpo_inv3)(const REAL* M, REAL* Mi) {
    const REAL c00 = M[4] * M[8] - M[5] * M[7], c01 = M[2] * M[7] - M[1] * M[8], c02 = M[1] * M[5] - M[2] * M[4];
    const REAL c10 = M[5] * M[6] - M[3] * M[8], c11 = M[0] * M[8] - M[2] * M[6], c12 = M[2] * M[3] - M[0] * M[5];
    const REAL c20 = M[3] * M[7] - M[4] * M[6], c21 = M[1] * M[6] - M[0] * M[7], c22 = M[0] * M[4] - M[1] * M[3];
    const REAL det = M[0] * c00 + M[1] * c10 + M[2] * c20;
    if (!(det > (REAL)1e-12) || !isfinite(det)) return 0;
    const REAL id = (REAL)1 / det;
    Mi[0] = c00 * id; Mi[1] = c01 * id; Mi[2] = c02 * id;
    Mi[3] = c10 * id; Mi[4] = c11 * id; Mi[5] = c12 * id;
    Mi[6] = c20 * id; Mi[7] = c21 * id; Mi[8] = c22 * id;
    return 1;
}

static REAL GFN(gpo_clamp)(REAL v, REAL lo, REAL hi) { return GMIN(GMAX(v, lo), hi); }

static REAL GFN(gpo_det_norm)(REAL d, REAL gamma) {
    if (gamma == 0) return 1;
    if (GABS(gamma - (REAL)0.25) < (REAL)1e-7) return (REAL)1 / GSQRT(GSQRT(d));
    if (GABS(gamma - (REAL)0.5) < (REAL)1e-7) return (REAL)1 / GSQRT(d);
    if (GABS(gamma - 1) < (REAL)1e-7) return (REAL)1 / d;
    return GPOW(d, -gamma);
}

/* compute_us_focus_footprint_mm (us_focus_device.cuh:179-316). */
static int GFN(gpo_footprint)(const REAL* m, const REAL* s, const REAL* q, const GFN(gpo_axes) * A, REAL near_mm,
                              REAL k_sigma, const REAL* P, GFN(gpo_fp) * F) {
    const REAL d[3] = {m[0] - A->o[0], m[1] - A->o[1], m[2] - A->o[2]};
    F->mu_lat = GFN(gd3)(d, A->lat);
    F->mu_ax = GFN(gd3)(d, A->ax);
    F->mu_ele = GFN(gd3)(d, A->ele);
    REAL R[9];
    GFN(gpo_quat)(q, R);
    const REAL sc[3] = {GMAX(s[0], (REAL)1e-6), GMAX(s[1], (REAL)1e-6), GMAX(s[2], (REAL)1e-6)};
    REAL Sw[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            Sw[i * 3 + j] = R[i * 3 + 0] * sc[0] * sc[0] * R[j] + R[i * 3 + 1] * sc[1] * sc[1] * R[3 + j] +
                            R[i * 3 + 2] * sc[2] * sc[2] * R[6 + j];
    const REAL* ax3[3] = {A->lat, A->ax, A->ele};
    REAL Sc[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            REAL c[3];
            for (int r = 0; r < 3; ++r) c[r] = Sw[r * 3 + 0] * ax3[j][0] + Sw[r * 3 + 1] * ax3[j][1] + Sw[r * 3 + 2] * ax3[j][2];
            Sc[i * 3 + j] = GFN(gd3)(ax3[i], c);
        }
    Sc[0] += (REAL)1e-6;
    Sc[4] += (REAL)1e-6;
    Sc[8] += (REAL)1e-6;
    if (!GFN(gpo_inv3)(Sc, F->Lc)) return 0;
    const REAL depth = GMAX(F->mu_ax - near_mm, (REAL)0);
    F->sigma_ele = GFN(gpo_clamp)(P[0] + P[1] * depth, P[2], P[3]);
    F->sigma_lat = GFN(gpo_clamp)(P[4] + P[5] * depth, P[6], P[7]);
    REAL Le[9];
    for (int i = 0; i < 9; ++i) Le[i] = F->Lc[i];
    if (P[11] != 0) Le[0] += (REAL)1 / GMAX(F->sigma_lat * F->sigma_lat, (REAL)1e-12);
    Le[8] += (REAL)1 / GMAX(F->sigma_ele * F->sigma_ele, (REAL)1e-12);
    if (!GFN(gpo_inv3)(Le, F->Se)) return 0;
    const REAL mc[3] = {F->mu_lat, F->mu_ax, F->mu_ele};
    REAL t[3];
    for (int r = 0; r < 3; ++r) t[r] = F->Lc[r * 3] * mc[0] + F->Lc[r * 3 + 1] * mc[1] + F->Lc[r * 3 + 2] * mc[2];
    F->mu2_lat = F->Se[0] * t[0] + F->Se[1] * t[1] + F->Se[2] * t[2];
    F->mu2_ax = F->Se[3] * t[0] + F->Se[4] * t[1] + F->Se[5] * t[2];
    const REAL il = GMAX(P[12], (REAL)0), ia = GMAX(P[13], (REAL)0);
    F->s2_00 = F->Se[0] + il * il;
    F->s2_01 = (REAL)0.5 * (F->Se[1] + F->Se[3]);
    F->s2_11 = F->Se[4] + ia * ia;
    F->det2 = F->s2_00 * F->s2_11 - F->s2_01 * F->s2_01;
    if (!(F->det2 > P[9]) || !isfinite(F->det2)) return 0;
    const REAL idet = (REAL)1 / F->det2;
    F->inv00 = F->s2_11 * idet;
    F->inv01 = -F->s2_01 * idet;
    F->inv11 = F->s2_00 * idet;
    F->sc22 = Sc[8];
    const REAL cross = GABS(F->s2_01);
    F->r_lat = k_sigma * GSQRT(GMAX(F->s2_00 + cross, (REAL)1e-12));
    F->r_ax = k_sigma * GSQRT(GMAX(F->s2_11 + cross, (REAL)1e-12));
    return 1;
}

/* Tile rectangles (core_tile.cu:124-173); zero depth keys; touched counts.
 * grid: slice grid pack (16). */
void GFN(gpo_mapper)(int64_t G, const REAL* means, const REAL* scales, const REAL* quats, const REAL* pose,
                     const REAL* grid, const REAL* params, int H, int W, REAL lat_mm, REAL ax_mm, REAL near_mm,
                     int tile, REAL k_sigma, int32_t* rects, int32_t* touched) {
    GFN(gpo_axes) A;
    GFN(gpo_axes_from_pose)(pose, &A);
    const int tx = (W + tile - 1) / tile, ty = (H + tile - 1) / tile;
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < G; ++g) {
        GFN(gpo_fp) F;
        int32_t* r = rects + 4 * g;
        r[0] = r[1] = r[2] = r[3] = 0;
        touched[g] = 0;
        if (!GFN(gpo_footprint)(means + 3 * g, scales + 3 * g, quats + 4 * g, &A, near_mm, k_sigma, params, &F)) continue;
        const REAL u = F.mu2_lat / lat_mm + grid[6];
        const REAL v = (F.mu2_ax - near_mm) / ax_mm;
        const REAL rl = GMAX((REAL)1, F.r_lat / GMAX((REAL)1e-8, lat_mm));
        const REAL ra = GMAX((REAL)1, F.r_ax / GMAX((REAL)1e-8, ax_mm));
        const REAL ts = (REAL)tile;
        int x0 = gpo_to_i32((double)GFLOOR((u - rl) / ts)), y0 = gpo_to_i32((double)GFLOOR((v - ra) / ts));
        int x1 = gpo_to_i32((double)GCEIL((u + rl) / ts)), y1 = gpo_to_i32((double)GCEIL((v + ra) / ts));
        x0 = x0 > 0 ? x0 : 0;
        y0 = y0 > 0 ? y0 : 0;
        x1 = x1 < tx ? x1 : tx;
        y1 = y1 < ty ? y1 : ty;
        if (x0 >= x1 || y0 >= y1) continue;
        r[0] = x0; r[1] = y0; r[2] = x1; r[3] = y1;
        touched[g] = (x1 - x0) * (y1 - y0);
    }
}

/* Per-tile lists in the reference's order (stable sort of (tile << 32) keys emitted
 * Gaussian by Gaussian = ascending Gaussian index within a tile) and ranges. */
void GFN(gpo_tile_lists)(int64_t G, const int32_t* rects, int tiles_x, int n_tiles, int32_t* range_start,
                         int32_t* range_end, int32_t* sorted_ids) {
    int64_t* cnt = (int64_t*)calloc((size_t)n_tiles + 1, sizeof(int64_t));
    for (int64_t g = 0; g < G; ++g) {
        const int32_t* r = rects + 4 * g;
        for (int y = r[1]; y < r[3]; ++y)
            for (int x = r[0]; x < r[2]; ++x) cnt[y * tiles_x + x + 1]++;
    }
    for (int t = 0; t < n_tiles; ++t) cnt[t + 1] += cnt[t];
    for (int t = 0; t < n_tiles; ++t) {
        range_start[t] = cnt[t + 1] > cnt[t] ? (int32_t)cnt[t] : -1;
        range_end[t] = cnt[t + 1] > cnt[t] ? (int32_t)cnt[t + 1] : -1;
    }
    int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)n_tiles);
    for (int t = 0; t < n_tiles; ++t) cur[t] = cnt[t];
    for (int64_t g = 0; g < G; ++g) {
        const int32_t* r = rects + 4 * g;
        for (int y = r[1]; y < r[3]; ++y)
            for (int x = r[0]; x < r[2]; ++x) sorted_ids[cur[y * tiles_x + x]++] = (int32_t)g;
    }
    free(cur);
    free(cnt);
}

/* Additive forward (forward.cu:27-210): per pixel, over its tile's list in order. */
void GFN(gpo_forward)(int64_t G, const REAL* means, const REAL* scales, const REAL* quats, const REAL* opac,
                      const REAL* inten, const REAL* pose, const REAL* grid, const REAL* params, int H, int W, int tile,
                      REAL k_sigma, const int32_t* range_start, const int32_t* range_end, const int32_t* sorted_ids,
                      REAL* image) {
    GFN(gpo_axes) A;
    GFN(gpo_axes_from_pose)(pose, &A);
    const int tx = (W + tile - 1) / tile;
    /* per-Gaussian candidate (the reference recomputes it per tile; values are identical) */
    REAL* cand = (REAL*)malloc(sizeof(REAL) * 10 * (size_t)(G > 0 ? G : 1));
#pragma omp parallel for schedule(static)
    for (int64_t g = 0; g < G; ++g) {
        GFN(gpo_fp) F;
        REAL* c = cand + 10 * g;
        c[9] = 0;
        if (!GFN(gpo_footprint)(means + 3 * g, scales + 3 * g, quats + 4 * g, &A, grid[5], k_sigma, params, &F)) continue;
        const REAL de = GMAX(F.sc22 + F.sigma_ele * F.sigma_ele + params[9], (REAL)1e-12);
        const REAL sr = GEXP((REAL)-0.5 * F.mu_ele * F.mu_ele / de);
        const REAL bw = opac[g] * sr * GFN(gpo_det_norm)(F.det2 + params[9], params[8]);
        if (!isfinite(bw)) continue;
        c[0] = bw; c[1] = inten[g]; c[2] = F.mu2_lat; c[3] = F.mu2_ax; c[4] = F.inv00; c[5] = F.inv01;
        c[6] = F.inv11; c[7] = F.r_lat; c[8] = F.r_ax; c[9] = 1;
    }
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t p = 0; p < (int64_t)H * W; ++p) {
        const int x = (int)(p % W), y = (int)(p / W);
        const int t = (y / tile) * tx + x / tile;
        const REAL xl = ((REAL)x - grid[6]) * grid[3];
        const REAL xa = (REAL)y * grid[4] + grid[5];
        REAL acc = 0;
        const int s = range_start[t], e = range_end[t];
        if (s >= 0 && e > s)
            for (int i = s; i < e; ++i) {
                const REAL* c = cand + 10 * (int64_t)sorted_ids[i];
                if (c[9] == 0) continue;
                if (GABS(xl - c[2]) > c[7] || GABS(xa - c[3]) > c[8]) continue;
                const REAL dl = xl - c[2], da = xa - c[3];
                const REAL quad = dl * (c[4] * dl + c[5] * da) + da * (c[5] * dl + c[6] * da);
                if (!(quad >= 0) || !isfinite(quad)) continue;
                const REAL w = c[0] * GEXP((REAL)-0.5 * quad);
                if (!isfinite(w) || w < params[10]) continue;
                acc += c[1] * w;
            }
        image[p] = acc;
    }
    free(cand);
}

static REAL GFN(gpo_sanitize)(REAL g) {
    if (!isfinite(g)) return 0;
    if (GABS(g) > (REAL)1e3) return g > 0 ? (REAL)1e3 : (REAL)-1e3;
    return g;
}

static void GFN(gpo_inv3_bwd)(const REAL* Inv, const REAL* gI, REAL* gM) {
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) {
            REAL acc = 0;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) acc += Inv[a * 3 + r] * gI[a * 3 + b] * Inv[c * 3 + b];
            gM[r * 3 + c] -= acc;
        }
}

static REAL GFN(gpo_fp_dot)(const GFN(gpo_fp) * F, const REAL* a) {
    return a[0] * F->mu2_lat + a[1] * F->mu2_ax + a[2] * F->inv00 + a[3] * F->inv01 + a[4] * F->inv11 + a[5] * F->det2 +
           a[6] * F->mu_ele + a[7] * F->sc22 + a[8] * F->sigma_ele;
}

/* Backward (us_focus.cu:398-966): per (tile, Gaussian) sufficient statistics over the
 * footprint's pixels inside the tile, summed per Gaussian in tile order, then the
 * per-Gaussian finalize (chain rule through Se/Lc, finite-difference shape gradients with
 * step 1e-3, sanitising) and the pose gradient. d_pose is (16,) row-major. */
void GFN(gpo_backward)(int64_t G, const REAL* means, const REAL* scales, const REAL* quats, const REAL* opac,
                       const REAL* inten, const REAL* pose, const REAL* grid, const REAL* params, int H, int W,
                       int tile, REAL k_sigma, const int32_t* rects, const int32_t* range_start,
                       const int32_t* range_end, const int32_t* sorted_ids, const REAL* grad_image, int pose_grad,
                       REAL* d_means, REAL* d_scales, REAL* d_quats, REAL* d_opac, REAL* d_inten, REAL* d_pose) {
    GFN(gpo_axes) A;
    GFN(gpo_axes_from_pose)(pose, &A);
    const int tx = (W + tile - 1) / tile, ty = (H + tile - 1) / tile;
    const REAL near_mm = grid[5], lat_d = grid[3], ax_d = grid[4], col_off = grid[6];
    const REAL det_eps = params[9], gamma = params[8], wmin = params[10];
    enum { NS = 19 };
    REAL* acc = (REAL*)calloc((size_t)NS * (size_t)(G > 0 ? G : 1), sizeof(REAL));
    /* tiles in order; each Gaussian's statistics accumulate in tile order */
    for (int t = 0; t < tx * ty; ++t) {
        const int s = range_start[t], e = range_end[t];
        if (s < 0 || e <= s) continue;
        const int x0 = (t % tx) * tile, y0 = (t / tx) * tile;
        const int x1 = x0 + tile < W ? x0 + tile : W, y1 = y0 + tile < H ? y0 + tile : H;
#pragma omp parallel for schedule(dynamic, 16)
        for (int i = s; i < e; ++i) {
            const int g = sorted_ids[i];
            GFN(gpo_fp) F;
            if (!GFN(gpo_footprint)(means + 3 * g, scales + 3 * g, quats + 4 * g, &A, near_mm, k_sigma, params, &F)) continue;
            int cx0 = gpo_to_i32((double)GCEIL((F.mu2_lat - F.r_lat) / lat_d + col_off));
            int cx1 = gpo_to_i32((double)GFLOOR((F.mu2_lat + F.r_lat) / lat_d + col_off)) + 1;
            int cy0 = gpo_to_i32((double)GCEIL((F.mu2_ax - F.r_ax - near_mm) / ax_d));
            int cy1 = gpo_to_i32((double)GFLOOR((F.mu2_ax + F.r_ax - near_mm) / ax_d)) + 1;
            cx0 = cx0 > x0 ? cx0 : x0; cx1 = cx1 < x1 ? cx1 : x1;
            cy0 = cy0 > y0 ? cy0 : y0; cy1 = cy1 < y1 ? cy1 : y1;
            const REAL o = opac[g], c = inten[g];
            const REAL de = GMAX(F.sc22 + F.sigma_ele * F.sigma_ele + det_eps, (REAL)1e-12);
            const REAL sr = GEXP((REAL)-0.5 * F.mu_ele * F.mu_ele / de);
            const REAL nf = GFN(gpo_det_norm)(F.det2 + det_eps, gamma);
            const REAL depth = GMAX(F.mu_ax - near_mm, (REAL)0);
            const REAL se_raw = params[0] + params[1] * depth;
            const REAL dse = (F.mu_ax > near_mm && se_raw > params[2] && se_raw < params[3]) ? params[1] : 0;
            const REAL idn = (REAL)1 / GMAX(F.det2 + det_eps, (REAL)1e-12);
            const REAL ide = (REAL)1 / de;
            REAL a[NS];
            for (int k = 0; k < NS; ++k) a[k] = 0;
            for (int y = cy0; y < cy1; ++y) {
                const REAL xa = (REAL)y * ax_d + near_mm;
                for (int x = cx0; x < cx1; ++x) {
                    const REAL xl = ((REAL)x - col_off) * lat_d;
                    if (GABS(xl - F.mu2_lat) > F.r_lat || GABS(xa - F.mu2_ax) > F.r_ax) continue;
                    const REAL dl = xl - F.mu2_lat, da = xa - F.mu2_ax;
                    const REAL ql = F.inv00 * dl + F.inv01 * da, qa = F.inv01 * dl + F.inv11 * da;
                    const REAL quad = dl * ql + da * qa;
                    if (!(quad >= 0) || !isfinite(quad)) continue;
                    const REAL bno = sr * nf * GEXP((REAL)-0.5 * quad);
                    const REAL w = o * bno;
                    if (!isfinite(w) || w < wmin) continue;
                    const REAL up = grad_image[(int64_t)y * W + x];
                    const REAL gw = up * c, cm = gw * w;
                    a[9] += up * w;        /* intensity */
                    a[8] += gw * bno;      /* opacity */
                    a[3] += cm * ql;       /* mu_e sum (lat) */
                    a[4] += cm * qa;       /* mu_e sum (ax) */
                    a[10] += cm * ql;      /* adjoint: mu2_lat */
                    a[11] += cm * qa;      /* mu2_ax */
                    a[12] += cm * ((REAL)-0.5 * dl * dl);
                    a[13] += cm * (-dl * da);
                    a[14] += cm * ((REAL)-0.5 * da * da);
                    a[15] += cm * (-gamma * idn);
                    a[5] += cm * ((REAL)0.5 * ql * ql - gamma * F.s2_11 * idn);
                    a[6] += (REAL)0.5 * (cm * (ql * qa + 2 * gamma * F.s2_01 * idn));
                    a[7] += cm * ((REAL)0.5 * qa * qa - gamma * F.s2_00 * idn);
                    a[1] += cm * (-F.mu_ele * ide);
                    a[2] += cm * ((REAL)0.5 * F.mu_ele * F.mu_ele * ide * ide);
                    a[0] += cm * (F.mu_ele * F.mu_ele * dse * ide * ide);
                    a[16] += cm * (-F.mu_ele * ide);
                    a[17] += cm * ((REAL)0.5 * F.mu_ele * F.mu_ele * ide * ide);
                    a[18] += cm * (F.mu_ele * F.mu_ele * F.sigma_ele * ide * ide);
                }
            }
            REAL* dst = acc + (int64_t)NS * g;
            for (int k = 0; k < NS; ++k) dst[k] += a[k];
        }
    }
    for (int i = 0; i < 16; ++i) d_pose[i] = 0;
    memset(d_means, 0, sizeof(REAL) * 3 * G);
    memset(d_scales, 0, sizeof(REAL) * 3 * G);
    memset(d_quats, 0, sizeof(REAL) * 4 * G);
    memset(d_opac, 0, sizeof(REAL) * G);
    memset(d_inten, 0, sizeof(REAL) * G);
    REAL* pose_part = (REAL*)calloc((size_t)12 * (size_t)(G > 0 ? G : 1), sizeof(REAL));
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t g = 0; g < G; ++g) {
        const int32_t* r = rects + 4 * g;
        if (r[0] >= r[2] || r[1] >= r[3]) continue;
        const REAL* m = means + 3 * g;
        const REAL* s = scales + 3 * g;
        const REAL* q = quats + 4 * g;
        GFN(gpo_fp) F;
        if (!GFN(gpo_footprint)(m, s, q, &A, near_mm, k_sigma, params, &F)) continue;
        const REAL* a = acc + (int64_t)NS * g;
        const REAL depth = GMAX(F.mu_ax - near_mm, (REAL)0);
        const int active = F.mu_ax > near_mm;
        const REAL se_raw = params[0] + params[1] * depth, sl_raw = params[4] + params[5] * depth;
        const int use_lat = params[11] != 0;
        const REAL dse = (active && se_raw > params[2] && se_raw < params[3]) ? params[1] : 0;
        const REAL dsl = (use_lat && active && sl_raw > params[6] && sl_raw < params[7]) ? params[5] : 0;
        const REAL dle = -2 * dse / GMAX(F.sigma_ele * F.sigma_ele * F.sigma_ele, (REAL)1e-12);
        const REAL dll = use_lat ? -2 * dsl / GMAX(F.sigma_lat * F.sigma_lat * F.sigma_lat, (REAL)1e-12) : 0;
        const REAL mc[3] = {F.mu_lat, F.mu_ax, F.mu_ele};
        REAL gmp[3] = {0, a[0], a[1]};
        REAL gSc[9] = {0, 0, 0, 0, 0, 0, 0, 0, a[2]};
        const REAL gme[3] = {a[3], a[4], 0};
        REAL gSe[9] = {a[5], a[6], 0, a[6], a[7], 0, 0, 0, 0};
        REAL ylc[3], gy[3], gLc[9], gLe[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = 0; i < 3; ++i) ylc[i] = F.Lc[i * 3] * mc[0] + F.Lc[i * 3 + 1] * mc[1] + F.Lc[i * 3 + 2] * mc[2];
        for (int i = 0; i < 3; ++i) gy[i] = F.Se[i] * gme[0] + F.Se[3 + i] * gme[1] + F.Se[6 + i] * gme[2];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) gLc[i * 3 + j] = gy[i] * mc[j];
        for (int i = 0; i < 3; ++i) gmp[i] += F.Lc[i] * gy[0] + F.Lc[3 + i] * gy[1] + F.Lc[6 + i] * gy[2];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) gSe[i * 3 + j] += gme[i] * ylc[j];
        GFN(gpo_inv3_bwd)(F.Se, gSe, gLe);
        for (int i = 0; i < 9; ++i) gLc[i] += gLe[i];
        gmp[1] += gLe[0] * dll + gLe[8] * dle;
        GFN(gpo_inv3_bwd)(F.Lc, gLc, gSc);
        d_inten[g] = GFN(gpo_sanitize)(a[9]);
        d_opac[g] = GFN(gpo_sanitize)(a[8]);
        const REAL* adj = a + 10;
        for (int k = 0; k < 7; ++k) {
            REAL sp[3] = {s[0], s[1], s[2]}, sm[3] = {s[0], s[1], s[2]};
            REAL qp[4] = {q[0], q[1], q[2], q[3]}, qm[4] = {q[0], q[1], q[2], q[3]};
            const REAL eps = (REAL)1e-3;
            if (k < 3) { sp[k] += eps; sm[k] -= eps; } else { qp[k - 3] += eps; qm[k - 3] -= eps; }
            GFN(gpo_fp) Fp, Fm;
            const REAL lp = GFN(gpo_footprint)(m, sp, qp, &A, near_mm, k_sigma, params, &Fp) ? GFN(gpo_fp_dot)(&Fp, adj) : 0;
            const REAL lm = GFN(gpo_footprint)(m, sm, qm, &A, near_mm, k_sigma, params, &Fm) ? GFN(gpo_fp_dot)(&Fm, adj) : 0;
            const REAL fd = GFN(gpo_sanitize)((lp - lm) / (2 * eps));
            if (k < 3) d_scales[3 * g + k] = fd; else d_quats[4 * g + k - 3] = fd;
        }
        REAL gd[3];
        for (int i = 0; i < 3; ++i) gd[i] = gmp[0] * A.lat[i] + gmp[1] * A.ax[i] + gmp[2] * A.ele[i];
        for (int i = 0; i < 3; ++i) d_means[3 * g + i] = GFN(gpo_sanitize)(gd[i]);
        if (!pose_grad) continue;
        REAL R[9], Sw[9];
        GFN(gpo_quat)(q, R);
        const REAL sc[3] = {GMAX(s[0], (REAL)1e-6), GMAX(s[1], (REAL)1e-6), GMAX(s[2], (REAL)1e-6)};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j)
                Sw[i * 3 + j] = R[i * 3] * sc[0] * sc[0] * R[j] + R[i * 3 + 1] * sc[1] * sc[1] * R[3 + j] +
                                R[i * 3 + 2] * sc[2] * sc[2] * R[6 + j];
        const REAL* axs[3] = {A.lat, A.ax, A.ele};
        const REAL* raws[3] = {A.raw_lat, A.raw_ax, A.raw_ele};
        REAL ga[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                REAL Sai[3], Saj[3];
                for (int rr = 0; rr < 3; ++rr) {
                    Sai[rr] = Sw[rr * 3] * axs[i][0] + Sw[rr * 3 + 1] * axs[i][1] + Sw[rr * 3 + 2] * axs[i][2];
                    Saj[rr] = Sw[rr * 3] * axs[j][0] + Sw[rr * 3 + 1] * axs[j][1] + Sw[rr * 3 + 2] * axs[j][2];
                }
                for (int rr = 0; rr < 3; ++rr) {
                    ga[i][rr] += gSc[i * 3 + j] * Saj[rr];
                    ga[j][rr] += gSc[i * 3 + j] * Sai[rr];
                }
            }
        const REAL dw[3] = {m[0] - A.o[0], m[1] - A.o[1], m[2] - A.o[2]};
        REAL* pp = pose_part + 12 * g;
        for (int k = 0; k < 3; ++k) {
            REAL gv[3];
            for (int rr = 0; rr < 3; ++rr) gv[rr] = gmp[k] * dw[rr] + ga[k][rr];
            const REAL len = GSQRT(GMAX((REAL)1e-12, GFN(gd3)(raws[k], raws[k])));
            const REAL dn = GFN(gd3)(axs[k], gv);
            for (int rr = 0; rr < 3; ++rr) pp[3 * k + rr] = (gv[rr] - axs[k][rr] * dn) / len;
        }
        for (int rr = 0; rr < 3; ++rr) pp[9 + rr] = -gd[rr];
    }
    if (pose_grad) {
        const int idx[12] = {0, 4, 8, 1, 5, 9, 2, 6, 10, 3, 7, 11};
        for (int64_t g = 0; g < G; ++g)
            for (int k = 0; k < 12; ++k) d_pose[idx[k]] += pose_part[12 * g + k];
    }
    free(pose_part);
    free(acc);
}

#undef GFN
#undef GCAT
#undef GCAT2
