/*
 * TEST INFRASTRUCTURE ONLY — never part of the product path.
 *
 * CPU restatement of the reference UltraGS-baseline surfel rasteriser (KevinWCCC/
 * ultrasound-3d-reconstruction, ops/ultrags_baseline_renderer/cuda_rasterizer). Included
 * twice by surfel_oracle.c with REAL = float (suffix _f32) and REAL = double (suffix _f64).
 * Matrices are column-major (m[c*R + r]) as in the GLM code the reference uses, and the
 * products sum k ascending. IEEE arithmetic (no FMA contraction, exact division, libm exp)
 * instead of the reference's fast-math build, so decisions within rounding of a threshold
 * can differ.
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUFFIX)

/* (C1 x R1) * (C2 x C1) column-major product */
static void FN(mmul)(const REAL* a, int C1, int R1, const REAL* b, int C2, REAL* o) {
    for (int c = 0; c < C2; ++c)
        for (int r = 0; r < R1; ++r) {
            REAL acc = a[0 * R1 + r] * b[c * C1 + 0];
            for (int k = 1; k < C1; ++k) acc = acc + a[k * R1 + r] * b[c * C1 + k];
            o[c * R1 + r] = acc;
        }
}

static void FN(transp)(const REAL* a, int C, int R, REAL* o) {
    for (int c = 0; c < C; ++c)
        for (int r = 0; r < R; ++r) o[r * C + c] = a[c * R + r];
}

/* cuda_rasterizer/auxiliary.h:199-222 */
static void FN(quat_rot)(const REAL* q, REAL* R) {
    const REAL s = 1 / SQRT(q[3] * q[3] + q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    const REAL w = q[0] * s, x = q[1] * s, y = q[2] * s, z = q[3] * s;
    R[0] = 1 - 2 * (y * y + z * z); R[1] = 2 * (x * y + w * z); R[2] = 2 * (x * z - w * y);
    R[3] = 2 * (x * y - w * z); R[4] = 1 - 2 * (x * x + z * z); R[5] = 2 * (y * z + w * x);
    R[6] = 2 * (x * z + w * y); R[7] = 2 * (y * z - w * x); R[8] = 1 - 2 * (x * x + y * y);
}

/* auxiliary.h:225-271; g column-major dL/dR */
static void FN(quat_rot_vjp)(const REAL* q, const REAL* g, REAL* o) {
    const REAL s = 1 / SQRT(q[3] * q[3] + q[0] * q[0] + q[1] * q[1] + q[2] * q[2]);
    const REAL w = q[0] * s, x = q[1] * s, y = q[2] * s, z = q[3] * s;
#define G(c, r) g[(c) * 3 + (r)]
    o[0] = 2 * (x * (G(1, 2) - G(2, 1)) + y * (G(2, 0) - G(0, 2)) + z * (G(0, 1) - G(1, 0)));
    o[1] = 2 * (-2 * x * (G(1, 1) + G(2, 2)) + y * (G(0, 1) + G(1, 0)) + z * (G(0, 2) + G(2, 0)) + w * (G(1, 2) - G(2, 1)));
    o[2] = 2 * (x * (G(0, 1) + G(1, 0)) - 2 * y * (G(0, 0) + G(2, 2)) + z * (G(1, 2) + G(2, 1)) + w * (G(2, 0) - G(0, 2)));
    o[3] = 2 * (x * (G(0, 2) + G(2, 0)) + y * (G(1, 2) + G(2, 1)) - 2 * z * (G(0, 0) + G(1, 1)) + w * (G(0, 1) - G(1, 0)));
#undef G
}

static REAL FN(dot3)(const REAL* a, const REAL* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* T = transpose(S2W) * W2N * N2P (forward.cu:69-107) or, with assoc_right, the backward's
 * transpose(S2W) * (W2N * N2P) (backward.cu:440-465); also returns L and P (= W2N * N2P). */
static void FN(homography)(const REAL* q, REAL sx, REAL sy, REAL mod, const REAL* p, const REAL* pm, int W, int H,
                           int assoc_right, REAL* T, REAL* R, REAL* L, REAL* Pout) {
    REAL S[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    S[0] = mod * sx;
    S[4] = mod * sy;
    FN(quat_rot)(q, R);
    FN(mmul)(R, 3, 3, S, 3, L);
    REAL s2w[12] = {L[0], L[1], L[2], 0, L[3], L[4], L[5], 0, p[0], p[1], p[2], 1};
    REAL w2n[16], n2p[12] = {(REAL)W / 2, 0, 0, (REAL)(W - 1) / 2, 0, (REAL)H / 2, 0, (REAL)(H - 1) / 2, 0, 0, 0, 1};
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r) w2n[c * 4 + r] = pm[4 * r + c];
    REAL t43[12];
    FN(transp)(s2w, 3, 4, t43);
    if (!assoc_right) {
        REAL A[12];
        FN(mmul)(t43, 4, 3, w2n, 4, A);
        FN(mmul)(A, 4, 3, n2p, 3, T);
    } else {
        REAL Pm[12];
        FN(mmul)(w2n, 4, 4, n2p, 3, Pm);
        FN(mmul)(t43, 4, 3, Pm, 3, T);
        if (Pout)
            for (int i = 0; i < 12; ++i) Pout[i] = Pm[i];
    }
}

static void FN(xform_point)(const REAL* p, const REAL* m, REAL* o) {
    o[0] = m[0] * p[0] + m[4] * p[1] + m[8] * p[2] + m[12];
    o[1] = m[1] * p[0] + m[5] * p[1] + m[9] * p[2] + m[13];
    o[2] = m[2] * p[0] + m[6] * p[1] + m[10] * p[2] + m[14];
}
static void FN(xform_vec)(const REAL* p, const REAL* m, REAL* o) {
    o[0] = m[0] * p[0] + m[4] * p[1] + m[8] * p[2];
    o[1] = m[1] * p[0] + m[5] * p[1] + m[9] * p[2];
    o[2] = m[2] * p[0] + m[6] * p[1] + m[10] * p[2];
}

typedef struct {
    int P, D, M, W, H;
    REAL scale_modifier;
    const REAL *means, *shs, *colors, *opac, *scales, *rots, *transmat;
    const REAL *view, *proj;
    const REAL *campos, *bg;
} FN(GsIn);

/* Per-Gaussian preprocess (forward.cu:141-246). rec per Gaussian: T (9, column-major),
 * xy (2), normal (3), opacity, rgb (3), depth, clamped bits -> 20 REAL. */
#ifndef GSO_REC
#define GSO_REC 20
#endif

static void FN(preprocess)(const FN(GsIn) * in, int g, int* radius_out, int* rect, REAL* rec) {
    const int gx = (in->W + 15) / 16, gy = (in->H + 15) / 16;
    *radius_out = 0;
    rect[0] = rect[1] = rect[2] = rect[3] = 0;
    const REAL* po = in->means + 3 * (int64_t)g;
    REAL pv[3];
    FN(xform_point)(po, in->view, pv);
    if (pv[2] <= (REAL)0.2f) return;
    REAL T[9], R[9], L[9], n[3];
    if (!in->transmat) {
        FN(homography)(in->rots + 4 * (int64_t)g, in->scales[2 * g], in->scales[2 * g + 1], in->scale_modifier, po,
                       in->proj, in->W, in->H, 0, T, R, L, NULL);
        FN(xform_vec)(L + 6, in->view, n);
    } else {
        for (int i = 0; i < 9; ++i) T[i] = in->transmat[9 * (int64_t)g + i];
        n[0] = 0; n[1] = 0; n[2] = 1;
    }
    const REAL cosv = -(pv[0] * n[0] + pv[1] * n[1] + pv[2] * n[2]);
    if (cosv == 0) return;
    const REAL mult = cosv > 0 ? 1 : -1;
    for (int i = 0; i < 3; ++i) n[i] *= mult;
    const REAL t[3] = {9, 9, -1};
    const REAL *T0 = T, *T1 = T + 3, *T2 = T + 6;
    REAL tmp[3];
    for (int i = 0; i < 3; ++i) tmp[i] = T2[i] * T2[i];
    const REAL d = FN(dot3)(t, tmp);
    if (d == 0) return;
    REAL f[3];
    for (int i = 0; i < 3; ++i) f[i] = (1 / d) * t[i];
    REAL a[3], b[3], c0[3], c1[3];
    for (int i = 0; i < 3; ++i) {
        a[i] = T0[i] * T2[i];
        b[i] = T1[i] * T2[i];
        c0[i] = T0[i] * T0[i];
        c1[i] = T1[i] * T1[i];
    }
    const REAL px = FN(dot3)(f, a), py = FN(dot3)(f, b);
    const REAL h0x = px * px - FN(dot3)(f, c0), h0y = py * py - FN(dot3)(f, c1);
    const REAL hx = SQRT(h0x > (REAL)1e-4f ? h0x : (REAL)1e-4f), hy = SQRT(h0y > (REAL)1e-4f ? h0y : (REAL)1e-4f);
    REAL m = hx > hy ? hx : hy;
    const REAL lo = (REAL)3.0f * (REAL)0.707106f;
    if (lo > m) m = lo;
    const int r = (int)CEIL(m);
    int x0 = (int)((px - r) / 16), y0 = (int)((py - r) / 16);
    int x1 = (int)((px + r + 16 - 1) / 16), y1 = (int)((py + r + 16 - 1) / 16);
    x0 = x0 < 0 ? 0 : (x0 > gx ? gx : x0);
    y0 = y0 < 0 ? 0 : (y0 > gy ? gy : y0);
    x1 = x1 < 0 ? 0 : (x1 > gx ? gx : x1);
    y1 = y1 < 0 ? 0 : (y1 > gy ? gy : y1);
    if ((x1 - x0) * (y1 - y0) == 0) return;
    REAL rgb[3];
    int clamped = 0;
    if (!in->colors) {
        /* forward.cu:20-65 */
        REAL dir[3] = {po[0] - in->campos[0], po[1] - in->campos[1], po[2] - in->campos[2]};
        const REAL len = SQRT(FN(dot3)(dir, dir));
        for (int i = 0; i < 3; ++i) dir[i] /= len;
        const REAL* sh = in->shs + (int64_t)g * in->M * 3;
        for (int ch = 0; ch < 3; ++ch) {
            REAL res = (REAL)0.28209479177387814 * sh[ch];
            if (in->D > 0) {
                const REAL C1 = (REAL)0.4886025119029199;
                const REAL x = dir[0], y = dir[1], z = dir[2];
                res = res - C1 * y * sh[3 + ch] + C1 * z * sh[6 + ch] - C1 * x * sh[9 + ch];
                if (in->D > 1) {
                    const REAL att = EXP(-x), refl = -(x * x + y * y + z * z);
                    res = res - att * sh[12 + ch] + refl * sh[15 + ch] - (x * z) * sh[18 + ch] + (x * y) * sh[21 + ch] -
                          (z * y) * sh[24 + ch];
                }
            }
            res += (REAL)0.5;
            if (res < 0) clamped |= 1 << ch;
            rgb[ch] = res > 0 ? res : 0;
        }
    } else {
        for (int ch = 0; ch < 3; ++ch) rgb[ch] = in->colors[3 * (int64_t)g + ch];
    }
    *radius_out = r;
    rect[0] = x0; rect[1] = y0; rect[2] = x1; rect[3] = y1;
    for (int i = 0; i < 9; ++i) rec[i] = T[i];
    rec[9] = px; rec[10] = py;
    rec[11] = n[0]; rec[12] = n[1]; rec[13] = n[2];
    rec[14] = in->opac[g];
    rec[15] = rgb[0]; rec[16] = rgb[1]; rec[17] = rgb[2];
    rec[18] = pv[2];
    rec[19] = (REAL)clamped;
}

typedef struct {
    REAL key;
    int g;
} FN(Ent);
static int FN(ent_cmp)(const void* a, const void* b) {
    const FN(Ent)* x = (const FN(Ent)*)a;
    const FN(Ent)* y = (const FN(Ent)*)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return x->g < y->g ? -1 : (x->g > y->g);
}

/* Preprocess + per-tile lists ordered by (view depth, Gaussian) (rasterizer_impl.cu:70-137).
 * Returns the instance total; fills point_list / ranges (T x 2) when non-NULL. */
int64_t FN(gso_bin)(const FN(GsIn) * in, int* radii, REAL* recs, int32_t* point_list, int64_t cap, int32_t* ranges) {
    const int gx = (in->W + 15) / 16, gy = (in->H + 15) / 16, T = gx * gy;
    int* rects = (int*)malloc(sizeof(int) * 4 * (size_t)(in->P > 0 ? in->P : 1));
    int64_t* cnt = (int64_t*)calloc((size_t)T + 1, sizeof(int64_t));
#pragma omp parallel for schedule(static)
    for (int g = 0; g < in->P; ++g) FN(preprocess)(in, g, radii + g, rects + 4 * g, recs + (int64_t)GSO_REC * g);
    for (int g = 0; g < in->P; ++g)
        if (radii[g] > 0)
            for (int y = rects[4 * g + 1]; y < rects[4 * g + 3]; ++y)
                for (int x = rects[4 * g]; x < rects[4 * g + 2]; ++x) cnt[y * gx + x + 1]++;
    for (int t = 0; t < T; ++t) cnt[t + 1] += cnt[t];
    const int64_t total = cnt[T];
    if (point_list && total <= cap) {
        FN(Ent)* e = (FN(Ent)*)malloc(sizeof(FN(Ent)) * (size_t)(total > 0 ? total : 1));
        int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)T);
        for (int t = 0; t < T; ++t) cur[t] = cnt[t];
        for (int g = 0; g < in->P; ++g)
            if (radii[g] > 0)
                for (int y = rects[4 * g + 1]; y < rects[4 * g + 3]; ++y)
                    for (int x = rects[4 * g]; x < rects[4 * g + 2]; ++x) {
                        const int t = y * gx + x;
                        e[cur[t]].key = recs[(int64_t)GSO_REC * g + 18];
                        e[cur[t]].g = g;
                        cur[t]++;
                    }
        for (int t = 0; t < T; ++t) qsort(e + cnt[t], (size_t)(cnt[t + 1] - cnt[t]), sizeof(FN(Ent)), FN(ent_cmp));
        for (int64_t i = 0; i < total; ++i) point_list[i] = e[i].g;
        for (int t = 0; t < T; ++t) {
            ranges[2 * t] = cnt[t + 1] > cnt[t] ? (int32_t)cnt[t] : 0;
            ranges[2 * t + 1] = cnt[t + 1] > cnt[t] ? (int32_t)cnt[t + 1] : 0;
        }
        free(e);
        free(cur);
    }
    free(rects);
    free(cnt);
    return total;
}

/* Ray-splat intersection (forward.cu:335-358); returns 0 when skipped before alpha. */
static int FN(hit)(REAL pxf, REAL pyf, const REAL* rc, REAL* k, REAL* l, REAL* p, REAL* s, REAL* rho3d, REAL* rho2d,
                   REAL* d, REAL* depth) {
    const REAL *Tu = rc, *Tv = rc + 3, *Tw = rc + 6;
    for (int i = 0; i < 3; ++i) {
        k[i] = pxf * Tw[i] - Tu[i];
        l[i] = pyf * Tw[i] - Tv[i];
    }
    p[0] = k[1] * l[2] - k[2] * l[1];
    p[1] = k[2] * l[0] - k[0] * l[2];
    p[2] = k[0] * l[1] - k[1] * l[0];
    if (p[2] == 0) return 0;
    s[0] = p[0] / p[2];
    s[1] = p[1] / p[2];
    *rho3d = s[0] * s[0] + s[1] * s[1];
    d[0] = rc[9] - pxf;
    d[1] = rc[10] - pyf;
    *rho2d = 2 * (d[0] * d[0] + d[1] * d[1]);
    *depth = (s[0] * Tw[0] + s[1] * Tw[1]) + Tw[2];
    return !(*depth < (REAL)0.2f);
}

/* Front-to-back compositing (forward.cu:249-439). color (3,H,W), others (7,H,W), accum
 * (3,H,W: T, M1, M2), n_contrib (2,H,W). */
void FN(gso_forward)(const FN(GsIn) * in, const REAL* recs, const int32_t* point_list, const int32_t* ranges,
                     REAL* color, REAL* others, REAL* accum, uint32_t* n_contrib) {
    const int W = in->W, H = in->H, gx = (W + 15) / 16;
    const int64_t HW = (int64_t)W * H;
    const REAL nearn = (REAL)0.2f, farn = (REAL)100.0f, ms = farn / (farn - nearn);
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int t = (y / 16) * gx + x / 16;
            REAL T = 1, C[3] = {0, 0, 0}, N[3] = {0, 0, 0}, D = 0, M1 = 0, M2 = 0, dist = 0, med = 0;
            REAL medc = -1;
            uint32_t contributor = 0, last = 0;
            for (int i = ranges[2 * t]; i < ranges[2 * t + 1]; ++i) {
                ++contributor;
                const REAL* rc = recs + (int64_t)GSO_REC * point_list[i];
                REAL k[3], l[3], p[3], s[2], r3, r2, d[2], depth;
                if (!FN(hit)((REAL)x, (REAL)y, rc, k, l, p, s, &r3, &r2, d, &depth)) continue;
                const REAL power = (REAL)-0.5 * (r3 < r2 ? r3 : r2);
                if (power > 0) continue;
                REAL alpha = rc[14] * EXP(power);
                if (alpha > (REAL)0.99f) alpha = (REAL)0.99f;
                if (alpha < (REAL)(1.0f / 255.0f)) continue;
                const REAL test_T = T * (1 - alpha);
                if (test_T < (REAL)0.0001f) break;
                const REAL w = alpha * T, A = 1 - T;
                const REAL m = ms * (1 - nearn / depth);
                dist += (m * m * A + M2 - 2 * m * M1) * w;
                D += depth * w;
                M1 += m * w;
                M2 += m * m * w;
                if (T > 0.5) {
                    med = depth;
                    medc = (REAL)contributor;
                }
                for (int c = 0; c < 3; ++c) {
                    N[c] += rc[11 + c] * w;
                    C[c] += rc[15 + c] * w;
                }
                T = test_T;
                last = contributor;
            }
            const int64_t pix = (int64_t)y * W + x;
            accum[pix] = T; accum[pix + HW] = M1; accum[pix + 2 * HW] = M2;
            n_contrib[pix] = last;
            n_contrib[pix + HW] = medc < 0 ? 0u : (uint32_t)medc;
            for (int c = 0; c < 3; ++c) color[c * HW + pix] = C[c] + T * in->bg[c];
            others[pix] = D; others[pix + HW] = 1 - T;
            for (int c = 0; c < 3; ++c) others[pix + (2 + c) * HW] = N[c];
            others[pix + 5 * HW] = med; others[pix + 6 * HW] = dist;
        }
}

/* Backward (backward.cu:103-602). Outputs as the reference returns them: dmeans2D (P,3),
 * dcolors (P,3), dopac (P), dmeans3D (P,3), dtrans (P,9), dsh (P,M,3), dscales (P,2),
 * drot (P,4); all overwritten. tan_fov are the values the reference's backward gets. */
void FN(gso_backward)(const FN(GsIn) * in, const REAL* recs, const int* radii, const int32_t* point_list,
                      const int32_t* ranges, const REAL* accum, const uint32_t* n_contrib, const REAL* dpix_img,
                      const REAL* dothers, float tanfx, float tanfy, REAL* dm2, REAL* dcol, REAL* dop, REAL* dm3,
                      REAL* dtr, REAL* dsh, REAL* dsc, REAL* drot) {
    const int W = in->W, H = in->H, gx = (W + 15) / 16, P = in->P;
    const int64_t HW = (int64_t)W * H;
    const REAL nearn = (REAL)0.2f, farn = (REAL)100.0f, ms = farn / (farn - nearn);
    const int NG = 18;
    REAL* acc = (REAL*)calloc((size_t)(P > 0 ? P : 1) * NG, sizeof(REAL));
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int t = (y / 16) * gx + x / 16;
            const int64_t pix = (int64_t)y * W + x;
            const int n = ranges[2 * t + 1] - ranges[2 * t];
            const REAL T_final = accum[pix];
            REAL T = T_final;
            uint32_t contributor = (uint32_t)n;
            const int lastc = (int)n_contrib[pix], medc = (int)n_contrib[pix + HW];
            REAL dp[3], dn[3];
            for (int c = 0; c < 3; ++c) {
                dp[c] = dpix_img[c * HW + pix];
                dn[c] = dothers[(2 + c) * HW + pix];
            }
            const REAL dd = dothers[pix], da = dothers[HW + pix], dreg = dothers[6 * HW + pix],
                       dmed = dothers[5 * HW + pix];
            const REAL fD = accum[pix + HW], fD2 = accum[pix + 2 * HW], fA = 1 - T_final;
            REAL arec[3] = {0, 0, 0}, lcol[3] = {0, 0, 0}, lnrm[3] = {0, 0, 0}, anrm[3] = {0, 0, 0};
            REAL ldepth = 0, adepth = 0, aalpha = 0, ldT = 0, lalpha = 0;
            const REAL bgdot = in->bg[0] * dp[0] + in->bg[1] * dp[1] + in->bg[2] * dp[2];
            for (int j = ranges[2 * t + 1] - 1; j >= ranges[2 * t]; --j) {
                --contributor;
                if (contributor >= (uint32_t)lastc) continue;
                const int g = point_list[j];
                const REAL* rc = recs + (int64_t)GSO_REC * g;
                REAL k[3], l[3], p[3], s[2], r3, r2, d[2], cd;
                if (!FN(hit)((REAL)x, (REAL)y, rc, k, l, p, s, &r3, &r2, d, &cd)) continue;
                const REAL power = (REAL)-0.5 * (r3 < r2 ? r3 : r2);
                if (power > 0) continue;
                const REAL G = EXP(power);
                REAL alpha = rc[14] * G;
                if (alpha > (REAL)0.99f) alpha = (REAL)0.99f;
                if (alpha < (REAL)(1.0f / 255.0f)) continue;
                REAL* a = acc + (size_t)g * NG;
                T = T / (1 - alpha);
                REAL dalpha = 0;
                for (int c = 0; c < 3; ++c) {
                    arec[c] = lalpha * lcol[c] + (1 - lalpha) * arec[c];
                    lcol[c] = rc[15 + c];
                    dalpha += (rc[15 + c] - arec[c]) * dp[c];
                    a[15 + c] += alpha * T * dp[c];
                }
                REAL dz = 0;
                const REAL md = ms * (1 - nearn / cd);
                const REAL dmd = (farn * nearn) / ((farn - nearn) * cd * cd);
                if (contributor == (uint32_t)(medc - 1)) dz += dmed;
                const REAL dw = (fD2 + md * md * fA - 2 * md * fD) * dreg;
                dalpha += dw - ldT;
                ldT = dw * alpha + (1 - alpha) * ldT;
                dz += 2 * (T * alpha) * (md * fA - fD) * dreg * dmd;
                adepth = lalpha * ldepth + (1 - lalpha) * adepth;
                ldepth = cd;
                dalpha += (cd - adepth) * dd;
                aalpha = lalpha + (1 - lalpha) * aalpha;
                dalpha += (1 - aalpha) * da;
                for (int c = 0; c < 3; ++c) {
                    anrm[c] = lalpha * lnrm[c] + (1 - lalpha) * anrm[c];
                    lnrm[c] = rc[11 + c];
                    dalpha += (rc[11 + c] - anrm[c]) * dn[c];
                    a[11 + c] += alpha * T * dn[c];
                }
                dalpha *= T;
                lalpha = alpha;
                dalpha += (-T_final / (1 - alpha)) * bgdot;
                const REAL dG = rc[14] * dalpha;
                dz += alpha * T * dd;
                if (r3 <= r2) {
                    const REAL dsx = dG * -G * s[0] + dz * rc[6], dsy = dG * -G * s[1] + dz * rc[7];
                    const REAL ax = dsx / p[2], ay = dsy / p[2];
                    const REAL dpv[3] = {ax, ay, -(ax * s[0] + ay * s[1])};
                    const REAL dk[3] = {l[1] * dpv[2] - l[2] * dpv[1], l[2] * dpv[0] - l[0] * dpv[2],
                                        l[0] * dpv[1] - l[1] * dpv[0]};
                    const REAL dl[3] = {dpv[1] * k[2] - dpv[2] * k[1], dpv[2] * k[0] - dpv[0] * k[2],
                                        dpv[0] * k[1] - dpv[1] * k[0]};
                    const REAL dzw[3] = {s[0], s[1], 1};
                    for (int c = 0; c < 3; ++c) {
                        a[c] += -dk[c];
                        a[3 + c] += -dl[c];
                        a[6 + c] += (REAL)x * dk[c] + (REAL)y * dl[c] + dz * dzw[c];
                    }
                } else {
                    a[9] += dG * (-G * 2 * d[0]);
                    a[10] += dG * (-G * 2 * d[1]);
                    a[6] += s[0] * dz;
                    a[7] += s[1] * dz;
                    a[8] += dz;
                }
                a[14] += G * dalpha;
            }
        }
    const int Wb = (int)((in->W / (2.0f * tanfx)) * tanfx * 2);
    const int Hb = (int)((in->H / (2.0f * tanfy)) * tanfy * 2);
    for (int g = 0; g < P; ++g) {
        const REAL* a = acc + (size_t)g * NG;
        REAL dT[9], m3[3] = {0, 0, 0}, sc[2] = {0, 0}, dr[4] = {0, 0, 0, 0}, m2x = 0, m2y = 0;
        for (int i = 0; i < 9; ++i) dT[i] = a[i];
        if (in->shs)
            for (int i = 0; i < in->M * 3; ++i) dsh[(int64_t)g * in->M * 3 + i] = 0;
        if (radii[g] > 0) {
            const int precomp = in->scales == NULL;
            const REAL* po = in->means + 3 * (int64_t)g;
            REAL T[9], R[9], L[9], Pm[12], n[3] = {0, 0, 0};
            if (precomp) {
                for (int i = 0; i < 9; ++i) T[i] = in->transmat[9 * (int64_t)g + i];
            } else {
                FN(homography)(in->rots + 4 * (int64_t)g, in->scales[2 * g], in->scales[2 * g + 1], 1, po,
                               in->proj, Wb, Hb, 1, T, R, L, Pm);
                FN(xform_vec)(L + 6, in->view, n);
            }
            REAL dLT[9];
            for (int i = 0; i < 9; ++i) dLT[i] = dT[i];
            int early = 0;
            const REAL dmx = a[9], dmy = a[10];
            if (dmx != 0 || dmy != 0) {
                const REAL tv[3] = {9, 9, -1};
                const REAL *T0 = T, *T1 = T + 3, *T2 = T + 6;
                REAL tmp[3];
                for (int i = 0; i < 3; ++i) tmp[i] = T2[i] * T2[i];
                const REAL dd = FN(dot3)(tv, tmp);
                REAL fv[3], dfv[3], d3[3];
                for (int i = 0; i < 3; ++i) fv[i] = tv[i] * (1 / dd);
                for (int i = 0; i < 3; ++i) {
                    dfv[i] = dmx * T0[i] * T2[i] + dmy * T1[i] * T2[i];
                    d3[i] = dmx * fv[i] * T0[i] + dmy * fv[i] * T1[i];
                }
                const REAL dLdd = FN(dot3)(dfv, fv) * (-1 / dd);
                for (int i = 0; i < 3; ++i) {
                    dLT[i] += dmx * fv[i] * T2[i];
                    dLT[3 + i] += dmy * fv[i] * T2[i];
                    dLT[6 + i] += d3[i] + dLdd * (tv[i] * T2[i] * 2);
                }
                if (precomp) {
                    for (int i = 0; i < 9; ++i) dT[i] = dLT[i];
                    early = 1;
                }
            }
            if (!precomp && !early) {
                REAL tr[9], dM[12];
                FN(transp)(dLT, 3, 3, tr);
                FN(mmul)(Pm, 3, 4, tr, 3, dM);
                REAL dn[3] = {a[11], a[12], a[13]}, dtn[3], pv[3];
                const REAL* vm = in->view;
                dtn[0] = vm[0] * dn[0] + vm[1] * dn[1] + vm[2] * dn[2];
                dtn[1] = vm[4] * dn[0] + vm[5] * dn[1] + vm[6] * dn[2];
                dtn[2] = vm[8] * dn[0] + vm[9] * dn[1] + vm[10] * dn[2];
                FN(xform_point)(po, in->view, pv);
                const REAL cosv = -(pv[0] * n[0] + pv[1] * n[1] + pv[2] * n[2]);
                const REAL mult = cosv > 0 ? 1 : -1;
                REAL dR[9];
                for (int i = 0; i < 3; ++i) {
                    dR[i] = dM[i] * in->scales[2 * g];
                    dR[3 + i] = dM[4 + i] * in->scales[2 * g + 1];
                    dR[6 + i] = mult * dtn[i];
                }
                FN(quat_rot_vjp)(in->rots + 4 * (int64_t)g, dR, dr);
                sc[0] = dM[0] * R[0] + dM[1] * R[1] + dM[2] * R[2];
                sc[1] = dM[4] * R[3] + dM[5] * R[4] + dM[6] * R[5];
                m3[0] = dM[8]; m3[1] = dM[9]; m3[2] = dM[10];
            }
            if (in->shs) {
                REAL dir0[3] = {po[0] - in->campos[0], po[1] - in->campos[1], po[2] - in->campos[2]};
                const REAL len = SQRT(FN(dot3)(dir0, dir0));
                const REAL x = dir0[0] / len, y = dir0[1] / len, z = dir0[2] / len;
                const REAL* sh = in->shs + (int64_t)g * in->M * 3;
                REAL* o = dsh + (int64_t)g * in->M * 3;
                const int cl = (int)recs[(int64_t)GSO_REC * g + 19];
                REAL dRGB[3];
                for (int c = 0; c < 3; ++c) dRGB[c] = (cl >> c & 1) ? 0 : a[15 + c];
                REAL ddx[3] = {0, 0, 0}, ddy[3] = {0, 0, 0}, ddz[3] = {0, 0, 0};
                const REAL C0 = (REAL)0.28209479177387814, C1 = (REAL)0.4886025119029199;
                for (int c = 0; c < 3; ++c) o[c] = C0 * dRGB[c];
                if (in->D > 0) {
                    for (int c = 0; c < 3; ++c) {
                        o[3 + c] = -C1 * y * dRGB[c];
                        o[6 + c] = C1 * z * dRGB[c];
                        o[9 + c] = -C1 * x * dRGB[c];
                        ddx[c] = -C1 * sh[9 + c];
                        ddy[c] = -C1 * sh[3 + c];
                        ddz[c] = C1 * sh[6 + c];
                    }
                    if (in->D > 1) {
                        const REAL d4 = EXP(-x), d5 = x * x + y * y + z * z, d6 = x * y, d7 = y * z, d8 = x * z;
                        for (int c = 0; c < 3; ++c) {
                            o[12 + c] = d4 * dRGB[c];
                            o[15 + c] = d5 * dRGB[c];
                            o[18 + c] = d6 * dRGB[c];
                            o[21 + c] = d7 * dRGB[c];
                            o[24 + c] = d8 * dRGB[c];
                            ddx[c] = ddx[c] - d4 - d5 + d6 - d8;
                            ddy[c] = ddy[c] - d5 - d6 + d7;
                            ddz[c] = ddz[c] - d5 - d7 + d8;
                        }
                    }
                }
                const REAL dv[3] = {FN(dot3)(ddx, dRGB), FN(dot3)(ddy, dRGB), FN(dot3)(ddz, dRGB)};
                const REAL s2 = FN(dot3)(dir0, dir0);
                const REAL inv32 = 1 / SQRT(s2 * s2 * s2);
                m3[0] += ((s2 - dir0[0] * dir0[0]) * dv[0] - dir0[1] * dir0[0] * dv[1] - dir0[2] * dir0[0] * dv[2]) * inv32;
                m3[1] += (-dir0[0] * dir0[1] * dv[0] + (s2 - dir0[1] * dir0[1]) * dv[1] - dir0[2] * dir0[1] * dv[2]) * inv32;
                m3[2] += (-dir0[0] * dir0[2] * dv[0] - dir0[1] * dir0[2] * dv[1] + (s2 - dir0[2] * dir0[2]) * dv[2]) * inv32;
            }
            const REAL depth = recs[(int64_t)GSO_REC * g + 8];
            m2x = dT[2] * depth * (REAL)0.5 * (REAL)Wb;
            m2y = dT[5] * depth * (REAL)0.5 * (REAL)Hb;
        }
        dm2[3 * g] = m2x; dm2[3 * g + 1] = m2y; dm2[3 * g + 2] = 0;
        for (int c = 0; c < 3; ++c) {
            dcol[3 * g + c] = a[15 + c];
            dm3[3 * g + c] = m3[c];
        }
        dop[g] = a[14];
        for (int i = 0; i < 9; ++i) dtr[9 * g + i] = dT[i];
        if (dsc) { dsc[2 * g] = sc[0]; dsc[2 * g + 1] = sc[1]; }
        if (drot)
            for (int i = 0; i < 4; ++i) drot[4 * g + i] = dr[i];
    }
    free(acc);
}

#undef FN
#undef CAT
#undef CAT2
