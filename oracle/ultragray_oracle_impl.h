/*
 * TEST INFRASTRUCTURE ONLY — never part of the product path.
 *
 * CPU restatement of the reference UltraGray scanline renderer (KevinWCCC/ultrasound-3d-
 * reconstruction, ops/ultragray_renderer). Included twice by ultragray_oracle.c with
 * REAL = float (suffix _f32) and REAL = double (suffix _f64). Each function names the
 * reference lines it follows. The reference tree lacks the header that defines the
 * quaternion rotation, the precision matrix and their gradients (covariance.cuh); those
 * four pieces follow the mathematics their call sites imply: R of the normalised (w,x,y,z)
 * quaternion with the Gaussian's axes as columns, precision R diag(1/s^2) R^T, and the
 * exact gradients of both.
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUFFIX)

static REAL FN(dot3)(const REAL* a, const REAL* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

/* Rotation of the normalised quaternion (w,x,y,z) = q[0..3], row-major. */
static void FN(rot)(const REAL* q, REAL* R) {
    const REAL n = (REAL)1 / SQRT(FMAX(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3], (REAL)1e-12));
    const REAL w = q[0] * n, x = q[1] * n, y = q[2] * n, z = q[3] * n;
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

/* Precision R diag(1/s^2) R^T. */
static void FN(prec)(const REAL* s, const REAL* R, REAL* P) {
    const REAL d[3] = {1 / (s[0] * s[0]), 1 / (s[1] * s[1]), 1 / (s[2] * s[2])};
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
            P[r * 3 + c] = R[r * 3] * d[0] * R[c * 3] + R[r * 3 + 1] * d[1] * R[c * 3 + 1] + R[r * 3 + 2] * d[2] * R[c * 3 + 2];
}

/* dL/dq of R(q/|q|) given dL/dR (row-major). */
static void FN(quat_grad)(const REAL* q, const REAL* g, REAL* dq) {
    const REAL len = SQRT(FMAX(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3], (REAL)1e-12));
    const REAL n = 1 / len;
    const REAL w = q[0] * n, x = q[1] * n, y = q[2] * n, z = q[3] * n;
    /* gradient w.r.t. the normalised quaternion, from R's entries above */
    const REAL gw = 2 * (-z * g[1] + y * g[2] + z * g[3] - x * g[5] - y * g[6] + x * g[7]);
    const REAL gx = 2 * (y * g[1] + z * g[2] + y * g[3] - 2 * x * g[4] - w * g[5] + z * g[6] + w * g[7] - 2 * x * g[8]);
    const REAL gy = 2 * (-2 * y * g[0] + x * g[1] + w * g[2] + x * g[3] + z * g[5] - w * g[6] + z * g[7] - 2 * y * g[8]);
    const REAL gz = 2 * (-2 * z * g[0] - w * g[1] + x * g[2] + w * g[3] - 2 * z * g[4] + y * g[5] + x * g[6] + y * g[7]);
    /* through q/|q|: (I - u u^T) g / |q| */
    const REAL dot = w * gw + x * gx + y * gy + z * gz;
    dq[0] = (gw - w * dot) * n;
    dq[1] = (gx - x * dot) * n;
    dq[2] = (gy - y * dot) * n;
    dq[3] = (gz - z * dot) * n;
}

/* Ray frame in the Gaussian's canonical coordinates and the quadrature nodes
 * (include/shader/shared.cuh:27-85). Returns 0 when the integral is empty. */
typedef struct {
    REAL diff[3], og[3], dg[3], is[3], half, t[3], f[3];
} FN(Quad);

static int FN(quad_setup)(const REAL* ro, const REAL* rd, const REAL* mu, const REAL* s, const REAL* R, REAL l,
                          REAL wr, FN(Quad)* Q) {
    static const REAL xi[3] = {(REAL)-0.7745966692, (REAL)0.0, (REAL)0.7745966692};
    if (l <= 0) return 0;
    for (int i = 0; i < 3; ++i) Q->diff[i] = ro[i] - mu[i];
    REAL ol[3], dl[3];
    for (int c = 0; c < 3; ++c) {
        ol[c] = R[c] * Q->diff[0] + R[3 + c] * Q->diff[1] + R[6 + c] * Q->diff[2];
        dl[c] = R[c] * rd[0] + R[3 + c] * rd[1] + R[6 + c] * rd[2];
    }
    for (int c = 0; c < 3; ++c) {
        Q->is[c] = 1 / s[c];
        Q->og[c] = ol[c] / s[c];
        Q->dg[c] = dl[c] / s[c];
    }
    const REAL dg2 = FN(dot3)(Q->dg, Q->dg);
    const REAL tc = -FN(dot3)(Q->og, Q->dg) / (dg2 + (REAL)1e-8);
    REAL t0 = 0, t1 = l;
    if (wr > 0) {
        t0 = FMAX((REAL)0, tc - wr);
        t1 = FMIN(l, tc + wr);
    }
    if (t1 <= t0) return 0;
    Q->half = (REAL)0.5 * (t1 - t0);
    const REAL c = (REAL)0.5 * (t1 + t0);
    for (int k = 0; k < 3; ++k) {
        Q->t[k] = Q->half * xi[k] + c;
        REAL xq[3];
        for (int i = 0; i < 3; ++i) xq[i] = Q->og[i] + Q->dg[i] * Q->t[k];
        Q->f[k] = EXP((REAL)-0.5 * FN(dot3)(xq, xq));
    }
    return 1;
}

static const REAL FN(gl_w)[3] = {(REAL)0.5555555556, (REAL)0.8888888889, (REAL)0.5555555556};

static REAL FN(integral)(const REAL* ro, const REAL* rd, const REAL* mu, const REAL* s, const REAL* R, REAL l,
                         REAL wr) {
    FN(Quad) Q;
    if (!FN(quad_setup)(ro, rd, mu, s, R, l, wr, &Q)) return 0;
    return Q.half * (FN(gl_w)[0] * Q.f[0] + FN(gl_w)[1] * Q.f[1] + FN(gl_w)[2] * Q.f[2]);
}

/* Reference mapper (src/mapper/core.cu:3-129, wrapper_mapper.cu:7-128): culls, ray range,
 * per-ray lists ordered by (quantised depth, Gaussian index), sorted depths. Returns the
 * instance total; fills the CSR only when indices != NULL and total <= cap. */
typedef struct {
    uint32_t dq;
    int32_t g;
} FN(RayEntry);

static int FN(entry_cmp)(const void* a, const void* b) {
    const FN(RayEntry)* x = (const FN(RayEntry)*)a;
    const FN(RayEntry)* y = (const FN(RayEntry)*)b;
    if (x->dq != y->dq) return x->dq < y->dq ? -1 : 1;
    return x->g < y->g ? -1 : (x->g > y->g);
}

int64_t FN(ugro_map)(int64_t G, int W, const REAL* means, const REAL* scales, const REAL* origin, const REAL* lat,
                     const REAL* ele, const REAL* ax, REAL width_mm, REAL near_mm, REAL col_off, REAL elev_cut,
                     REAL k_sigma, int32_t* counts, int32_t* offsets, int32_t* indices, REAL* depths, int64_t cap) {
    const REAL spacing = width_mm / (REAL)W;
    int32_t* r0s = (int32_t*)malloc(sizeof(int32_t) * 2 * (size_t)(G > 0 ? G : 1));
    uint32_t* dqs = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)(G > 0 ? G : 1));
    int64_t* cnt = (int64_t*)calloc((size_t)W + 1, sizeof(int64_t));
    for (int64_t g = 0; g < G; ++g) {
        r0s[2 * g] = 0;
        r0s[2 * g + 1] = -1;
        const REAL* m = means + 3 * g;
        const REAL* s = scales + 3 * g;
        const REAL diff[3] = {m[0] - origin[0], m[1] - origin[1], m[2] - origin[2]};
        const REAL px = FN(dot3)(diff, lat), py = FN(dot3)(diff, ele), pz = FN(dot3)(diff, ax);
        const REAL radius = FMAX(s[0], FMAX(s[1], s[2])) * k_sigma;
        if (pz + radius < near_mm) continue;
        if (FABS(py) > radius + elev_cut) continue;
        const REAL centre = px / spacing + col_off;
        const REAL rad = radius / spacing;
        int a = ugro_i32((double)FLOOR(centre - rad)), b = ugro_i32((double)CEIL(centre + rad));
        a = a > 0 ? a : 0;
        b = b < W - 1 ? b : W - 1;
        if (a > b) continue;
        r0s[2 * g] = a;
        r0s[2 * g + 1] = b;
        dqs[g] = ugro_u32_sat((double)(FMAX((REAL)0, pz) * (REAL)1000));
        for (int x = a; x <= b; ++x) cnt[x + 1]++;
    }
    for (int x = 0; x < W; ++x) cnt[x + 1] += cnt[x];
    const int64_t total = cnt[W];
    if (counts)
        for (int x = 0; x < W; ++x) {
            counts[x] = (int32_t)(cnt[x + 1] - cnt[x]);
            offsets[x] = counts[x] > 0 ? (int32_t)cnt[x] : 0;
        }
    if (indices && total <= cap) {
        FN(RayEntry)* e = (FN(RayEntry)*)malloc(sizeof(FN(RayEntry)) * (size_t)(total > 0 ? total : 1));
        int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)(W > 0 ? W : 1));
        for (int x = 0; x < W; ++x) cur[x] = cnt[x];
        for (int64_t g = 0; g < G; ++g)
            for (int x = r0s[2 * g]; x <= r0s[2 * g + 1]; ++x) {
                e[cur[x]].dq = dqs[g];
                e[cur[x]].g = (int32_t)g;
                cur[x]++;
            }
        for (int x = 0; x < W; ++x)
            qsort(e + cnt[x], (size_t)(cnt[x + 1] - cnt[x]), sizeof(FN(RayEntry)), FN(entry_cmp));
        for (int64_t i = 0; i < total; ++i) {
            indices[i] = e[i].g;
            depths[i] = (REAL)((float)e[i].dq * 0.001f);
        }
        free(e);
        free(cur);
    }
    free(r0s);
    free(dqs);
    free(cnt);
    return total;
}

/* Per-pixel walk shared by the forward and the backward: the entries of the ray that the
 * pixel visits, and for each whether it attenuates (transmission) and/or echoes
 * (src/shader/forward.cu:67-111, backward.cu:187-233). */
typedef struct {
    REAL ro[3], rd[3], p[3], t_pixel;
} FN(PixelGeo);

static void FN(pixel_geo)(int x, int y, int H, const REAL* pixels, const REAL* ray_o, const REAL* ray_d,
                          const REAL* ele, const REAL* pert, FN(PixelGeo)* g) {
    const REAL* pp = pixels + ((int64_t)x * H + y) * 3;
    for (int i = 0; i < 3; ++i) {
        g->p[i] = pp[i];
        g->ro[i] = ray_o[3 * x + i] + ele[i] * pert[x];
        g->rd[i] = ray_d[3 * x + i];
    }
    const REAL v[3] = {g->p[0] - g->ro[0], g->p[1] - g->ro[1], g->p[2] - g->ro[2]};
    g->t_pixel = FMAX((REAL)0, FN(dot3)(v, g->rd));
}

/* 0 = skip, bit 0 = transmission, bit 1 = echo */
static int FN(visit)(const FN(PixelGeo)* pg, const REAL* mu, const REAL* s, REAL depth, REAL k_sigma, REAL wr,
                     int local, REAL maxwin) {
    if (local && (depth < pg->t_pixel - maxwin || depth > pg->t_pixel + maxwin)) return 0;
    const REAL v[3] = {mu[0] - pg->ro[0], mu[1] - pg->ro[1], mu[2] - pg->ro[2]};
    const REAL tg = FN(dot3)(v, pg->rd);
    const REAL dr = FMAX(s[0], FMAX(s[1], s[2])) * k_sigma;
    int need_t = tg < pg->t_pixel;
    if (local) need_t = need_t && ((pg->t_pixel - tg) <= dr + wr);
    const int need_e = FABS(tg - pg->t_pixel) <= dr;
    return need_t | (need_e << 1);
}

static REAL FN(weight)(const REAL* p, const REAL* mu, const REAL* P, REAL* d) {
    d[0] = p[0] - mu[0];
    d[1] = p[1] - mu[1];
    d[2] = p[2] - mu[2];
    const REAL pw = (REAL)-0.5 * ((P[0] * d[0] + P[1] * d[1] + P[2] * d[2]) * d[0] +
                                  (P[3] * d[0] + P[4] * d[1] + P[5] * d[2]) * d[1] +
                                  (P[6] * d[0] + P[7] * d[1] + P[8] * d[2]) * d[2]);
    return EXP(pw);
}

static REAL FN(sigmoid)(REAL a) { return 1 / (1 + EXP(-a)); }

/* Forward (src/shader/forward.cu:22-119). state (W*H*4, optional): T, num, den, S per pixel
 * at index x*H + y. */
void FN(ugro_forward)(int W, int H, const int32_t* counts, const int32_t* offsets, const int32_t* indices,
                      const REAL* depths, const REAL* means, const REAL* scales, const REAL* quats,
                      const REAL* attens, const REAL* sh, const REAL* pixels, const REAL* ray_o, const REAL* ray_d,
                      const REAL* ele, const REAL* pert, REAL k_sigma, REAL wr, int local, REAL maxwin,
                      REAL* image, REAL* state) {
#pragma omp parallel for schedule(dynamic, 1)
    for (int x = 0; x < W; ++x) {
        for (int y = 0; y < H; ++y) {
            if (counts[x] == 0) {
                image[(int64_t)y * W + x] = 0;
                if (state) {
                    REAL* st = state + 4 * ((int64_t)x * H + y);
                    st[0] = 1; st[1] = 0; st[2] = 0; st[3] = 0;
                }
                continue;
            }
            FN(PixelGeo) pg;
            FN(pixel_geo)(x, y, H, pixels, ray_o, ray_d, ele, pert, &pg);
            REAL T = 1, num = 0, den = 0, S = 0;
            for (int k = 0; k < counts[x]; ++k) {
                const int i = offsets[x] + k;
                const int g = indices[i];
                const REAL* mu = means + 3 * (int64_t)g;
                const REAL* s = scales + 3 * (int64_t)g;
                const int v = FN(visit)(&pg, mu, s, depths[i], k_sigma, wr, local, maxwin);
                if (!v) continue;
                REAL R[9];
                FN(rot)(quats + 4 * (int64_t)g, R);
                if (v & 1) {
                    const REAL tau = FN(sigmoid)(attens[g]);
                    const REAL psi = FN(integral)(pg.ro, pg.rd, mu, s, R, pg.t_pixel, wr);
                    T *= tau + (1 - tau) * EXP(-psi);
                }
                if (v & 2) {
                    REAL P[9], d[3];
                    FN(prec)(s, R, P);
                    const REAL w = FN(weight)(pg.p, mu, P, d);
                    const REAL* c = sh + 4 * (int64_t)g;
                    const REAL I = c[0] + c[1] * pg.rd[0] + c[2] * pg.rd[1] + c[3] * pg.rd[2];
                    num += I * w;
                    den += w;
                    S += w;
                }
            }
            const REAL gamma = 1 - EXP(-S);
            image[(int64_t)y * W + x] = T * (gamma * (num / (den + (REAL)1e-6)));
            if (state) {
                REAL* st = state + 4 * ((int64_t)x * H + y);
                st[0] = T; st[1] = num; st[2] = den; st[3] = S;
            }
        }
    }
}

/* Backward (src/shader/backward.cu:26-325) with per-thread accumulators reduced in thread
 * order. Gradient arrays: dm (G,3), ds (G,3), dq (G,4), da (G), dsh (G,4), overwritten. */
void FN(ugro_backward)(int64_t G, int W, int H, const int32_t* counts, const int32_t* offsets,
                       const int32_t* indices, const REAL* depths, const REAL* means, const REAL* scales,
                       const REAL* quats, const REAL* attens, const REAL* sh, const REAL* pixels, const REAL* ray_o,
                       const REAL* ray_d, const REAL* ele, const REAL* pert, REAL k_sigma, REAL wr, int local,
                       REAL maxwin, const REAL* state, const REAL* grad_image, REAL* dm, REAL* ds, REAL* dq,
                       REAL* da, REAL* dsh) {
    enum { NF = 15 };
    const int nt = ugo_max_threads_ugr();
    REAL* acc = (REAL*)calloc((size_t)nt * (size_t)(G > 0 ? G : 1) * NF, sizeof(REAL));
#pragma omp parallel for schedule(dynamic, 1)
    for (int x = 0; x < W; ++x) {
        REAL* A = acc + (size_t)ugo_thread_id_ugr() * (size_t)G * NF;
        if (counts[x] == 0) continue;
        for (int y = 0; y < H; ++y) {
            const REAL gB = grad_image[(int64_t)y * W + x];
            if (FABS(gB) < (REAL)1e-6) continue;
            FN(PixelGeo) pg;
            FN(pixel_geo)(x, y, H, pixels, ray_o, ray_d, ele, pert, &pg);
            const REAL* st = state + 4 * ((int64_t)x * H + y);
            const REAL T = st[0], num = st[1], den = st[2], S = st[3];
            const REAL eps = (REAL)1e-6;
            const REAL gamma = 1 - EXP(-S);
            const REAL e_raw = num / (den + eps);
            const REAL dT = gB * (gamma * e_raw);
            const REAL dE = gB * T;
            const REAL dgam = dE * e_raw, de_raw = dE * gamma;
            const REAL dS = dgam * EXP(-S);
            const REAL dnum = de_raw * (1 / (den + eps));
            const REAL dden = de_raw * (-num / ((den + eps) * (den + eps)));
            for (int k = 0; k < counts[x]; ++k) {
                const int i = offsets[x] + k;
                const int g = indices[i];
                const REAL* mu = means + 3 * (int64_t)g;
                const REAL* s = scales + 3 * (int64_t)g;
                const int v = FN(visit)(&pg, mu, s, depths[i], k_sigma, wr, local, maxwin);
                if (!v) continue;
                REAL R[9], dR[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
                FN(rot)(quats + 4 * (int64_t)g, R);
                REAL* a = A + (size_t)g * NF; /* dm 0-2, ds 3-5, dq 6-9, da 10, dsh 11-14 */
                if (v & 1) {
                    const REAL tau = FN(sigmoid)(attens[g]);
                    const REAL psi = FN(integral)(pg.ro, pg.rd, mu, s, R, pg.t_pixel, wr);
                    const REAL ep = EXP(-psi);
                    const REAL Ti = tau + (1 - tau) * ep;
                    const REAL dTi = Ti > (REAL)1e-6 ? dT * (T / Ti) : 0;
                    a[10] += dTi * (1 - ep) * (tau * (1 - tau));
                    const REAL dpsi = -dTi * (1 - tau) * ep;
                    FN(Quad) Q;
                    if (FN(quad_setup)(pg.ro, pg.rd, mu, s, R, pg.t_pixel, wr, &Q)) {
                        const REAL coeff = dpsi * Q.half;
                        REAL gog[3] = {0, 0, 0}, gdg[3] = {0, 0, 0};
                        for (int q = 0; q < 3; ++q)
                            for (int c = 0; c < 3; ++c) {
                                const REAL xq = Q.og[c] + Q.dg[c] * Q.t[q];
                                gog[c] += xq * (-coeff * FN(gl_w)[q] * Q.f[q]);
                                gdg[c] += xq * (-coeff * FN(gl_w)[q] * Q.f[q] * Q.t[q]);
                            }
                        REAL gol[3], gdl[3];
                        for (int c = 0; c < 3; ++c) {
                            gol[c] = gog[c] * Q.is[c];
                            gdl[c] = gdg[c] * Q.is[c];
                            a[3 + c] += gog[c] * (-Q.og[c] * Q.is[c]) + gdg[c] * (-Q.dg[c] * Q.is[c]);
                        }
                        for (int r = 0; r < 3; ++r) {
                            a[r] += -(R[r * 3] * gol[0] + R[r * 3 + 1] * gol[1] + R[r * 3 + 2] * gol[2]);
                            for (int c = 0; c < 3; ++c) dR[r * 3 + c] += gol[c] * Q.diff[r] + gdl[c] * pg.rd[r];
                        }
                    }
                }
                if (v & 2) {
                    REAL P[9], d[3];
                    FN(prec)(s, R, P);
                    const REAL w = FN(weight)(pg.p, mu, P, d);
                    const REAL* c = sh + 4 * (int64_t)g;
                    const REAL I = c[0] + c[1] * pg.rd[0] + c[2] * pg.rd[1] + c[3] * pg.rd[2];
                    a[11] += dnum * w;
                    a[12] += dnum * w * pg.rd[0];
                    a[13] += dnum * w * pg.rd[1];
                    a[14] += dnum * w * pg.rd[2];
                    const REAL dw = dnum * I + dden + dS;
                    const REAL dQ = dw * w * (REAL)-0.5;
                    REAL Gm[9];
                    for (int r = 0; r < 3; ++r) {
                        const REAL vr = P[r * 3] * d[0] + P[r * 3 + 1] * d[1] + P[r * 3 + 2] * d[2];
                        a[r] += dQ * (-2 * vr);
                        for (int cc = 0; cc < 3; ++cc) Gm[r * 3 + cc] = dQ * d[r] * d[cc];
                    }
                    /* dL/dP -> dL/dR, dL/ds for P = R diag(1/s^2) R^T */
                    const REAL dd[3] = {1 / (s[0] * s[0]), 1 / (s[1] * s[1]), 1 / (s[2] * s[2])};
                    for (int r = 0; r < 3; ++r)
                        for (int kk = 0; kk < 3; ++kk) {
                            REAL t = 0;
                            for (int j = 0; j < 3; ++j) t += (Gm[r * 3 + j] + Gm[j * 3 + r]) * R[j * 3 + kk];
                            dR[r * 3 + kk] += t * dd[kk];
                        }
                    for (int kk = 0; kk < 3; ++kk) {
                        REAL t = 0;
                        for (int i2 = 0; i2 < 3; ++i2)
                            for (int j = 0; j < 3; ++j) t += R[i2 * 3 + kk] * Gm[i2 * 3 + j] * R[j * 3 + kk];
                        a[3 + kk] += -2 * t * dd[kk] / s[kk];
                    }
                }
                REAL gq[4];
                FN(quat_grad)(quats + 4 * (int64_t)g, dR, gq);
                for (int c = 0; c < 4; ++c) a[6 + c] += gq[c];
            }
        }
    }
    for (int64_t g = 0; g < G; ++g) {
        REAL t[NF];
        for (int f = 0; f < NF; ++f) t[f] = 0;
        for (int th = 0; th < nt; ++th)
            for (int f = 0; f < NF; ++f) t[f] += acc[((size_t)th * (size_t)G + (size_t)g) * NF + f];
        for (int c = 0; c < 3; ++c) {
            dm[3 * g + c] = t[c];
            ds[3 * g + c] = t[3 + c];
        }
        for (int c = 0; c < 4; ++c) {
            dq[4 * g + c] = t[6 + c];
            dsh[4 * g + c] = t[11 + c];
        }
        da[g] = t[10];
    }
    free(acc);
}

#undef FN
#undef CAT
#undef CAT2
