/*
 * TEST INFRASTRUCTURE ONLY — checker for the slice-adapted 3DGS tests; nothing in the
 * product links or calls it. Restatement of the reference's bounded additive splat
 * (ops/slice_adapted_3dgs_renderer/src/render.cu:158-600) in fp32 and fp64: pixel mapping,
 * bounding boxes, 16x16 tile binning (keys tile << 32, stable -> Gaussian order), forward
 * per pixel over its tile list, backward per (pixel, Gaussian) pair.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static int32_t sao_i32(double x) {
    if (x != x) return 0;
    if (x >= 2147483647.0) return 2147483647;
    if (x <= -2147483648.0) return (int32_t)-2147483647 - 1;
    return (int32_t)x;
}

#define SAO_TILE 16

#define SAO_BODY(REAL, SUF, FMAX, SQRT, FLOOR, CEIL, EXP)                                                              \
    static REAL sao_px_##SUF(int x, int W, REAL hw) { return W <= 1 ? 0 : -hw + (2 * hw) * (REAL)x / (REAL)(W - 1); } \
    static void sao_bbox_##SUF(const REAL* inv, REAL mx, REAL my, int H, int W, REAL hw, REAL hh, REAL rs, int* b) {  \
        REAL det = inv[0] * inv[3] - inv[1] * inv[2];                                                                  \
        det = FMAX(det, (REAL)1e-8);                                                                                   \
        const REAL sx_ = SQRT(FMAX(inv[3] / det, (REAL)1e-8)), sy_ = SQRT(FMAX(inv[0] / det, (REAL)1e-8));            \
        const REAL rx = rs * sx_, ry = rs * sy_;                                                                       \
        const REAL kx = W > 1 ? (REAL)(W - 1) / (2 * hw) : 0, ky = H > 1 ? (REAL)(H - 1) / (2 * hh) : 0;               \
        int x0 = sao_i32((double)FLOOR((mx - rx + hw) * kx)), x1 = sao_i32((double)CEIL((mx + rx + hw) * kx));         \
        int y0 = sao_i32((double)FLOOR((my - ry + hh) * ky)), y1 = sao_i32((double)CEIL((my + ry + hh) * ky));         \
        b[0] = x0 > 0 ? x0 : 0;                                                                                        \
        b[1] = y0 > 0 ? y0 : 0;                                                                                        \
        b[2] = x1 < W - 1 ? x1 : W - 1;                                                                                \
        b[3] = y1 < H - 1 ? y1 : H - 1;                                                                                \
    }                                                                                                                  \
    /* tile lists in Gaussian order; rs/re -1 for empty tiles; ids sized by the caller */                            \
    int64_t sao_bin_##SUF(int64_t N, int H, int W, REAL hw, REAL hh, const REAL* means, const REAL* inv, REAL rsig,   \
                          int32_t* bbox, int32_t* rs, int32_t* re, int32_t* ids, int64_t ids_cap) {                    \
        const int gw = (W + SAO_TILE - 1) / SAO_TILE, gh = (H + SAO_TILE - 1) / SAO_TILE, T = gw * gh;               \
        int64_t* cnt = (int64_t*)calloc((size_t)T + 1, sizeof(int64_t));                                              \
        int32_t* rect = (int32_t*)calloc((size_t)4 * (N > 0 ? N : 1), sizeof(int32_t));                               \
        for (int64_t g = 0; g < N; ++g) {                                                                              \
            int* b = bbox + 4 * g;                                                                                     \
            sao_bbox_##SUF(inv + 4 * g, means[2 * g], means[2 * g + 1], H, W, hw, hh, rsig, b);                        \
            if (b[2] < b[0] || b[3] < b[1]) continue;                                                                  \
            int x0 = b[0] / SAO_TILE, y0 = b[1] / SAO_TILE, x1 = b[2] / SAO_TILE + 1, y1 = b[3] / SAO_TILE + 1;       \
            x0 = x0 > 0 ? x0 : 0; y0 = y0 > 0 ? y0 : 0; x1 = x1 < gw ? x1 : gw; y1 = y1 < gh ? y1 : gh;                \
            if (x0 >= x1 || y0 >= y1) continue;                                                                        \
            rect[4 * g] = x0; rect[4 * g + 1] = y0; rect[4 * g + 2] = x1; rect[4 * g + 3] = y1;                        \
            for (int y = y0; y < y1; ++y)                                                                              \
                for (int x = x0; x < x1; ++x) cnt[y * gw + x + 1]++;                                                   \
        }                                                                                                              \
        for (int t = 0; t < T; ++t) cnt[t + 1] += cnt[t];                                                              \
        for (int t = 0; t < T; ++t) {                                                                                  \
            rs[t] = cnt[t + 1] > cnt[t] ? (int32_t)cnt[t] : -1;                                                        \
            re[t] = cnt[t + 1] > cnt[t] ? (int32_t)cnt[t + 1] : -1;                                                    \
        }                                                                                                              \
        int64_t total = cnt[T];                                                                                        \
        if (ids && total <= ids_cap) {                                                                                 \
            int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)T);                                              \
            for (int t = 0; t < T; ++t) cur[t] = cnt[t];                                                               \
            for (int64_t g = 0; g < N; ++g) {                                                                          \
                const int32_t* r = rect + 4 * g;                                                                       \
                for (int y = r[1]; y < r[3]; ++y)                                                                      \
                    for (int x = r[0]; x < r[2]; ++x) ids[cur[y * gw + x]++] = (int32_t)g;                             \
            }                                                                                                          \
            free(cur);                                                                                                 \
        }                                                                                                              \
        free(rect);                                                                                                    \
        free(cnt);                                                                                                     \
        return total;                                                                                                  \
    }                                                                                                                  \
    void sao_forward_##SUF(int H, int W, REAL hw, REAL hh, const REAL* means, const REAL* inv, const REAL* weights,   \
                           const REAL* colors, REAL rsig, const int32_t* rs, const int32_t* re, const int32_t* ids,   \
                           REAL* image, REAL* alpha) {                                                                 \
        const int gw = (W + SAO_TILE - 1) / SAO_TILE;                                                                  \
        const REAL r2 = rsig * rsig;                                                                                   \
        for (int64_t p = 0; p < (int64_t)H * W; ++p) {                                                                 \
            const int x = (int)(p % W), y = (int)(p / W);                                                              \
            const int t = (y / SAO_TILE) * gw + x / SAO_TILE;                                                          \
            const REAL px = sao_px_##SUF(x, W, hw), py = sao_px_##SUF(y, H, hh);                                       \
            REAL o[4] = {0, 0, 0, 0};                                                                                  \
            if (rs[t] >= 0)                                                                                            \
                for (int i = rs[t]; i < re[t]; ++i) {                                                                  \
                    const int g = ids[i];                                                                              \
                    const REAL* iv = inv + 4 * (int64_t)g;                                                             \
                    const REAL dx = px - means[2 * g], dy = py - means[2 * g + 1];                                     \
                    const REAL quad = dx * (iv[0] * dx + iv[1] * dy) + dy * (iv[2] * dx + iv[3] * dy);                 \
                    if (quad > r2) continue;                                                                           \
                    REAL power = (REAL)-0.5 * quad;                                                                    \
                    if (power < (REAL)-50) continue;                                                                   \
                    if (power > 0) power = 0;                                                                          \
                    const REAL w = EXP(power) * weights[g];                                                            \
                    for (int c = 0; c < 3; ++c) o[c] += w * colors[3 * g + c];                                         \
                    o[3] += w;                                                                                         \
                }                                                                                                      \
            for (int c = 0; c < 3; ++c) image[3 * p + c] = o[c];                                                       \
            alpha[p] = o[3];                                                                                           \
        }                                                                                                              \
    }                                                                                                                  \
    void sao_backward_##SUF(int64_t N, int H, int W, REAL hw, REAL hh, const REAL* means, const REAL* inv,            \
                            const REAL* weights, const REAL* colors, REAL rsig, const int32_t* rs, const int32_t* re, \
                            const int32_t* ids, const REAL* gimg, const REAL* galpha, REAL* dm, REAL* di, REAL* dw,   \
                            REAL* dc) {                                                                                \
        memset(dm, 0, sizeof(REAL) * 2 * N);                                                                           \
        memset(di, 0, sizeof(REAL) * 4 * N);                                                                           \
        memset(dw, 0, sizeof(REAL) * N);                                                                               \
        memset(dc, 0, sizeof(REAL) * 3 * N);                                                                           \
        const int gw = (W + SAO_TILE - 1) / SAO_TILE;                                                                  \
        const REAL r2 = rsig * rsig;                                                                                   \
        for (int64_t p = 0; p < (int64_t)H * W; ++p) {                                                                 \
            const int x = (int)(p % W), y = (int)(p / W);                                                              \
            const int t = (y / SAO_TILE) * gw + x / SAO_TILE;                                                          \
            if (rs[t] < 0) continue;                                                                                   \
            const REAL px = sao_px_##SUF(x, W, hw), py = sao_px_##SUF(y, H, hh);                                       \
            const REAL* go = gimg + 3 * p;                                                                             \
            const REAL ga = galpha[p];                                                                                 \
            for (int i = rs[t]; i < re[t]; ++i) {                                                                      \
                const int g = ids[i];                                                                                  \
                const REAL* iv = inv + 4 * (int64_t)g;                                                                 \
                const REAL dx = px - means[2 * g], dy = py - means[2 * g + 1];                                         \
                const REAL quad = dx * (iv[0] * dx + iv[1] * dy) + dy * (iv[2] * dx + iv[3] * dy);                     \
                if (quad > r2) continue;                                                                               \
                REAL power = (REAL)-0.5 * quad;                                                                        \
                if (power < (REAL)-50) continue;                                                                       \
                if (power > 0) power = 0;                                                                              \
                const REAL e = EXP(power), wt = weights[g];                                                            \
                const REAL dot = go[0] * colors[3 * g] + go[1] * colors[3 * g + 1] + go[2] * colors[3 * g + 2];       \
                dw[g] += e * (dot + ga);                                                                               \
                for (int c = 0; c < 3; ++c) dc[3 * g + c] += e * wt * go[c];                                           \
                const REAL dpow = wt * (dot + ga) * e, cm = (REAL)-0.5 * dpow;                                         \
                di[4 * g] += cm * dx * dx;                                                                             \
                di[4 * g + 1] += cm * dx * dy;                                                                         \
                di[4 * g + 2] += cm * dy * dx;                                                                         \
                di[4 * g + 3] += cm * dy * dy;                                                                         \
                dm[2 * g] += (REAL)0.5 * dpow * ((iv[0] + iv[0]) * dx + (iv[1] + iv[2]) * dy);                         \
                dm[2 * g + 1] += (REAL)0.5 * dpow * ((iv[2] + iv[1]) * dx + (iv[3] + iv[3]) * dy);                     \
            }                                                                                                          \
        }                                                                                                              \
    }

SAO_BODY(float, f32, fmaxf, sqrtf, floorf, ceilf, expf)
SAO_BODY(double, f64, fmax, sqrt, floor, ceil, exp)
