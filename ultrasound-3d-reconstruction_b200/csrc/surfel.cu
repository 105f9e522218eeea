// UltraGS baseline: 2D-Gaussian-surfel rasterisation (ray-splat intersection, front-to-back
// alpha compositing, seven auxiliary maps) with its backward.
//
// Reference behaviour restated here (paths inside KevinWCCC/ultrasound-3d-reconstruction,
// ops/ultrags_baseline_renderer):
//   cuda_rasterizer/forward.cu:20-65       SH -> RGB (degree-2 "ultrasound" terms), clamp
//   cuda_rasterizer/forward.cu:69-107      splat-to-pixel homography T = S2W^T * W2N * N2P
//   cuda_rasterizer/forward.cu:109-139     screen-space AABB of the 3-sigma ellipse
//   cuda_rasterizer/forward.cu:141-246     preprocess: near cull, dual-visible normal, radius
//   cuda_rasterizer/forward.cu:249-439     tile compositing, early termination, aux maps
//   cuda_rasterizer/rasterizer_impl.cu:70-137  keys (tile << 32 | depth bits), tile ranges
//   cuda_rasterizer/backward.cu:103-404    back-to-front replay and per-pair gradients
//   cuda_rasterizer/backward.cu:406-602    homography / AABB / rotation / SH gradients
//
// B200 design. Binning puts every (tile, Gaussian) instance into its tile's bucket and orders
// each bucket in shared memory by (depth bits, Gaussian index), the order the reference's
// stable radix sort produces. The forward stages 256 80-byte records per batch and gives
// each thread one pixel. The backward keeps the reference's per-pixel back-to-front replay
// (its recurrences need it) but replaces the per-pair float atomics by a fixed-order
// reduction: per staged Gaussian, each warp reduces its 32 pixels' 18 gradient terms with a
// transposed butterfly (27 shuffles), the 8 warp sums are added in warp order into one
// per-instance partial, and one thread per Gaussian sums its instances in order and runs
// the preprocess backward in the same kernel. Results are deterministic.
//
// Matrix products are evaluated with the summation order of the GLM operators the
// reference uses (column-major, k ascending, zero entries included), so that pixel
// rectangles, keys and contributor counts agree bit for bit under the same compiler flags.
#include "us3d_common.cuh"
#include "scan.cuh"
#include "binning.cuh"

namespace us3d {
namespace gs {

constexpr int TILE = 16;
constexpr int BLOCK = TILE * TILE;
constexpr int REC_F4 = 5;        // 80-byte per-Gaussian render record
constexpr int BWD_BATCH = 64;    // Gaussians staged per backward batch
constexpr int NGRAD = 18;        // per-instance gradient terms
constexpr int PARTIAL_F4 = 5;    // 20 floats per instance partial (2 pad)
constexpr float NEAR_N = 0.2f;
constexpr float FAR_N = 100.0f;
constexpr float FILTER_SIZE = 0.707106f;
constexpr float FILTER_INV_SQUARE = 2.0f;
constexpr float SH_C0 = 0.28209479177387814f;
constexpr float SH_C1 = 0.4886025119029199f;
enum { FLAG_PREFILTERED = 4 };

// Column-major small matrix: m[c][r] is column c, row r (C columns, R rows).
template <int C, int R>
struct Mat {
    float m[C][R];
};

// (C1 x R1) * (C2 x C1): out[c][r] = sum_k a[k][r] * b[c][k], k ascending, left to right.
template <int C1, int R1, int C2>
__device__ __forceinline__ Mat<C2, R1> mmul(const Mat<C1, R1>& a, const Mat<C2, C1>& b) {
    Mat<C2, R1> o;
#pragma unroll
    for (int c = 0; c < C2; ++c)
#pragma unroll
        for (int r = 0; r < R1; ++r) {
            float acc = a.m[0][r] * b.m[c][0];
#pragma unroll
            for (int k = 1; k < C1; ++k) acc = acc + a.m[k][r] * b.m[c][k];
            o.m[c][r] = acc;
        }
    return o;
}

template <int C, int R>
__device__ __forceinline__ Mat<R, C> transpose(const Mat<C, R>& a) {
    Mat<R, C> o;
#pragma unroll
    for (int c = 0; c < C; ++c)
#pragma unroll
        for (int r = 0; r < R; ++r) o.m[r][c] = a.m[c][r];
    return o;
}

struct V3 {
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{x, y, z}; }
__device__ __forceinline__ V3 vmul(const V3 a, const V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ V3 vscale(float s, const V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
__device__ __forceinline__ V3 vadd(const V3 a, const V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 vsub(const V3 a, const V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
// Dot product as a product vector summed x + y + z (the GLM form).
__device__ __forceinline__ float vdot(const V3 a, const V3 b) {
    const V3 t = vmul(a, b);
    return t.x + t.y + t.z;
}
__device__ __forceinline__ V3 vcross(const V3 a, const V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ V3 col3(const Mat<3, 3>& a, int c) { return v3(a.m[c][0], a.m[c][1], a.m[c][2]); }

// Rotation of the (w,x,y,z) quaternion stored as (q.x, q.y, q.z, q.w), column-major
// (gsplat's quat_to_rotmat, reference auxiliary.h:199-222).
__device__ __forceinline__ Mat<3, 3> quat_rot(const float4 q) {
    const float s = rsqrtf(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    const float w = q.x * s, x = q.y * s, y = q.z * s, z = q.w * s;
    Mat<3, 3> R;
    R.m[0][0] = 1.f - 2.f * (y * y + z * z);
    R.m[0][1] = 2.f * (x * y + w * z);
    R.m[0][2] = 2.f * (x * z - w * y);
    R.m[1][0] = 2.f * (x * y - w * z);
    R.m[1][1] = 1.f - 2.f * (x * x + z * z);
    R.m[1][2] = 2.f * (y * z + w * x);
    R.m[2][0] = 2.f * (x * z + w * y);
    R.m[2][1] = 2.f * (y * z - w * x);
    R.m[2][2] = 1.f - 2.f * (x * x + y * y);
    return R;
}

// Vector-Jacobian product of quat_rot given dL/dR (column-major), returned in the same
// (w,x,y,z)-in-(x,y,z,w) storage (reference auxiliary.h:225-271).
__device__ __forceinline__ float4 quat_rot_vjp(const float4 q, const Mat<3, 3>& g) {
    const float s = rsqrtf(q.w * q.w + q.x * q.x + q.y * q.y + q.z * q.z);
    const float w = q.x * s, x = q.y * s, y = q.z * s, z = q.w * s;
    float4 o;
    o.x = 2.f * (x * (g.m[1][2] - g.m[2][1]) + y * (g.m[2][0] - g.m[0][2]) + z * (g.m[0][1] - g.m[1][0]));
    o.y = 2.f * (-2.f * x * (g.m[1][1] + g.m[2][2]) + y * (g.m[0][1] + g.m[1][0]) + z * (g.m[0][2] + g.m[2][0]) +
                 w * (g.m[1][2] - g.m[2][1]));
    o.z = 2.f * (x * (g.m[0][1] + g.m[1][0]) - 2.f * y * (g.m[0][0] + g.m[2][2]) + z * (g.m[1][2] + g.m[2][1]) +
                 w * (g.m[2][0] - g.m[0][2]));
    o.w = 2.f * (x * (g.m[0][2] + g.m[2][0]) + y * (g.m[1][2] + g.m[2][1]) - 2.f * z * (g.m[0][0] + g.m[1][1]) +
                 w * (g.m[0][1] - g.m[1][0]));
    return o;
}

__device__ __forceinline__ Mat<3, 3> scale_mat(float sx, float sy, float mod) {
    Mat<3, 3> S;
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int r = 0; r < 3; ++r) S.m[c][r] = (c == r) ? 1.f : 0.f;
    S.m[0][0] = mod * sx;
    S.m[1][1] = mod * sy;
    return S;
}

// world -> NDC as a column-major 4x4 from the row-major projection array.
__device__ __forceinline__ Mat<4, 4> world2ndc(const float* pm) {
    Mat<4, 4> w;
#pragma unroll
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int r = 0; r < 4; ++r) w.m[c][r] = pm[4 * r + c];
    return w;
}

__device__ __forceinline__ Mat<3, 4> ndc2pix(int W, int H) {
    Mat<3, 4> n;
    n.m[0][0] = (float)((double)W / 2.0); n.m[0][1] = 0.f; n.m[0][2] = 0.f; n.m[0][3] = (float)((double)(W - 1) / 2.0);
    n.m[1][0] = 0.f; n.m[1][1] = (float)((double)H / 2.0); n.m[1][2] = 0.f; n.m[1][3] = (float)((double)(H - 1) / 2.0);
    n.m[2][0] = 0.f; n.m[2][1] = 0.f; n.m[2][2] = 0.f; n.m[2][3] = 1.f;
    return n;
}

__device__ __forceinline__ Mat<3, 4> splat2world(const Mat<3, 3>& L, const float3 p) {
    Mat<3, 4> s;
    s.m[0][0] = L.m[0][0]; s.m[0][1] = L.m[0][1]; s.m[0][2] = L.m[0][2]; s.m[0][3] = 0.f;
    s.m[1][0] = L.m[1][0]; s.m[1][1] = L.m[1][1]; s.m[1][2] = L.m[1][2]; s.m[1][3] = 0.f;
    s.m[2][0] = p.x; s.m[2][1] = p.y; s.m[2][2] = p.z; s.m[2][3] = 1.f;
    return s;
}

__device__ __forceinline__ float3 xform_point(const float3 p, const float* m) {
    return make_float3(m[0] * p.x + m[4] * p.y + m[8] * p.z + m[12], m[1] * p.x + m[5] * p.y + m[9] * p.z + m[13],
                       m[2] * p.x + m[6] * p.y + m[10] * p.z + m[14]);
}
__device__ __forceinline__ V3 xform_vec(const V3 p, const float* m) {
    return v3(m[0] * p.x + m[4] * p.y + m[8] * p.z, m[1] * p.x + m[5] * p.y + m[9] * p.z,
              m[2] * p.x + m[6] * p.y + m[10] * p.z);
}
__device__ __forceinline__ V3 xform_vec_t(const V3 p, const float* m) {
    return v3(m[0] * p.x + m[1] * p.y + m[2] * p.z, m[4] * p.x + m[5] * p.y + m[6] * p.z,
              m[8] * p.x + m[9] * p.y + m[10] * p.z);
}

// SH colour with the reference's degree-2 "ultrasound" terms (forward.cu:20-65).
// Returns the clamp flags as bits 0..2.
__device__ __forceinline__ int sh_color(int g, int deg, int M, const float* means, const float* campos,
                                        const float* shs, float* rgb) {
    const V3 pos = v3(means[3 * g], means[3 * g + 1], means[3 * g + 2]);
    V3 dir = vsub(pos, v3(campos[0], campos[1], campos[2]));
    const float len = sqrtf(vdot(dir, dir));
    dir = v3(dir.x / len, dir.y / len, dir.z / len);
    const float* sh = shs + (int64_t)g * M * 3;
    auto c = [&](int k) { return v3(sh[3 * k], sh[3 * k + 1], sh[3 * k + 2]); };
    V3 res = vscale(SH_C0, c(0));
    if (deg > 0) {
        const float x = dir.x, y = dir.y, z = dir.z;
        res = vsub(vadd(vsub(res, vscale(SH_C1 * y, c(1))), vscale(SH_C1 * z, c(2))), vscale(SH_C1 * x, c(3)));
        if (deg > 1) {
            const float depth = x;
            const float refl_var = x * x + y * y + z * z;
            const float sc_x = x * y, sc_y = z * y, sc_z = x * z;
            const float att = __expf(-depth);
            const float refl = -refl_var;
            res = vsub(vadd(vsub(vadd(vsub(res, vscale(att, c(4))), vscale(refl, c(5))), vscale(sc_z, c(6))),
                            vscale(sc_x, c(7))),
                       vscale(sc_y, c(8)));
        }
    }
    res = v3(res.x + 0.5f, res.y + 0.5f, res.z + 0.5f);
    const int clamped = (res.x < 0) | ((res.y < 0) << 1) | ((res.z < 0) << 2);
    rgb[0] = fmaxf(res.x, 0.0f);
    rgb[1] = fmaxf(res.y, 0.0f);
    rgb[2] = fmaxf(res.z, 0.0f);
    return clamped;
}

struct Workspace {
    long long* header;
    float4* rec;           // G x 5
    float* depth;          // G (view depth, key bits)
    int4* rect;            // G tile rectangle [x0, y0, x1, y1)
    int* clamped;          // G (bits 0..2)
    int* touched;          // G
    int* inst_offset;      // G + 1
    long long* bs_g;
    int* tile_count;       // T
    int* tile_start;       // T + 1
    int* tile_cursor;      // T
    long long* bs_t;
    unsigned long long* keys;
    int* slot_inst;
    int* sorted_gid;
    int* sorted_inst;
    float* accum;          // 3P: final T, M1, M2
    uint32_t* n_contrib;   // 2P: last contributor, median contributor
    size_t bytes;
};

static Workspace carve(void* base, int64_t G, int64_t T, int64_t P, int64_t cap) {
    Carver c(base);
    Workspace w;
    w.header = c.take<long long>(H_WORDS);
    w.rec = c.take<float4>((size_t)G * REC_F4);
    w.depth = c.take<float>((size_t)G);
    w.rect = c.take<int4>((size_t)G);
    w.clamped = c.take<int>((size_t)G);
    w.touched = c.take<int>((size_t)G);
    w.inst_offset = c.take<int>((size_t)G + 1);
    w.bs_g = c.take<long long>((size_t)scan_num_blocks(G) + 1);
    w.tile_count = c.take<int>((size_t)T);
    w.tile_start = c.take<int>((size_t)T + 1);
    w.tile_cursor = c.take<int>((size_t)T);
    w.bs_t = c.take<long long>((size_t)scan_num_blocks(T) + 1);
    w.keys = c.take<unsigned long long>((size_t)cap);
    w.slot_inst = c.take<int>((size_t)cap);
    w.sorted_gid = c.take<int>((size_t)cap);
    w.sorted_inst = c.take<int>((size_t)cap);
    w.accum = c.take<float>((size_t)P * 3);
    w.n_contrib = c.take<uint32_t>((size_t)P * 2);
    w.bytes = align_up(c.off, 256);
    return w;
}

struct Params {
    int P, D, M, W, H, gx, gy;
    float scale_modifier;
    int prefiltered;
    const float* means;
    const float* shs;
    const float* colors;
    const float* opacities;
    const float* scales;
    const float* rotations;
    const float* transmat;
    const float* view;
    const float* proj;
    const float* campos;
};

// ------------------------------------------------------------------------------------
// Preprocess + binning
// ------------------------------------------------------------------------------------

__global__ void init_kernel(int64_t T, int* __restrict__ tile_count, int* __restrict__ tile_cursor,
                            long long* __restrict__ header, int64_t cap, int64_t G, int64_t P) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < H_WORDS) {
        long long v = 0;
        if (threadIdx.x == H_CAP) v = cap;
        if (threadIdx.x == H_G) v = G;
        if (threadIdx.x == H_T) v = T;
        if (threadIdx.x == H_P) v = P;
        header[threadIdx.x] = v;
    }
    if (t >= T) return;
    tile_count[t] = 0;
    tile_cursor[t] = 0;
}

// Per Gaussian: near cull, homography, dual-visible normal, AABB radius, tile rectangle,
// colour, render record, per-tile counts (forward.cu:141-246).
__global__ void __launch_bounds__(256)
preprocess_kernel(Params p, int* __restrict__ radii, float4* __restrict__ rec, float* __restrict__ depth_out,
                  int4* __restrict__ rect_out, int* __restrict__ clamped_out, int* __restrict__ touched,
                  int* __restrict__ tile_count, long long* __restrict__ header) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= p.P) return;
    radii[g] = 0;
    touched[g] = 0;
    clamped_out[g] = 0;
    rect_out[g] = make_int4(0, 0, 0, 0);
    const float3 po = make_float3(p.means[3 * g], p.means[3 * g + 1], p.means[3 * g + 2]);
    const float3 pv = xform_point(po, p.view);
    if (pv.z <= 0.2f) {
        if (p.prefiltered) atomicOr(reinterpret_cast<unsigned long long*>(header + H_FLAGS), (unsigned long long)FLAG_PREFILTERED);
        return;
    }
    Mat<3, 3> T;
    V3 normal;
    if (p.transmat == nullptr) {
        const float4 q = make_float4(p.rotations[4 * g], p.rotations[4 * g + 1], p.rotations[4 * g + 2],
                                     p.rotations[4 * g + 3]);
        const Mat<3, 3> R = quat_rot(q);
        const Mat<3, 3> S = scale_mat(p.scales[2 * g], p.scales[2 * g + 1], p.scale_modifier);
        const Mat<3, 3> L = mmul(R, S);
        const Mat<4, 3> A = mmul(transpose(splat2world(L, po)), world2ndc(p.proj));
        T = mmul(A, ndc2pix(p.W, p.H));
        normal = xform_vec(col3(L, 2), p.view);
    } else {
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r) T.m[c][r] = p.transmat[9 * g + 3 * c + r];
        normal = v3(0.f, 0.f, 1.f);
    }
    // dual-visible: orient the normal towards the camera
    const float cosv = -(pv.x * normal.x + pv.y * normal.y + pv.z * normal.z);
    if (cosv == 0) return;
    const float mult = cosv > 0 ? 1.f : -1.f;
    normal = vscale(mult, normal);
    // AABB of the cutoff ellipse (forward.cu:109-139), cutoff 3
    const float cutoff = 3.0f;
    const V3 t = v3(cutoff * cutoff, cutoff * cutoff, -1.0f);
    const V3 T0 = col3(T, 0), T1 = col3(T, 1), T2 = col3(T, 2);
    const float d = vdot(t, vmul(T2, T2));
    if (d == 0.0f) return;
    const V3 f = vscale(1.0f / d, t);
    const float px = vdot(f, vmul(T0, T2)), py = vdot(f, vmul(T1, T2));
    const float h0x = px * px - vdot(f, vmul(T0, T0));
    const float h0y = py * py - vdot(f, vmul(T1, T1));
    const float hx = sqrtf((1e-4f < h0x) ? h0x : 1e-4f);
    const float hy = sqrtf((1e-4f < h0y) ? h0y : 1e-4f);
    const float radius = ceilf(fmaxf(fmaxf(hx, hy), cutoff * FILTER_SIZE));
    const int r = (int)radius;
    const int x0 = min(p.gx, max(0, (int)((px - (float)r) / (float)TILE)));
    const int y0 = min(p.gy, max(0, (int)((py - (float)r) / (float)TILE)));
    const int x1 = min(p.gx, max(0, (int)((((px + (float)r) + (float)TILE) - 1.0f) / (float)TILE)));
    const int y1 = min(p.gy, max(0, (int)((((py + (float)r) + (float)TILE) - 1.0f) / (float)TILE)));
    if ((x1 - x0) * (y1 - y0) == 0) return;
    float rgb[3];
    int clamped = 0;
    if (p.colors == nullptr) {
        clamped = sh_color(g, p.D, p.M, p.means, p.campos, p.shs, rgb);
    } else {
        rgb[0] = p.colors[3 * g];
        rgb[1] = p.colors[3 * g + 1];
        rgb[2] = p.colors[3 * g + 2];
    }
    clamped_out[g] = clamped;
    depth_out[g] = pv.z;
    radii[g] = r;
    float4* o = rec + (int64_t)REC_F4 * g;
    o[0] = make_float4(T0.x, T0.y, T0.z, px);
    o[1] = make_float4(T1.x, T1.y, T1.z, py);
    o[2] = make_float4(T2.x, T2.y, T2.z, p.opacities[g]);
    o[3] = make_float4(normal.x, normal.y, normal.z, rgb[0]);
    o[4] = make_float4(rgb[1], rgb[2], 0.f, 0.f);
    rect_out[g] = make_int4(x0, y0, x1, y1);
    touched[g] = (x1 - x0) * (y1 - y0);
    (void)tile_count;  // counted per block by rect_count_kernel
}

__global__ void check_kernel(long long* __restrict__ header, int64_t cap) {
    const long long tg = header[H_SCAN_G], tt = header[H_SCAN_T];
    long long flags = header[H_FLAGS];
    if (tg != tt) flags |= FLAG_TABLE;
    if (tg > cap || tg > 0x7fffffffLL) flags |= FLAG_OVERFLOW;
    header[H_TOTAL] = tg;
    header[H_FLAGS] = flags;
}


// ------------------------------------------------------------------------------------
// Forward compositing
// ------------------------------------------------------------------------------------

// Ray-splat intersection of pixel (pxf, pyf) with the splat of homography rows Tu, Tv, Tw
// (forward.cu:335-350). Returns false when the pair is skipped before alpha.
struct Hit {
    V3 k, l, p;
    float sx, sy, rho3d, rho2d, dx, dy, depth;
};

__device__ __forceinline__ bool intersect(float pxf, float pyf, const float4 r0, const float4 r1, const float4 r2,
                                          Hit& h) {
    const V3 Tu = v3(r0.x, r0.y, r0.z), Tv = v3(r1.x, r1.y, r1.z), Tw = v3(r2.x, r2.y, r2.z);
    h.k = vsub(vscale(pxf, Tw), Tu);
    h.l = vsub(vscale(pyf, Tw), Tv);
    h.p = vcross(h.k, h.l);
    if (h.p.z == 0.0f) return false;
    h.sx = h.p.x / h.p.z;
    h.sy = h.p.y / h.p.z;
    h.rho3d = h.sx * h.sx + h.sy * h.sy;
    h.dx = r0.w - pxf;
    h.dy = r1.w - pyf;
    h.rho2d = FILTER_INV_SQUARE * (h.dx * h.dx + h.dy * h.dy);
    h.depth = (h.sx * Tw.x + h.sy * Tw.y) + Tw.z;
    return !(h.depth < NEAR_N);
}

// Asynchronous global -> shared copies (cp.async, sm_80 and later): the next batch of render
// records is gathered into the second staging buffer while the current one is shaded.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

__global__ void __launch_bounds__(BLOCK)
forward_kernel(int W, int H, int gx, const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
               const long long* __restrict__ header, const float4* __restrict__ rec, const float* __restrict__ bg,
               float* __restrict__ out_color, float* __restrict__ out_others, float* __restrict__ accum,
               uint32_t* __restrict__ n_contrib) {
    __shared__ float4 s_rec[2][REC_F4][BLOCK];  // double-buffered staging
    if (header[H_FLAGS] != 0) return;
    const int tile = blockIdx.x;
    const int tx = tile % gx, ty = tile / gx;
    const int lx = threadIdx.x % TILE, ly = threadIdx.x / TILE;
    const uint32_t pxi = (uint32_t)(tx * TILE + lx), pyi = (uint32_t)(ty * TILE + ly);
    const bool inside = pxi < (uint32_t)W && pyi < (uint32_t)H;
    const float pxf = (float)pxi, pyf = (float)pyi;
    bool done = !inside;
    const int s0 = tile_start[tile], n = tile_start[tile + 1] - s0;
    const int rounds = (n + BLOCK - 1) / BLOCK;
    int todo = n;
    float T = 1.0f;
    uint32_t contributor = 0, last_contributor = 0;
    float C[3] = {0.f, 0.f, 0.f};
    float N[3] = {0.f, 0.f, 0.f};
    float D = 0.f, M1 = 0.f, M2 = 0.f, distortion = 0.f, median_depth = 0.f, median_contributor = -1.f;
    const float mscale = FAR_N / (FAR_N - NEAR_N);
    // round i's records go to buffer i & 1; the copies of round i + 1 are issued once every
    // thread has passed round i's barrier (so nobody still reads that buffer from round i - 1)
    // and run while round i is shaded
    auto stage = [&](int i) {
        const int prog = i * BLOCK + threadIdx.x;
        if (prog < n) {
            const float4* r = rec + (int64_t)REC_F4 * sorted_gid[s0 + prog];
#pragma unroll
            for (int f = 0; f < REC_F4; ++f) cp_async16(&s_rec[i & 1][f][threadIdx.x], r + f);
        }
        cp_async_commit();
    };
    if (rounds > 0) stage(0);
    for (int i = 0; i < rounds; ++i, todo -= BLOCK) {
        cp_async_wait_all();  // this thread's copies of round i have landed
        if (__syncthreads_count(done) == BLOCK) break;  // ... and everyone's; no copy is in flight
        if (i + 1 < rounds) stage(i + 1);
        const float4(*sr)[BLOCK] = s_rec[i & 1];
        const int nb = min(BLOCK, todo);
        for (int j = 0; !done && j < nb; ++j) {
            ++contributor;
            const float4 r0 = sr[0][j], r1 = sr[1][j], r2 = sr[2][j];
            Hit h;
            if (!intersect(pxf, pyf, r0, r1, r2, h)) continue;
            const float rho = fminf(h.rho3d, h.rho2d);
            const float power = -0.5f * rho;
            if (power > 0.0f) continue;
            const float alpha = fminf(0.99f, r2.w * __expf(power));
            if (alpha < 1.0f / 255.0f) continue;
            const float test_T = T * (1 - alpha);
            if (test_T < 0.0001f) {
                done = true;
                continue;
            }
            const float w = alpha * T;
            const float A = 1 - T;
            const float m = mscale * (1 - NEAR_N / h.depth);
            distortion += (m * m * A + M2 - 2 * m * M1) * w;
            D += h.depth * w;
            M1 += m * w;
            M2 += m * m * w;
            if (T > 0.5) {
                median_depth = h.depth;
                median_contributor = (float)contributor;
            }
            const float4 r3 = sr[3][j], r4 = sr[4][j];
            N[0] += r3.x * w;
            N[1] += r3.y * w;
            N[2] += r3.z * w;
            C[0] += r3.w * w;
            C[1] += r4.x * w;
            C[2] += r4.y * w;
            T = test_T;
            last_contributor = contributor;
        }
    }
    if (inside) {
        const int64_t HW = (int64_t)H * W;
        const int64_t pix = (int64_t)W * pyi + pxi;
        accum[pix] = T;
        accum[pix + HW] = M1;
        accum[pix + 2 * HW] = M2;
        n_contrib[pix] = last_contributor;
        n_contrib[pix + HW] = f32_to_u32_sat(median_contributor);
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) out_color[ch * HW + pix] = C[ch] + T * bg[ch];
        out_others[pix] = D;
        out_others[pix + HW] = 1 - T;
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) out_others[pix + (2 + ch) * HW] = N[ch];
        out_others[pix + 5 * HW] = median_depth;
        out_others[pix + 6 * HW] = distortion;
    }
}

// ------------------------------------------------------------------------------------
// Backward
// ------------------------------------------------------------------------------------

// Sum of v[0..23] over the 32 lanes of a warp, transposed: on return lanes with
// (lane & 3) == 0 hold the totals of entries [3 (lane >> 2), 3 (lane >> 2) + 3) in o[0..2].
__device__ __forceinline__ void warp_reduce24(const float (&v)[24], float (&o)[3]) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    float a[12];
    const bool h16 = lane & 16;
#pragma unroll
    for (int i = 0; i < 12; ++i) {
        const float send = h16 ? v[i] : v[12 + i];
        const float keep = h16 ? v[12 + i] : v[i];
        a[i] = keep + __shfl_xor_sync(FULL, send, 16);
    }
    float b[6];
    const bool h8 = lane & 8;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
        const float send = h8 ? a[i] : a[6 + i];
        const float keep = h8 ? a[6 + i] : a[i];
        b[i] = keep + __shfl_xor_sync(FULL, send, 8);
    }
    const bool h4 = lane & 4;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float send = h4 ? b[i] : b[3 + i];
        const float keep = h4 ? b[3 + i] : b[i];
        o[i] = keep + __shfl_xor_sync(FULL, send, 4);
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        o[i] += __shfl_xor_sync(FULL, o[i], 2);
        o[i] += __shfl_xor_sync(FULL, o[i], 1);
    }
}

// One CTA per tile, one pixel per thread, Gaussians replayed back to front
// (backward.cu:103-404). Per staged Gaussian the block's 256 pixel contributions are summed
// in a fixed order into the instance's 18-term partial:
//   [0..2] dL/dTu  [3..5] dL/dTv  [6..8] dL/dTw  [9..10] dL/dmean2D  [11..13] dL/dnormal
//   [14] dL/dopacity  [15..17] dL/dcolor
__global__ void __launch_bounds__(BLOCK)
backward_kernel(int W, int H, int gx, const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
                const int* __restrict__ sorted_inst, const long long* __restrict__ header,
                const float4* __restrict__ rec, const float* __restrict__ bg, const float* __restrict__ accum,
                const uint32_t* __restrict__ n_contrib, const float* __restrict__ dL_dpix,
                const float* __restrict__ dL_dothers, float4* __restrict__ partial) {
    __shared__ float4 s_rec[2][REC_F4][BWD_BATCH];  // double-buffered staging
    __shared__ int s_inst[2][BWD_BATCH];
    __shared__ float s_red[BWD_BATCH][BLOCK / 32][NGRAD];
    __shared__ int s_last;
    if (header[H_FLAGS] != 0) return;
    const int tile = blockIdx.x;
    const int tx = tile % gx, ty = tile / gx;
    const int lx = threadIdx.x % TILE, ly = threadIdx.x / TILE;
    const uint32_t pxi = (uint32_t)(tx * TILE + lx), pyi = (uint32_t)(ty * TILE + ly);
    const bool inside = pxi < (uint32_t)W && pyi < (uint32_t)H;
    const float pxf = (float)pxi, pyf = (float)pyi;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s0 = tile_start[tile], n = tile_start[tile + 1] - s0;
    const int64_t HW = (int64_t)H * W;
    const int64_t pix = (int64_t)W * pyi + pxi;

    const float T_final = inside ? accum[pix] : 0.f;
    float T = T_final;
    const int last_contributor = inside ? (int)n_contrib[pix] : 0;
    // No pixel of the tile has a contributor at or beyond the largest last contributor: the
    // back-to-front replay starts there (its state changes only at contributors), and the
    // instances behind it get zero partials.
    if (threadIdx.x == 0) s_last = 0;
    __syncthreads();
    if (last_contributor > 0) atomicMax(&s_last, last_contributor);
    __syncthreads();
    const int n_live = min(s_last, n);
    for (int k = n_live + threadIdx.x; k < n; k += BLOCK) {
        float4* out = partial + (int64_t)PARTIAL_F4 * sorted_inst[s0 + k];
#pragma unroll
        for (int f = 0; f < PARTIAL_F4; ++f) out[f] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    uint32_t contributor = (uint32_t)n_live;
    const int median_contributor = inside ? (int)n_contrib[pix + HW] : 0;
    float dpix[3] = {0.f, 0.f, 0.f};
    float dd_depth = 0.f, dd_accum = 0.f, dd_reg = 0.f, dd_median = 0.f;
    float dd_normal[3] = {0.f, 0.f, 0.f};
    if (inside) {
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) dpix[ch] = dL_dpix[ch * HW + pix];
        dd_depth = dL_dothers[pix];
        dd_accum = dL_dothers[pix + HW];
        dd_reg = dL_dothers[pix + 6 * HW];
#pragma unroll
        for (int ch = 0; ch < 3; ++ch) dd_normal[ch] = dL_dothers[pix + (2 + ch) * HW];
        dd_median = dL_dothers[pix + 5 * HW];
    }
    const float final_D = inside ? accum[pix + HW] : 0.f;
    const float final_D2 = inside ? accum[pix + 2 * HW] : 0.f;
    const float final_A = 1 - T_final;
    float accum_rec[3] = {0.f, 0.f, 0.f}, last_color[3] = {0.f, 0.f, 0.f};
    float last_depth = 0.f, accum_depth_rec = 0.f, accum_alpha_rec = 0.f;
    float last_normal[3] = {0.f, 0.f, 0.f}, accum_normal_rec[3] = {0.f, 0.f, 0.f};
    float last_dL_dT = 0.f, last_alpha = 0.f;
    const float bg_dot_dpixel = bg[0] * dpix[0] + bg[1] * dpix[1] + bg[2] * dpix[2];
    const float mscale = FAR_N / (FAR_N - NEAR_N);

    // batch k (staged from the back of the tile list's live part) goes to buffer k & 1: thread
    // jj < BWD_BATCH copies Gaussian jj's record and instance id. The copies of batch k + 1 are
    // issued after batch k's first barrier (every thread is then done with that buffer's
    // previous batch) and run while batch k is replayed; the Gaussian index each copy needs is
    // read one batch earlier still, so no thread waits on it.
    static_assert(BWD_BATCH <= BLOCK, "one staging thread per batch entry");
    auto load_gid = [&](int b0) {
        const int jj = threadIdx.x;
        return (jj < BWD_BATCH && b0 + jj < n_live) ? sorted_gid[s0 + n_live - 1 - (b0 + jj)] : -1;
    };
    auto stage = [&](int b0, int buf, int gid) {
        const int jj = threadIdx.x;
        if (gid >= 0) {
            const float4* r = rec + (int64_t)REC_F4 * gid;
#pragma unroll
            for (int f = 0; f < REC_F4; ++f) cp_async16(&s_rec[buf][f][jj], r + f);
            cp_async4(&s_inst[buf][jj], sorted_inst + (s0 + n_live - 1 - (b0 + jj)));
        }
        cp_async_commit();
    };
    int gid_next = 0;
    if (n_live > 0) {
        stage(0, 0, load_gid(0));
        gid_next = load_gid(BWD_BATCH);
    }
    for (int b0 = 0, k = 0; b0 < n_live; b0 += BWD_BATCH, ++k) {
        const int nb = min(BWD_BATCH, n_live - b0);
        cp_async_wait_all();  // this thread's copies of batch k have landed
        __syncthreads();      // ... and everyone's; the previous batch's partials are written
        if (b0 + BWD_BATCH < n_live) {
            stage(b0 + BWD_BATCH, (k + 1) & 1, gid_next);
            gid_next = load_gid(b0 + 2 * BWD_BATCH);
        }
        const float4(*sr)[BWD_BATCH] = s_rec[k & 1];
        const int* si = s_inst[k & 1];
        for (int jj = 0; jj < nb; ++jj) {
            float v[24];
#pragma unroll
            for (int q = 0; q < 24; ++q) v[q] = 0.f;
            bool contrib = false;
            if (inside) {
                --contributor;
                if (contributor < (uint32_t)last_contributor) {
                    const float4 r0 = sr[0][jj], r1 = sr[1][jj], r2 = sr[2][jj];
                    Hit h;
                    const bool hit = intersect(pxf, pyf, r0, r1, r2, h);
                    float G = 0.f, alpha = 0.f;
                    bool ok = hit;
                    if (ok) {
                        const float rho = fminf(h.rho3d, h.rho2d);
                        const float power = -0.5f * rho;
                        if (power > 0.0f) ok = false;
                        if (ok) {
                            G = __expf(power);
                            alpha = fminf(0.99f, r2.w * G);
                            if (alpha < 1.0f / 255.0f) ok = false;
                        }
                    }
                    if (ok) {
                        contrib = true;
                        const float4 r3 = sr[3][jj], r4 = sr[4][jj];
                        const float col[3] = {r3.w, r4.x, r4.y};
                        const float nrm[3] = {r3.x, r3.y, r3.z};
                        T = T / (1.f - alpha);
                        const float wT = alpha * T;
                        float dL_dalpha = 0.0f;
#pragma unroll
                        for (int ch = 0; ch < 3; ++ch) {
                            accum_rec[ch] = last_alpha * last_color[ch] + (1.f - last_alpha) * accum_rec[ch];
                            last_color[ch] = col[ch];
                            dL_dalpha += (col[ch] - accum_rec[ch]) * dpix[ch];
                            v[15 + ch] = wT * dpix[ch];
                        }
                        float dL_dz = 0.0f;
                        const float c_d = h.depth;
                        const float m_d = mscale * (1 - NEAR_N / c_d);
                        const float dmd_dd = (FAR_N * NEAR_N) / ((FAR_N - NEAR_N) * c_d * c_d);
                        if (contributor == (uint32_t)(median_contributor - 1)) dL_dz += dd_median;
                        const float dL_dweight = (final_D2 + m_d * m_d * final_A - 2 * m_d * final_D) * dd_reg;
                        dL_dalpha += dL_dweight - last_dL_dT;
                        last_dL_dT = dL_dweight * alpha + (1 - alpha) * last_dL_dT;
                        const float dL_dmd = 2.0f * (T * alpha) * (m_d * final_A - final_D) * dd_reg;
                        dL_dz += dL_dmd * dmd_dd;
                        accum_depth_rec = last_alpha * last_depth + (1.f - last_alpha) * accum_depth_rec;
                        last_depth = c_d;
                        dL_dalpha += (c_d - accum_depth_rec) * dd_depth;
                        // the reference adds last_alpha * 1.0 in double precision
                        accum_alpha_rec = (float)((double)last_alpha + (double)__fmul_rn(1.f - last_alpha, accum_alpha_rec));
                        dL_dalpha += (1 - accum_alpha_rec) * dd_accum;
#pragma unroll
                        for (int ch = 0; ch < 3; ++ch) {
                            accum_normal_rec[ch] = last_alpha * last_normal[ch] + (1.f - last_alpha) * accum_normal_rec[ch];
                            last_normal[ch] = nrm[ch];
                            dL_dalpha += (nrm[ch] - accum_normal_rec[ch]) * dd_normal[ch];
                            v[11 + ch] = alpha * T * dd_normal[ch];
                        }
                        dL_dalpha *= T;
                        last_alpha = alpha;
                        dL_dalpha += (-T_final / (1.f - alpha)) * bg_dot_dpixel;
                        const float dL_dG = r2.w * dL_dalpha;
                        dL_dz += alpha * T * dd_depth;
                        if (h.rho3d <= h.rho2d) {
                            const float dsx = dL_dG * -G * h.sx + dL_dz * r2.x;
                            const float dsy = dL_dG * -G * h.sy + dL_dz * r2.y;
                            const float dsx_pz = dsx / h.p.z, dsy_pz = dsy / h.p.z;
                            const V3 dL_dp = v3(dsx_pz, dsy_pz, -(dsx_pz * h.sx + dsy_pz * h.sy));
                            const V3 dL_dk = vcross(h.l, dL_dp);
                            const V3 dL_dl = vcross(dL_dp, h.k);
                            v[0] = -dL_dk.x; v[1] = -dL_dk.y; v[2] = -dL_dk.z;
                            v[3] = -dL_dl.x; v[4] = -dL_dl.y; v[5] = -dL_dl.z;
                            v[6] = pxf * dL_dk.x + pyf * dL_dl.x + dL_dz * h.sx;
                            v[7] = pxf * dL_dk.y + pyf * dL_dl.y + dL_dz * h.sy;
                            v[8] = pxf * dL_dk.z + pyf * dL_dl.z + dL_dz * 1.0f;
                        } else {
                            const float dG_ddelx = -G * FILTER_INV_SQUARE * h.dx;
                            const float dG_ddely = -G * FILTER_INV_SQUARE * h.dy;
                            v[9] = dL_dG * dG_ddelx;
                            v[10] = dL_dG * dG_ddely;
                            v[6] = h.sx * dL_dz;
                            v[7] = h.sy * dL_dz;
                            v[8] = dL_dz;
                        }
                        v[14] = G * dL_dalpha;
                    }
                }
            }
            if (__any_sync(0xffffffffu, contrib)) {
                float o[3];
                warp_reduce24(v, o);
                const int base = 3 * (lane >> 2);
                if ((lane & 3) == 0 && base < NGRAD) {
                    s_red[jj][warp][base] = o[0];
                    s_red[jj][warp][base + 1] = o[1];
                    s_red[jj][warp][base + 2] = o[2];
                }
            } else if (lane < NGRAD) {
                s_red[jj][warp][lane] = 0.f;
            }
        }
        __syncthreads();
        for (int jj = threadIdx.x; jj < nb; jj += BLOCK) {
            float s[20];
#pragma unroll
            for (int q = 0; q < NGRAD; ++q) {
                float a = s_red[jj][0][q];
#pragma unroll
                for (int w = 1; w < BLOCK / 32; ++w) a += s_red[jj][w][q];
                s[q] = a;
            }
            s[18] = 0.f;
            s[19] = 0.f;
            float4* out = partial + (int64_t)PARTIAL_F4 * si[jj];
#pragma unroll
            for (int f = 0; f < PARTIAL_F4; ++f) out[f] = make_float4(s[4 * f], s[4 * f + 1], s[4 * f + 2], s[4 * f + 3]);
        }
    }
}

// d|v|/dv applied to dv (reference auxiliary.h:110-121).
__device__ __forceinline__ V3 dnormvdv(const V3 v, const V3 dv) {
    const float sum2 = v.x * v.x + v.y * v.y + v.z * v.z;
    const float invsum32 = 1.0f / sqrtf(sum2 * sum2 * sum2);
    return v3(((+sum2 - v.x * v.x) * dv.x - v.y * v.x * dv.y - v.z * v.x * dv.z) * invsum32,
              (-v.x * v.y * dv.x + (sum2 - v.y * v.y) * dv.y - v.z * v.y * dv.z) * invsum32,
              (-v.x * v.z * dv.x - v.y * v.z * dv.y + (sum2 - v.z * v.z) * dv.z) * invsum32);
}

// One thread per Gaussian: sum its instance partials in order, then the preprocess backward
// (backward.cu:406-602): mean2D -> homography, homography -> mean / scale / rotation, normal
// -> rotation, SH -> colour and mean, and the reference's screen-space mean gradient.
// Per-Gaussian sums of its instances' partials, in instance order, written over its first
// instance's partial: PARTIAL_F4 threads per Gaussian, thread f summing float4 column f, so that
// the threads of a Gaussian read each 80-byte partial together and many Gaussians' loads are in
// flight (the sums are the ones a thread summing all columns would form).
constexpr int REDUCE_THREADS = 32 * PARTIAL_F4;  // 32 Gaussians per block
__global__ void __launch_bounds__(REDUCE_THREADS)
reduce_partials_kernel(int64_t n_gauss, const int* __restrict__ radii, const int* __restrict__ inst_offset,
                       const long long* __restrict__ header, float4* __restrict__ partial) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t g = t / PARTIAL_F4;
    const int f = (int)(t % PARTIAL_F4);
    if (g >= n_gauss || radii[g] <= 0 || header[H_FLAGS] != 0) return;
    const int i0 = inst_offset[g], i1 = inst_offset[g + 1];
    if (i1 <= i0) return;
    float4 s = make_float4(0.f, 0.f, 0.f, 0.f);
    int i = i0;
    for (; i + 4 <= i1; i += 4) {  // four instances' loads in flight
        float4 v[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) v[u] = partial[(int64_t)PARTIAL_F4 * (i + u) + f];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            s.x += v[u].x;
            s.y += v[u].y;
            s.z += v[u].z;
            s.w += v[u].w;
        }
    }
    for (; i < i1; ++i) {
        const float4 v = partial[(int64_t)PARTIAL_F4 * i + f];
        s.x += v.x;
        s.y += v.y;
        s.z += v.z;
        s.w += v.w;
    }
    partial[(int64_t)PARTIAL_F4 * i0 + f] = s;
}

__global__ void __launch_bounds__(128)
reduce_preprocess_kernel(Params p, float focal_x, float focal_y, float tan_fovx, float tan_fovy,
                         const int* __restrict__ radii, const int* __restrict__ inst_offset,
                         const long long* __restrict__ header, const float4* __restrict__ partial,
                         const float4* __restrict__ rec, const int* __restrict__ clamped_bits,
                         float* __restrict__ d_mean2D, float* __restrict__ d_colors, float* __restrict__ d_opacity,
                         float* __restrict__ d_means3D, float* __restrict__ d_transmat, float* __restrict__ d_sh,
                         float* __restrict__ d_scales, float* __restrict__ d_rot) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= p.P) return;
    float s[20];
#pragma unroll
    for (int q = 0; q < 20; ++q) s[q] = 0.f;
    const bool vis = radii[g] > 0 && header[H_FLAGS] == 0;
    if (vis) {  // the instance sums reduce_partials_kernel left in the first instance's partial
        const int i0 = inst_offset[g];
        if (inst_offset[g + 1] > i0) {
            const float4* r = partial + (int64_t)PARTIAL_F4 * i0;
#pragma unroll
            for (int f = 0; f < PARTIAL_F4; ++f) {
                const float4 x = r[f];
                s[4 * f] = x.x;
                s[4 * f + 1] = x.y;
                s[4 * f + 2] = x.z;
                s[4 * f + 3] = x.w;
            }
        }
    }
    // defaults: everything zero, render sums passed through
    float dT[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) dT[q] = s[q];
    float dmean3[3] = {0.f, 0.f, 0.f};
    float dscale[2] = {0.f, 0.f};
    float4 drot = make_float4(0.f, 0.f, 0.f, 0.f);
    float m2x = 0.f, m2y = 0.f;
    const int M = p.M;
    if (p.shs != nullptr)
        for (int k = 0; k < M * 3; ++k) d_sh[(int64_t)g * M * 3 + k] = 0.f;
    float dcol[3] = {s[15], s[16], s[17]};
    if (vis) {
        const int Wb = (int)(focal_x * tan_fovx * 2);
        const int Hb = (int)(focal_y * tan_fovy * 2);
        const bool precomp = (p.scales == nullptr);
        const float3 po = make_float3(p.means[3 * g], p.means[3 * g + 1], p.means[3 * g + 2]);
        Mat<3, 3> T, R, Lm;
        Mat<3, 4> Pm;
        V3 normal;
        float4 rot = make_float4(0.f, 0.f, 0.f, 0.f);
        float scx = 0.f, scy = 0.f;
        if (precomp) {
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int r = 0; r < 3; ++r) T.m[c][r] = p.transmat[9 * g + 3 * c + r];
            normal = v3(0.f, 0.f, 0.f);
        } else {
            rot = make_float4(p.rotations[4 * g], p.rotations[4 * g + 1], p.rotations[4 * g + 2], p.rotations[4 * g + 3]);
            scx = p.scales[2 * g];
            scy = p.scales[2 * g + 1];
            R = quat_rot(rot);
            Lm = mmul(R, scale_mat(scx, scy, 1.0f));
            Pm = mmul(world2ndc(p.proj), ndc2pix(Wb, Hb));
            T = mmul(transpose(splat2world(Lm, po)), Pm);
            normal = xform_vec(col3(Lm, 2), p.view);
        }
        Mat<3, 3> dLT;
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int r = 0; r < 3; ++r) dLT.m[c][r] = dT[3 * c + r];
        const float dmx = s[9], dmy = s[10];
        bool early = false;
        if (dmx != 0 || dmy != 0) {
            const V3 tv = v3(9.0f, 9.0f, -1.0f);
            const V3 T0 = col3(T, 0), T1 = col3(T, 1), T2 = col3(T, 2);
            const float d = vdot(tv, vmul(T2, T2));
            const V3 fv = vscale(1.0f / d, tv);
            const V3 dT0 = vmul(vscale(dmx, fv), T2);
            const V3 dT1 = vmul(vscale(dmy, fv), T2);
            V3 dT3 = vadd(vmul(vscale(dmx, fv), T0), vmul(vscale(dmy, fv), T1));
            const V3 dL_df = vadd(vmul(vscale(dmx, T0), T2), vmul(vscale(dmy, T1), T2));
            const float dL_dd = (float)((double)vdot(dL_df, fv) * (-1.0 / (double)d));
            const V3 dd_dT3 = v3((tv.x * T2.x) * 2.0f, (tv.y * T2.y) * 2.0f, (tv.z * T2.z) * 2.0f);
            dT3 = vadd(dT3, vscale(dL_dd, dd_dT3));
            dLT.m[0][0] += dT0.x; dLT.m[0][1] += dT0.y; dLT.m[0][2] += dT0.z;
            dLT.m[1][0] += dT1.x; dLT.m[1][1] += dT1.y; dLT.m[1][2] += dT1.z;
            dLT.m[2][0] += dT3.x; dLT.m[2][1] += dT3.y; dLT.m[2][2] += dT3.z;
            if (precomp) {
#pragma unroll
                for (int c = 0; c < 3; ++c)
#pragma unroll
                    for (int r = 0; r < 3; ++r) dT[3 * c + r] = dLT.m[c][r];
                early = true;
            }
        }
        if (!precomp && !early) {
            const Mat<3, 4> dM = mmul(Pm, transpose(dLT));
            V3 dtn = xform_vec_t(v3(s[11], s[12], s[13]), p.view);
            const float3 pv = xform_point(po, p.view);
            const float cosv = -(pv.x * normal.x + pv.y * normal.y + pv.z * normal.z);
            const float mult = cosv > 0 ? 1.f : -1.f;
            dtn = vscale(mult, dtn);
            const V3 dRS0 = v3(dM.m[0][0], dM.m[0][1], dM.m[0][2]);
            const V3 dRS1 = v3(dM.m[1][0], dM.m[1][1], dM.m[1][2]);
            Mat<3, 3> dR;
            dR.m[0][0] = dRS0.x * scx; dR.m[0][1] = dRS0.y * scx; dR.m[0][2] = dRS0.z * scx;
            dR.m[1][0] = dRS1.x * scy; dR.m[1][1] = dRS1.y * scy; dR.m[1][2] = dRS1.z * scy;
            dR.m[2][0] = dtn.x; dR.m[2][1] = dtn.y; dR.m[2][2] = dtn.z;
            drot = quat_rot_vjp(rot, dR);
            dscale[0] = vdot(dRS0, col3(R, 0));
            dscale[1] = vdot(dRS1, col3(R, 1));
            dmean3[0] = dM.m[2][0];
            dmean3[1] = dM.m[2][1];
            dmean3[2] = dM.m[2][2];
        }
        // SH backward (backward.cu:20-98), with the reference's degree-2 gradient terms
        if (p.shs != nullptr) {
            const int deg = p.D;
            const V3 pos = v3(po.x, po.y, po.z);
            const V3 dir_orig = vsub(pos, v3(p.campos[0], p.campos[1], p.campos[2]));
            const float len = sqrtf(vdot(dir_orig, dir_orig));
            const V3 dir = v3(dir_orig.x / len, dir_orig.y / len, dir_orig.z / len);
            const float* sh = p.shs + (int64_t)g * M * 3;
            auto c = [&](int k) { return v3(sh[3 * k], sh[3 * k + 1], sh[3 * k + 2]); };
            const int cl = clamped_bits[g];
            V3 dRGB = v3(dcol[0] * ((cl & 1) ? 0.f : 1.f), dcol[1] * ((cl & 2) ? 0.f : 1.f),
                         dcol[2] * ((cl & 4) ? 0.f : 1.f));
            V3 dRGBdx = v3(0, 0, 0), dRGBdy = v3(0, 0, 0), dRGBdz = v3(0, 0, 0);
            const float x = dir.x, y = dir.y, z = dir.z;
            float* dsh = d_sh + (int64_t)g * M * 3;
            auto put = [&](int k, const V3 a) {
                dsh[3 * k] = a.x;
                dsh[3 * k + 1] = a.y;
                dsh[3 * k + 2] = a.z;
            };
            put(0, vscale(SH_C0, dRGB));
            if (deg > 0) {
                put(1, vscale(-SH_C1 * y, dRGB));
                put(2, vscale(SH_C1 * z, dRGB));
                put(3, vscale(-SH_C1 * x, dRGB));
                dRGBdx = vscale(-SH_C1, c(3));
                dRGBdy = vscale(-SH_C1, c(1));
                dRGBdz = vscale(SH_C1, c(2));
                if (deg > 1) {
                    const float depth = x;
                    const float d4 = __expf(-depth);
                    put(4, vscale(d4, dRGB));
                    const float d5 = x * x + y * y + z * z;
                    put(5, vscale(d5, dRGB));
                    const float d6 = x * y, d7 = y * z, d8 = x * z;
                    put(6, vscale(d6, dRGB));
                    put(7, vscale(d7, dRGB));
                    put(8, vscale(d8, dRGB));
                    // vector minus scalar, componentwise, as the reference writes it
                    auto sub = [](V3 a, float b) { return v3(a.x - b, a.y - b, a.z - b); };
                    auto add = [](V3 a, float b) { return v3(a.x + b, a.y + b, a.z + b); };
                    dRGBdx = sub(add(sub(sub(dRGBdx, d4), d5), d6), d8);
                    dRGBdy = add(sub(sub(dRGBdy, d5), d6), d7);
                    dRGBdz = add(sub(sub(dRGBdz, d5), d7), d8);
                }
            }
            const V3 dL_ddir = v3(vdot(dRGBdx, dRGB), vdot(dRGBdy, dRGB), vdot(dRGBdz, dRGB));
            const V3 dm = dnormvdv(dir_orig, dL_ddir);
            dmean3[0] += dm.x;
            dmean3[1] += dm.y;
            dmean3[2] += dm.z;
        }
        // screen-space mean gradient as the reference reports it (backward.cu:558-560)
        const float depth = rec[(int64_t)REC_F4 * g + 2].z;
        m2x = (float)(((double)(dT[2] * depth) * 0.5) * (double)(float)Wb);
        m2y = (float)(((double)(dT[5] * depth) * 0.5) * (double)(float)Hb);
    }
    d_mean2D[3 * g] = m2x;
    d_mean2D[3 * g + 1] = m2y;
    d_mean2D[3 * g + 2] = 0.f;
    d_colors[3 * g] = dcol[0];
    d_colors[3 * g + 1] = dcol[1];
    d_colors[3 * g + 2] = dcol[2];
    d_opacity[g] = s[14];
    d_means3D[3 * g] = dmean3[0];
    d_means3D[3 * g + 1] = dmean3[1];
    d_means3D[3 * g + 2] = dmean3[2];
#pragma unroll
    for (int q = 0; q < 9; ++q) d_transmat[9 * g + q] = dT[q];
    if (d_scales) {
        d_scales[2 * g] = dscale[0];
        d_scales[2 * g + 1] = dscale[1];
    }
    if (d_rot) {
        d_rot[4 * g] = drot.x;
        d_rot[4 * g + 1] = drot.y;
        d_rot[4 * g + 2] = drot.z;
        d_rot[4 * g + 3] = drot.w;
    }
}

// Reference-format binning and per-pixel state (rasterizer_impl.cu:116-137, ImageState).
__global__ void export_kernel(int T, const int* __restrict__ tile_start, const unsigned long long* __restrict__ keys,
                              const int* __restrict__ sorted_gid, uint32_t* __restrict__ point_list,
                              unsigned long long* __restrict__ ref_keys, uint32_t* __restrict__ ranges) {
    const int t = blockIdx.x;
    if (t >= T) return;
    const int s0 = tile_start[t], s1 = tile_start[t + 1];
    if (threadIdx.x == 0) {
        ranges[2 * t] = s1 > s0 ? (uint32_t)s0 : 0u;
        ranges[2 * t + 1] = s1 > s0 ? (uint32_t)s1 : 0u;
    }
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        point_list[s] = (uint32_t)sorted_gid[s];
        if (ref_keys) ref_keys[s] = ((unsigned long long)(uint32_t)t << 32) | (keys[s] >> 32);
    }
}

__global__ void mark_visible_kernel(int P, const float* __restrict__ means, const float* __restrict__ view,
                                    uint8_t* __restrict__ present) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= P) return;
    const float3 po = make_float3(means[3 * g], means[3 * g + 1], means[3 * g + 2]);
    present[g] = (xform_point(po, view).z <= 0.2f) ? 0 : 1;
}

}  // namespace gs
}  // namespace us3d

using namespace us3d;
using namespace us3d::gs;

static bool g_gs_sort_attr[128];

static inline int64_t gs_tiles(int32_t W, int32_t H) {
    return (int64_t)((W + TILE - 1) / TILE) * ((H + TILE - 1) / TILE);
}

extern "C" size_t us3d_gs_workspace_bytes(int64_t n_gauss, int32_t width, int32_t height, int64_t cap) {
    if (n_gauss < 0 || width <= 0 || height <= 0 || cap < 0) return 0;
    return carve(nullptr, n_gauss, gs_tiles(width, height), (int64_t)width * height, cap).bytes;
}

extern "C" size_t us3d_gs_backward_scratch_bytes(int64_t cap) {
    return cap < 0 ? 0 : (size_t)cap * PARTIAL_F4 * sizeof(float4);
}

static Params make_params(int64_t P, int32_t D, int32_t M, int32_t W, int32_t H, const float* means,
                          const float* shs, const float* colors, const float* opac, const float* scales, float mod,
                          const float* rots, const float* transmat, const float* view, const float* proj,
                          const float* campos, int32_t prefiltered) {
    Params p;
    p.P = (int)P; p.D = D; p.M = M; p.W = W; p.H = H;
    p.gx = (W + TILE - 1) / TILE;
    p.gy = (H + TILE - 1) / TILE;
    p.scale_modifier = mod;
    p.prefiltered = prefiltered;
    p.means = means; p.shs = shs; p.colors = colors; p.opacities = opac; p.scales = scales;
    p.rotations = rots; p.transmat = transmat; p.view = view; p.proj = proj; p.campos = campos;
    return p;
}

extern "C" int us3d_gs_forward(void* workspace, size_t workspace_bytes, int64_t n_gauss, int32_t sh_degree,
                               int32_t sh_coeffs, const float* background, int32_t width, int32_t height,
                               const float* means3D, const float* shs, const float* colors_precomp,
                               const float* opacities, const float* scales, float scale_modifier,
                               const float* rotations, const float* transmat_precomp, const float* viewmatrix,
                               const float* projmatrix, const float* campos, int32_t prefiltered, int64_t cap,
                               float* out_color, float* out_others, int32_t* out_radii, void* stream_) {
    US3D_CHECK_ARG(width > 0 && height > 0, "image_width/image_height must be positive");
    US3D_CHECK_ARG(n_gauss >= 0 && n_gauss <= 0x7fffffffLL, "n_gauss out of range");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    US3D_CHECK_ARG(workspace && background && viewmatrix && projmatrix && out_color && out_others,
                   "NULL pointer argument");
    US3D_CHECK_ARG(n_gauss == 0 || (means3D && opacities && out_radii), "NULL Gaussian pointer");
    US3D_CHECK_ARG(n_gauss == 0 || (colors_precomp != nullptr) != (shs != nullptr),
                   "Please provide excatly one of either SHs or precomputed colors!");
    US3D_CHECK_ARG(n_gauss == 0 || ((scales && rotations) != (transmat_precomp != nullptr)),
                   "Please provide exactly one of either scale/rotation pair or precomputed 3D covariance!");
    US3D_CHECK_ARG(shs == nullptr || (sh_coeffs >= 1 && campos != nullptr && sh_degree >= 0 &&
                                      (sh_degree < 1 || sh_coeffs >= 4) && (sh_degree < 2 || sh_coeffs >= 9)),
                   "SH coefficients too few for the requested degree");
    const int64_t T = gs_tiles(width, height), P = (int64_t)width * height;
    const Workspace w = carve(workspace, n_gauss, T, P, cap);
    US3D_CHECK_ARG(workspace_bytes >= w.bytes, "workspace too small: %zu < %zu", workspace_bytes, w.bytes);
    cudaStream_t stream = (cudaStream_t)stream_;
    const Params p = make_params(n_gauss, sh_degree, sh_coeffs, width, height, means3D, shs, colors_precomp,
                                 opacities, scales, scale_modifier, rotations, transmat_precomp, viewmatrix,
                                 projmatrix, campos, prefiltered);
    const int prof = prof_begin("gs_forward", stream);
    init_kernel<<<(unsigned)((T + 255) / 256), 256, 0, stream>>>(T, w.tile_count, w.tile_cursor, w.header, cap,
                                                                 n_gauss, P);
    const unsigned gb = (unsigned)((n_gauss + 255) / 256);
    if (n_gauss > 0)
        preprocess_kernel<<<gb, 256, 0, stream>>>(p, out_radii, w.rec, w.depth, w.rect, w.clamped, w.touched,
                                                  w.tile_count, w.header);
    US3D_CHECK_LAUNCH("gs preprocess");
    US3D_CHECK_CUDA(launch_rect_count(n_gauss, p.gx, T, RectOf4{w.rect}, w.tile_count, stream));
    US3D_CHECK_CUDA(exclusive_scan(w.touched, n_gauss, w.inst_offset, w.bs_g, w.header + H_SCAN_G, stream));
    US3D_CHECK_CUDA(exclusive_scan(w.tile_count, T, w.tile_start, w.bs_t, w.header + H_SCAN_T, stream));
    check_kernel<<<1, 1, 0, stream>>>(w.header, cap);
    US3D_CHECK_CUDA(launch_rect_scatter(n_gauss, p.gx, T, RectOf4{w.rect}, reinterpret_cast<const uint32_t*>(w.depth),
                                        w.inst_offset, w.tile_start, w.tile_cursor, w.header, w.keys, w.slot_inst,
                                        stream));
    US3D_CHECK_CUDA(launch_tile_sort(T, n_gauss, w.tile_start, w.header, w.keys, w.slot_inst, w.sorted_gid, w.sorted_inst,
                                     g_gs_sort_attr, stream));
    forward_kernel<<<(unsigned)T, BLOCK, 0, stream>>>(width, height, p.gx, w.tile_start, w.sorted_gid, w.header, w.rec,
                                                      background, out_color, out_others, w.accum, w.n_contrib);
    US3D_CHECK_LAUNCH("gs forward");
    prof_end(prof, stream);
    count_launches(1 + 3 * (n_gauss > 0) + 6 + 1 + tile_sort_launches(n_gauss) + 1);
    return US3D_OK;
}

extern "C" int us3d_gs_read_status(const void* workspace, int64_t* total, int32_t* flags, void* stream_) {
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    long long hdr[H_WORDS];
    cudaStream_t stream = (cudaStream_t)stream_;
    US3D_CHECK_CUDA(cudaMemcpyAsync(hdr, workspace, sizeof(hdr), cudaMemcpyDeviceToHost, stream));
    US3D_CHECK_CUDA(cudaStreamSynchronize(stream));
    if (total) *total = hdr[H_TOTAL];
    if (flags) *flags = (int32_t)hdr[H_FLAGS];
    return US3D_OK;
}

extern "C" int us3d_gs_backward(void* workspace, int64_t n_gauss, int32_t sh_degree, int32_t sh_coeffs,
                                const float* background, int32_t width, int32_t height, const float* means3D,
                                const float* shs, const float* colors_precomp, const float* scales,
                                float scale_modifier, const float* rotations, const float* transmat_precomp,
                                const float* viewmatrix, const float* projmatrix, const float* campos,
                                float tan_fovx, float tan_fovy, const int32_t* radii, int64_t cap,
                                const float* dL_dcolor, const float* dL_dothers, void* scratch, size_t scratch_bytes,
                                float* d_means2D, float* d_colors, float* d_opacity, float* d_means3D,
                                float* d_transmat, float* d_sh, float* d_scales, float* d_rotations, void* stream_) {
    US3D_CHECK_ARG(width > 0 && height > 0 && n_gauss >= 0 && cap >= 0, "bad sizes");
    US3D_CHECK_ARG(workspace && background && viewmatrix && projmatrix && dL_dcolor && dL_dothers,
                   "NULL pointer argument");
    US3D_CHECK_ARG(scratch_bytes >= us3d_gs_backward_scratch_bytes(cap), "backward scratch too small");
    US3D_CHECK_ARG(n_gauss == 0 || (means3D && radii && d_means2D && d_colors && d_opacity && d_means3D && d_transmat),
                   "NULL gradient pointer");
    US3D_CHECK_ARG(shs == nullptr || (d_sh && campos), "NULL SH gradient pointer");
    (void)colors_precomp;
    (void)scale_modifier;  // the reference's backward rebuilds the homography at scale 1
    const int64_t T = gs_tiles(width, height), P = (int64_t)width * height;
    const Workspace w = carve(workspace, n_gauss, T, P, cap);
    cudaStream_t stream = (cudaStream_t)stream_;
    const Params p = make_params(n_gauss, sh_degree, sh_coeffs, width, height, means3D, shs, colors_precomp, nullptr,
                                 scales, scale_modifier, rotations, transmat_precomp, viewmatrix, projmatrix, campos, 0);
    // focal lengths exactly as the reference computes them on the host
    const float focal_y = (float)height / (2.0f * tan_fovy);
    const float focal_x = (float)width / (2.0f * tan_fovx);
    float4* partial = reinterpret_cast<float4*>(scratch);
    const int prof = prof_begin("gs_backward", stream);
    backward_kernel<<<(unsigned)T, BLOCK, 0, stream>>>(width, height, p.gx, w.tile_start, w.sorted_gid,
                                                       w.sorted_inst, w.header, w.rec, background, w.accum,
                                                       w.n_contrib, dL_dcolor, dL_dothers, partial);
    if (n_gauss > 0) {
        reduce_partials_kernel<<<(unsigned)((n_gauss * PARTIAL_F4 + REDUCE_THREADS - 1) / REDUCE_THREADS),
                                 REDUCE_THREADS, 0, stream>>>(n_gauss, radii, w.inst_offset, w.header, partial);
        reduce_preprocess_kernel<<<(unsigned)((n_gauss + 127) / 128), 128, 0, stream>>>(
            p, focal_x, focal_y, tan_fovx, tan_fovy, radii, w.inst_offset, w.header, partial, w.rec, w.clamped,
            d_means2D, d_colors, d_opacity, d_means3D, d_transmat, d_sh, d_scales, d_rotations);
    }
    US3D_CHECK_LAUNCH("gs backward");
    prof_end(prof, stream);
    count_launches(1 + 2 * (n_gauss > 0));
    return US3D_OK;
}

extern "C" int us3d_gs_export(const void* workspace, int64_t n_gauss, int32_t width, int32_t height, int64_t cap,
                              uint32_t* out_point_list, uint64_t* out_keys, uint32_t* out_ranges,
                              uint32_t* out_n_contrib, float* out_accum, float* out_records, void* stream_) {
    US3D_CHECK_ARG(workspace && out_point_list && out_ranges && width > 0 && height > 0, "bad argument");
    const int64_t T = gs_tiles(width, height), P = (int64_t)width * height;
    const Workspace w = carve(const_cast<void*>(workspace), n_gauss, T, P, cap);
    cudaStream_t stream = (cudaStream_t)stream_;
    export_kernel<<<(unsigned)T, 256, 0, stream>>>((int)T, w.tile_start, w.keys, w.sorted_gid, out_point_list,
                                                   reinterpret_cast<unsigned long long*>(out_keys), out_ranges);
    US3D_CHECK_LAUNCH("gs export");
    if (out_n_contrib)
        US3D_CHECK_CUDA(cudaMemcpyAsync(out_n_contrib, w.n_contrib, sizeof(uint32_t) * 2 * P, cudaMemcpyDeviceToDevice, stream));
    if (out_accum)
        US3D_CHECK_CUDA(cudaMemcpyAsync(out_accum, w.accum, sizeof(float) * 3 * P, cudaMemcpyDeviceToDevice, stream));
    if (out_records && n_gauss > 0)
        US3D_CHECK_CUDA(cudaMemcpyAsync(out_records, w.rec, sizeof(float4) * REC_F4 * n_gauss, cudaMemcpyDeviceToDevice,
                                        stream));
    count_launches(1);
    return US3D_OK;
}

extern "C" int us3d_gs_mark_visible(int64_t n_gauss, const float* means3D, const float* viewmatrix,
                                    uint8_t* out_present, void* stream_) {
    US3D_CHECK_ARG(n_gauss >= 0 && n_gauss <= 0x7fffffffLL, "n_gauss out of range");
    if (n_gauss == 0) return US3D_OK;
    US3D_CHECK_ARG(means3D && viewmatrix && out_present, "NULL pointer argument");
    mark_visible_kernel<<<(unsigned)((n_gauss + 255) / 256), 256, 0, (cudaStream_t)stream_>>>((int)n_gauss, means3D,
                                                                                             viewmatrix, out_present);
    US3D_CHECK_LAUNCH("gs mark_visible");
    count_launches(1);
    return US3D_OK;
}
