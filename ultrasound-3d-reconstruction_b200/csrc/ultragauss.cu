// UltraGauss probe-plane slice splatting: binning, forward shading, backward adjoint.
//
// Reference behaviour restated here (paths inside KevinWCCC/ultrasound-3d-reconstruction):
//   ops/ultragauss_renderer/src/mapper/core.cu:9-164    projection, window radii, cull,
//                                                       tile rectangles, keys, ranges
//   ops/ultragauss_renderer/src/mapper/core.cu:166-287  per-pixel window test (candidates)
//   ops/ultragauss_renderer/src/shader/forward.cu:17-76 per-pixel normalised compositing
//   ops/ultragauss_renderer/src/shader/backward.cu:17-131 adjoint
//   ops/ultragauss_renderer/include/shader/shared.cuh:4-52 precision from the raw factor
//
// B200 design (not the reference's): one launch sequence bins any number of frames at
// once; instances are bucketed straight into their tile (atomic cursor) and each tile's
// bucket is put into the reference's (depth key, Gaussian index) order by an in-shared-
// memory bitonic sort, so no global 64-bit radix sort and no host synchronisation is
// needed. The forward stages each tile's Gaussians in shared memory (one pixel per
// thread, reference summation order); the backward gives each thread one (tile, Gaussian)
// instance, walks the tile's pixels from shared memory and accumulates that instance's
// gradient in registers, so there are no float atomics and no warp reductions. Partials
// are reduced per Gaussian in a fixed order (deterministic gradients).
//
// Arithmetic that decides integer outputs (window radii, culling, tile rectangles, depth
// keys, the window test) is written with the same operations in the same order as the
// reference so that, compiled with the same fast-math flags, keys, ranges and candidate
// counts agree bit for bit.
#include <algorithm>

#include <atomic>
#include <type_traits>

#include "us3d_common.cuh"
#include "scan.cuh"
#include "binning.cuh"

namespace us3d {
namespace ug {

// Resident CTAs per SM the forward is compiled for (register budget 65536 / (256 x n)). Five
// measured fastest on the 1M-Gaussian 512x512 scene: 2.25 ms per 16 frames, against 2.39 ms with
// six (40 registers) and 2.50 ms with seven (32 registers).
#ifndef US3D_UG_FWD_MIN_CTAS
#define US3D_UG_FWD_MIN_CTAS 5
#endif

constexpr int TILE = 16;           // reference SLICE_TILE_SIZE (include/mapper/core.cuh:5)
constexpr int TILE_PIX = TILE * TILE;
// Launch shapes the shading kernels are instantiated for (us3d_ug_set_launch_config picks
// one of each at run time; the defaults are the fastest measured on the headline scene):
// Gaussians staged per forward batch, and threads of a backward CTA (compiled for 1024 /
// threads resident CTAs per SM).
constexpr int FWD_BATCH = 512;
constexpr int BWD_THREADS = 256;
// A tile's pixels are shaded by 8 warps, each owning a block of 8 columns x 4 rows (warp
// w = 2 * band + half). An instance's mask marks 4x4-pixel sub-blocks: bit (band * 4 + quarter)
// is set when the Gaussian can reach sub-block (4-row band, 4-column quarter) of the tile, so
// warp block w is sub-blocks 2w and 2w + 1. The forward visits an instance when either of its
// warp's sub-blocks is marked; the backward sweeps the marked sub-blocks only.
constexpr int BLK_W = 8, BLK_H = 4;
constexpr int SUB = 4;                                    // sub-block edge (pixels)
constexpr int NSUB = (TILE / SUB) * (TILE / SUB);         // 16 sub-blocks per tile
constexpr int SUB_PIX = SUB * SUB;                        // 16 pixels per sub-block
typedef uint16_t blockmask_t;
constexpr unsigned FULL_MASK = 0xffffu;
constexpr int BWD_CHUNK = 1024;      // instances regrouped per backward pass

// Header words at the start of the workspace.

struct Workspace {
    long long* header;
    float4* pack;            // G x 3 float4: (m.xyz, o) (t0..t3) (t4, t5, c, 0)
    int* gtasks;             // G: frames in which the Gaussian survives the cull (tasks)
    int* task_offset;        // G + 1: exclusive scan of gtasks
    long long* bs_g;         // scan block sums over G
    int* inst_offset;        // G + 1: first instance of each Gaussian
    int4* task_rect;         // TC: (g, f) task's tile rectangle
    int2* task_gf;           // TC: Gaussian, frame
    float* task_v;           // TC: axial pixel coordinate (depth key source)
    int* task_ntiles;        // TC: instances of the task
    int* task_inst;          // TC + 1: exclusive scan of task_ntiles
    long long* bs_k;         // scan block sums over TC
    int* tile_count;         // T
    int* tile_start;         // T + 1
    int* tile_cursor;        // T
    long long* bs_t;         // scan block sums over T
    int* tile_frame;
    float* tile_dev;     // per tile: largest distance of a pixel from its frame's grid (slice cull)
    unsigned* frame_dev; // at a frame's first tile: the largest deviation of its tiles (float bits)         // T
    unsigned long long* keys;  // cap: (depth_key << 32) | g, sorted in place per tile
    int* slot_inst;          // cap: instance index of each bucket slot (unsorted)
    int* sorted_gid;         // cap
    int* sorted_inst;        // cap
    blockmask_t* slot_mask;    // cap: sub-block mask of each bucket slot (unsorted)
    blockmask_t* sorted_mask;  // cap
    float2* pixel_aux;       // P: no-skip sums (sum a*c, sum a*depth) for the backward
    size_t bytes;
};

// (Gaussian, frame) tasks: every task yields at least one instance in a full binning, and
// a culled binning keeps about a tenth as many tasks as instances; an overflow is flagged
// with a total that makes the retried capacity large enough.
static inline int64_t task_capacity(int64_t cap) { return cap / 4 + 4096; }

// Layout of a workspace. The task arrays, used only while binning, come last, so the
// shading and export entry points find every other array at the same place whatever the
// task capacity (tc < 0: the default task_capacity(cap)).
static Workspace carve(void* base, int64_t G, int64_t T, int64_t P, int64_t cap, int64_t tc = -1) {
    Carver c(base);
    Workspace w;
    w.header = c.take<long long>(H_WORDS);
    w.pack = c.take<float4>((size_t)G * 3);
    w.gtasks = c.take<int>((size_t)G);
    w.task_offset = c.take<int>((size_t)G + 1);
    w.bs_g = c.take<long long>((size_t)scan_num_blocks(G) + 1);
    w.inst_offset = c.take<int>((size_t)G + 1);
    w.tile_count = c.take<int>((size_t)T);
    w.tile_start = c.take<int>((size_t)T + 1);
    w.tile_cursor = c.take<int>((size_t)T);
    w.bs_t = c.take<long long>((size_t)scan_num_blocks(T) + 1);
    w.tile_frame = c.take<int>((size_t)T);
    w.tile_dev = c.take<float>((size_t)T);
    w.frame_dev = c.take<unsigned>((size_t)T);
    w.keys = c.take<unsigned long long>((size_t)cap);
    w.slot_inst = c.take<int>((size_t)cap);
    w.sorted_gid = c.take<int>((size_t)cap);
    w.sorted_inst = c.take<int>((size_t)cap);
    w.slot_mask = c.take<blockmask_t>((size_t)cap);
    w.sorted_mask = c.take<blockmask_t>((size_t)cap);
    w.pixel_aux = c.take<float2>((size_t)P);
    if (tc < 0) tc = task_capacity(cap);
    w.task_rect = c.take<int4>((size_t)tc);
    w.task_gf = c.take<int2>((size_t)tc);
    w.task_v = c.take<float>((size_t)tc);
    w.task_ntiles = c.take<int>((size_t)tc);
    w.task_inst = c.take<int>((size_t)tc + 1);
    w.bs_k = c.take<long long>((size_t)scan_num_blocks(tc) + 1);
    w.bytes = align_up(c.off, 256);
    return w;
}

struct Geo {
    float3 o, lat, ax, ele;
    float dlat, dax, near, coloff;
    int H, W, tx, ty, pix_off, tile_off;
};

__device__ __forceinline__ Geo load_geo(const us3d_slice_frame* __restrict__ fr) {
    Geo g;
    g.o = make_float3(fr->origin[0], fr->origin[1], fr->origin[2]);
    g.lat = make_float3(fr->axis_lat[0], fr->axis_lat[1], fr->axis_lat[2]);
    g.ax = make_float3(fr->axis_ax[0], fr->axis_ax[1], fr->axis_ax[2]);
    g.ele = make_float3(fr->axis_ele[0], fr->axis_ele[1], fr->axis_ele[2]);
    g.dlat = fr->lateral_spacing;
    g.dax = fr->axial_spacing;
    g.near = fr->axial_near;
    g.coloff = fr->lateral_col_offset;
    g.H = fr->height;
    g.W = fr->width;
    g.tx = fr->tiles_x;
    g.ty = fr->tiles_y;
    g.pix_off = fr->pixel_offset;
    g.tile_off = fr->tile_offset;
    return g;
}

// Lateral / axial / elevational half-widths of the chi-square ellipsoid: for the
// precision Lambda = L L^T, the standard deviation along unit axis a is ||L^-1 a||,
// obtained by forward substitution (reference: src/mapper/core.cu:9-44).
__device__ __forceinline__ void window_radii(float t0, float t1, float t2, float t3, float t4,
                                             float t5, float chi2, float beta, float3 a_lat,
                                             float3 a_ax, float3 a_ele, float& r_lat,
                                             float& r_ax, float& r_ele) {
    const float d1 = t0 * t0 + beta;
    const float d2 = t3 * t3 + beta;
    const float d3 = t5 * t5 + beta;
    const float inv1 = fmaxf(d1, 1e-10f), inv2 = fmaxf(d2, 1e-10f), inv3 = fmaxf(d3, 1e-10f);
    const float la0 = a_lat.x / inv1;
    const float la1 = (a_lat.y - t1 * la0) / inv2;
    const float la2 = (a_lat.z - t2 * la0 - t4 * la1) / inv3;
    const float v_lat = fmaxf(la0 * la0 + la1 * la1 + la2 * la2, 1e-12f);
    const float xa0 = a_ax.x / inv1;
    const float xa1 = (a_ax.y - t1 * xa0) / inv2;
    const float xa2 = (a_ax.z - t2 * xa0 - t4 * xa1) / inv3;
    const float v_ax = fmaxf(xa0 * xa0 + xa1 * xa1 + xa2 * xa2, 1e-12f);
    const float ea0 = a_ele.x / inv1;
    const float ea1 = (a_ele.y - t1 * ea0) / inv2;
    const float ea2 = (a_ele.z - t2 * ea0 - t4 * ea1) / inv3;
    const float v_ele = fmaxf(ea0 * ea0 + ea1 * ea1 + ea2 * ea2, 1e-12f);
    const float k = sqrtf(chi2);
    r_lat = fmaxf(1e-3f, k * sqrtf(v_lat));
    r_ax = fmaxf(1e-3f, k * sqrtf(v_ax));
    r_ele = fmaxf(1e-3f, k * sqrtf(v_ele));
}

// Probe-frame projection, elevational cull and 16x16 tile rectangle of one Gaussian in
// one frame (reference: src/mapper/core.cu:46-116). Returns false when culled.
__device__ __forceinline__ bool project_rect(const float4 a, const float4 b, const float4 c,
                                             const Geo& F, float chi2, float beta, int4& rect,
                                             float& v_pix) {
    const float3 m = make_float3(a.x, a.y, a.z);
    const float3 v = f3_sub(m, F.o);
    const float lat = f3_dot(v, F.lat);
    const float ele = f3_dot(v, F.ele);
    const float ax = f3_dot(v, F.ax);
    float r_lat, r_ax, r_ele;
    window_radii(b.x, b.y, b.z, b.w, c.x, c.y, chi2, beta, F.lat, F.ax, F.ele, r_lat, r_ax, r_ele);
    if (fabsf(ele) > r_ele) return false;
    const float u_pix = lat / F.dlat + F.coloff;
    v_pix = (ax - F.near) / F.dax;
    const float r_u = fmaxf(1.0f, r_lat / F.dlat);
    const float r_v = fmaxf(1.0f, r_ax / F.dax);
    int x0 = (int)floorf((u_pix - r_u) / TILE);
    int y0 = (int)floorf((v_pix - r_v) / TILE);
    int x1 = (int)ceilf((u_pix + r_u) / TILE);
    int y1 = (int)ceilf((v_pix + r_v) / TILE);
    x0 = max(0, x0);
    y0 = max(0, y0);
    x1 = min(min((F.W + TILE - 1) / TILE, F.tx), x1);
    y1 = min(min((F.H + TILE - 1) / TILE, F.ty), y1);
    if (x0 >= x1 || y0 >= y1) return false;
    rect = make_int4(x0, y0, x1, y1);
    return true;
}

// Depth key of the reference (src/mapper/core.cu:134): truncation of (v + 500) * 1000 to
// uint32 with the saturating float->u32 conversion of the GPU.
__device__ __forceinline__ uint32_t depth_key(float v_pix, int sort_by_depth) {
    return sort_by_depth ? f32_to_u32_sat((v_pix + 500.0f) * 1000.0f) : 0u;
}

// ------------------------------------------------------------------------------------
// Binning kernels
// ------------------------------------------------------------------------------------

__device__ __forceinline__ bool frame_ok(const us3d_slice_frame* __restrict__ frp, int64_t T, int64_t P) {
    const us3d_slice_frame& fr = *frp;
    return fr.height >= 0 && fr.width >= 0 && fr.tiles_x == (fr.width + TILE - 1) / TILE &&
           fr.tiles_y == (fr.height + TILE - 1) / TILE && fr.tile_offset >= 0 && fr.pixel_offset >= 0 &&
           (int64_t)fr.tile_offset + (int64_t)fr.tiles_x * fr.tiles_y <= T &&
           (int64_t)fr.pixel_offset + (int64_t)fr.width * fr.height <= P;
}

// Clears the per-tile counters, marks every tile as belonging to no frame and records the
// sizes the workspace was carved with.
__global__ void init_tiles_kernel(int64_t T, int* __restrict__ tile_count, int* __restrict__ tile_cursor,
                                  int* __restrict__ tile_frame, unsigned* __restrict__ frame_dev,
                                  long long* __restrict__ header, int64_t cap, int64_t G, int64_t P, int mode) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < H_WORDS) {
        long long v = 0;
        if (threadIdx.x == H_MODE) v = mode;
        if (threadIdx.x == H_CAP) v = cap;
        if (threadIdx.x == H_G) v = G;
        if (threadIdx.x == H_T) v = T;
        if (threadIdx.x == H_P) v = P;
        header[threadIdx.x] = v;
    }
    if (t >= T) return;
    tile_count[t] = 0;
    tile_cursor[t] = 0;
    tile_frame[t] = -1;
    frame_dev[t] = 0u;
}

// Assigns each frame's tiles to it and validates the frame table against the sizes.
__global__ void setup_kernel(const us3d_slice_frame* __restrict__ frames, int F, int64_t T, int64_t P,
                             int* __restrict__ tile_frame, long long* __restrict__ header) {
    const int f = blockIdx.x;
    if (f >= F) return;
    const us3d_slice_frame fr = frames[f];
    if (!frame_ok(frames + f, T, P)) {
        if (threadIdx.x == 0) atomicOr(reinterpret_cast<unsigned long long*>(header + H_FLAGS), (unsigned long long)FLAG_TABLE);
        return;
    }
    const int n = fr.tiles_x * fr.tiles_y;
    for (int i = threadIdx.x; i < n; i += blockDim.x) tile_frame[fr.tile_offset + i] = f;
}

// logits != 0: opacities and intensities are raw logits, activated here by the logistic
// function (the training parameterisation).
__global__ void pack_kernel(int64_t G, const float* __restrict__ means, const float* __restrict__ tril,
                            const float* __restrict__ opac, const float* __restrict__ inten, int logits,
                            float4* __restrict__ pack) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const float* m = means + 3 * g;
    const float2* t = reinterpret_cast<const float2*>(tril + 6 * g);  // 8-byte aligned rows
    const float2 t01 = t[0], t23 = t[1], t45 = t[2];
    const float o = logits ? sigmoid_logit(opac[g]) : opac[g];
    const float c = logits ? sigmoid_logit(inten[g]) : inten[g];
    pack[3 * g + 0] = make_float4(m[0], m[1], m[2], o);
    pack[3 * g + 1] = make_float4(t01.x, t01.y, t23.x, t23.y);
    pack[3 * g + 2] = make_float4(t45.x, t45.y, c, 0.0f);
}

__device__ __forceinline__ void precision_from_raw(float t0, float t1, float t2, float t3, float t4,
                                                   float t5, float beta, float4& q1, float& s12, float& s22);

// ------------------------------------------------------------------------------------
// Slice cull (optional): a tile keeps a Gaussian only if the Gaussian's chi-square quadratic
// restricted to the frame's pixel grid can be <= chi2 somewhere in the tile. On the grid
// P(x, y) = o + (x - col_offset) dlat lat + (near + y dax) ax the quadratic is a 2D convex
// quadratic in pixel coordinates; its minimum over the tile's pixel-centre rectangle is
// found exactly (in double precision) and compared with chi2 plus a margin that bounds the
// distance of the real pixels from the grid (`tile_dev`) and the float rounding of the
// per-pixel test. A pixel that passes the chi-square test therefore always finds the
// Gaussian in its tile list, in the same relative order: images are unchanged and the
// dropped instances would have contributed nothing. Only the window-test counts (and the
// candidate lists built from them) change, so they are not produced after such a binning.
// ------------------------------------------------------------------------------------

struct SliceQuad {
    double w0[3], A[3], B[3];  // d(x, y) = P(x, y) - m = w0 + x A + y B
    double L[6];               // precision l00 l01 l02 l11 l12 l22
    double h00, h01, h11, xc, yc, lam;
    int ok;
};

__device__ __forceinline__ double lam_form_d(const double* L, double dx, double dy, double dz) {
    return dx * (L[0] * dx + L[1] * dy + L[2] * dz) + dy * (L[1] * dx + L[3] * dy + L[4] * dz) +
           dz * (L[2] * dx + L[4] * dy + L[5] * dz);
}

__device__ __forceinline__ double slice_q(const SliceQuad& S, double x, double y) {
    return lam_form_d(S.L, S.w0[0] + x * S.A[0] + y * S.B[0], S.w0[1] + x * S.A[1] + y * S.B[1],
                      S.w0[2] + x * S.A[2] + y * S.B[2]);
}

__device__ __forceinline__ void slice_setup(const float4 a, const float4 b, const float4 c, const Geo& F, float beta,
                                            SliceQuad& S) {
    float4 q1;
    float s12, s22;
    precision_from_raw(b.x, b.y, b.z, b.w, c.x, c.y, beta, q1, s12, s22);
    S.L[0] = q1.x; S.L[1] = q1.y; S.L[2] = q1.z; S.L[3] = q1.w; S.L[4] = s12; S.L[5] = s22;
    const double lat[3] = {F.lat.x, F.lat.y, F.lat.z}, ax[3] = {F.ax.x, F.ax.y, F.ax.z};
    const double o[3] = {F.o.x, F.o.y, F.o.z}, m[3] = {a.x, a.y, a.z};
    double LA[3], LB[3], LW[3];
    for (int i = 0; i < 3; ++i) {
        S.A[i] = (double)F.dlat * lat[i];
        S.B[i] = (double)F.dax * ax[i];
        S.w0[i] = (o[i] - m[i]) - (double)F.coloff * S.A[i] + (double)F.near * ax[i];
    }
    for (int i = 0; i < 3; ++i) {
        const int r0 = i == 0 ? 0 : (i == 1 ? 1 : 2), r1 = i == 0 ? 1 : (i == 1 ? 3 : 4), r2 = i == 0 ? 2 : (i == 1 ? 4 : 5);
        LA[i] = S.L[r0] * S.A[0] + S.L[r1] * S.A[1] + S.L[r2] * S.A[2];
        LB[i] = S.L[r0] * S.B[0] + S.L[r1] * S.B[1] + S.L[r2] * S.B[2];
        LW[i] = S.L[r0] * S.w0[0] + S.L[r1] * S.w0[1] + S.L[r2] * S.w0[2];
    }
    S.h00 = S.A[0] * LA[0] + S.A[1] * LA[1] + S.A[2] * LA[2];
    S.h01 = S.A[0] * LB[0] + S.A[1] * LB[1] + S.A[2] * LB[2];
    S.h11 = S.B[0] * LB[0] + S.B[1] * LB[1] + S.B[2] * LB[2];
    const double g0 = S.A[0] * LW[0] + S.A[1] * LW[1] + S.A[2] * LW[2];
    const double g1 = S.B[0] * LW[0] + S.B[1] * LW[1] + S.B[2] * LW[2];
    const double det = S.h00 * S.h11 - S.h01 * S.h01;
    S.lam = S.L[0] + S.L[3] + S.L[5];
    S.ok = S.h00 > 0.0 && S.h11 > 0.0 && det > 1e-12 * S.h00 * S.h11 && S.lam < 1e30;
    S.xc = S.ok ? (-g0 * S.h11 + g1 * S.h01) / det : 0.0;
    S.yc = S.ok ? (-g1 * S.h00 + g0 * S.h01) / det : 0.0;
}

// The region {q <= chi2 + tau} of one Gaussian on one frame's pixel grid: an ellipse
// (x - xc, y - yc) H (x - xc, y - yc)^T <= rho. tau bounds the pixels' distance from the grid
// (the frame's largest tile deviation `dev`) and the float rounding of the per-pixel test
// over the reference rectangle `r` (tiles). Returns false when no pixel can pass.
struct SliceEllipse {
    double xc, yc, h00, h01, h11, det, rho;
    // row-range constants: half-height, x-shear h01/h00, det/h00, 1/h00, y offset of the
    // rightmost point
    double ymax, s1, kk, inv_h00, dys;
    int ok;  // 0: degenerate quadratic, keep every tile of the rectangle
};

__device__ __forceinline__ bool slice_ellipse(const SliceQuad& S, const int4 r, const Geo& F, float chi2, float dev,
                                              SliceEllipse& E) {
    E.ok = S.ok;
    if (!S.ok) return true;
    E.xc = S.xc; E.yc = S.yc; E.h00 = S.h00; E.h01 = S.h01; E.h11 = S.h11;
    E.det = S.h00 * S.h11 - S.h01 * S.h01;
    const double qc = slice_q(S, S.xc, S.yc);
    const double x0 = r.x * TILE, x1 = min(r.z * TILE - 1, F.W - 1), y0 = r.y * TILE, y1 = min(r.w * TILE - 1, F.H - 1);
    double dmax2 = 0.0;
    for (int k = 0; k < 4; ++k) {
        const double xx = (k & 1) ? x1 : x0, yy = (k & 2) ? y1 : y0;
        const double dx = S.w0[0] + xx * S.A[0] + yy * S.B[0], dy = S.w0[1] + xx * S.A[1] + yy * S.B[1],
                     dz = S.w0[2] + xx * S.A[2] + yy * S.B[2];
        dmax2 = fmax(dmax2, dx * dx + dy * dy + dz * dz);
    }
    const double dv = (double)dev;
    const double dm = sqrt(dmax2) + dv;
    const double tau = 2.0 * sqrt(((double)chi2 + 1.0) * S.lam) * dv + S.lam * dv * dv + 1.2e-5 * S.lam * dm * dm + 1e-6;
    E.rho = (double)chi2 + tau - qc;
    if (E.rho < 0.0) return false;
    E.inv_h00 = 1.0 / E.h00;
    E.s1 = E.h01 * E.inv_h00;
    E.kk = E.det * E.inv_h00;
    E.ymax = sqrt(E.rho * E.h00 / E.det);
    E.dys = -E.h01 * sqrt(E.rho / (E.h11 * E.det));
    return true;
}

// Pixel-centre x-range [xl, xr] of the ellipse inside the tile row y in [y0, y1] (exact:
// the ellipse's x-extent over a horizontal band); false if the band misses the ellipse.
__device__ __forceinline__ bool ellipse_row_range(const SliceEllipse& E, double y0, double y1, double& xl,
                                                  double& xr) {
    const double a = fmax(y0 - E.yc, -E.ymax), b = fmin(y1 - E.yc, E.ymax);
    if (a > b) return false;
    const double dr = fmin(fmax(E.dys, a), b), dl = fmin(fmax(-E.dys, a), b);
    // The half-widths are rounded to float before their square root: a relative error of a
    // few 1e-7 of the half-width, well inside the slack below (at least 2e-6 of it, since
    // |xl| + |xr| >= xr - xl).
    const float hr = sqrtf((float)fmax(0.0, (E.rho - E.kk * dr * dr) * E.inv_h00));
    const float hl = sqrtf((float)fmax(0.0, (E.rho - E.kk * dl * dl) * E.inv_h00));
    xr = E.xc - E.s1 * dr + (double)hr;
    xl = E.xc - E.s1 * dl - (double)hl;
    const double slack = 1e-6 * (fabs(xl) + fabs(xr) + 1.0);
    xl -= slack;
    xr += slack;
    return true;
}

// Largest distance of a tile's pixels from its frame's grid (double precision grid).
__global__ void __launch_bounds__(TILE_PIX)
tile_dev_kernel(int64_t T, int64_t P, const us3d_slice_frame* __restrict__ frames, const int* __restrict__ tile_frame,
                const float* __restrict__ pixels, float* __restrict__ tile_dev, unsigned* __restrict__ frame_dev) {
    __shared__ unsigned s_max;
    const int64_t t = blockIdx.x;
    if (t >= T) return;
    if (tile_frame[t] < 0) {
        if (threadIdx.x == 0) tile_dev[t] = 0.f;
        return;
    }
    const Geo F = load_geo(frames + tile_frame[t]);
    const int lt = (int)(t - F.tile_off);
    const int tx = lt % F.tx, ty = lt / F.tx;
    const int x = tx * TILE + (threadIdx.x & (TILE - 1)), y = ty * TILE + threadIdx.x / TILE;
    if (threadIdx.x == 0) s_max = 0u;
    __syncthreads();
    if (x < F.W && y < F.H) {
        const int64_t p = (int64_t)F.pix_off + (int64_t)y * F.W + x;
        float e = 1e30f;
        if (p < P) {
            const double s = ((double)x - (double)F.coloff) * (double)F.dlat, u = (double)F.near + (double)y * (double)F.dax;
            const double gx = (double)F.o.x + s * F.lat.x + u * F.ax.x, gy = (double)F.o.y + s * F.lat.y + u * F.ax.y,
                         gz = (double)F.o.z + s * F.lat.z + u * F.ax.z;
            const double ex = pixels[3 * p] - gx, ey = pixels[3 * p + 1] - gy, ez = pixels[3 * p + 2] - gz;
            const double d = sqrt(ex * ex + ey * ey + ez * ez);
            e = (d <= 1e30) ? (float)(d * 1.0001 + 1e-9) : 1e30f;
        }
        atomicMax(&s_max, __float_as_uint(e));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        tile_dev[t] = __uint_as_float(s_max);
        atomicMax(frame_dev + F.tile_off, s_max);
    }
}

// Binning in three steps that keep every thread busy: (1) per Gaussian, the reference's
// elevational cull and tile rectangle in each frame -> surviving (Gaussian, frame) tasks,
// written in (g, f) order; (2) per task, the tiles of its rectangle (optionally only those
// its in-slice ellipse reaches) are counted; (3) per task, the same tiles receive the
// instance's key. Instance ids are the exclusive scan of the tasks' tile counts in (g, f)
// order, hence Gaussian-major and deterministic.

// Frames [f0, f1) that render Gaussian g. With Gaussian sets (frames grouped by set, sets in
// increasing gauss_offset order) two binary searches over the frame table find g's set's
// frames; otherwise every frame renders every Gaussian.
__device__ __forceinline__ void gaussian_frames(const us3d_slice_frame* __restrict__ frames, int F, int64_t g,
                                                int sets, int& f0, int& f1) {
    f0 = 0;
    f1 = F;
    if (!sets) return;
    int lo = 0, hi = F;  // first frame whose set starts after g
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if ((int64_t)frames[mid].gauss_offset <= g) lo = mid + 1; else hi = mid;
    }
    const int last = lo - 1;
    if (last < 0 || g >= (int64_t)frames[last].gauss_offset + frames[last].gauss_count) {
        f1 = 0;  // in no set
        return;
    }
    const int off = frames[last].gauss_offset;
    lo = 0;
    hi = last;  // first frame of that set
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (frames[mid].gauss_offset < off) lo = mid + 1; else hi = mid;
    }
    f0 = lo;
    f1 = last + 1;
}

__global__ void __launch_bounds__(256)
cull_kernel(int64_t G, int64_t T, int64_t P, const us3d_slice_frame* __restrict__ frames, int F, int sets,
            const float4* __restrict__ pack, float chi2, float beta, const int* __restrict__ task_offset,
            int64_t cap, int* __restrict__ gtasks, int4* __restrict__ task_rect, int2* __restrict__ task_gf,
            float* __restrict__ task_v) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= G) return;
    const float4 a = pack[3 * g], b = pack[3 * g + 1], c = pack[3 * g + 2];
    int k = task_offset ? task_offset[g] : 0;
    int n = 0;
    int fa, fb;
    gaussian_frames(frames, F, g, sets, fa, fb);
    for (int f = fa; f < fb; ++f) {
        if (!frame_ok(frames + f, T, P)) continue;
        const Geo geo = load_geo(frames + f);
        int4 r;
        float v_pix;
        if (!project_rect(a, b, c, geo, chi2, beta, r, v_pix)) continue;
        ++n;
        if (task_offset && k < cap) {
            task_rect[k] = r;
            task_gf[k] = make_int2((int)g, f);
            task_v[k] = v_pix;
        }
        ++k;
    }
    if (!task_offset) gtasks[g] = n;
}

__global__ void task_check_kernel(long long* __restrict__ header, int64_t tc) {
    const long long nt = header[H_NTASK];
    if (nt > tc || nt > 0x7fffffffLL) {
        header[H_FLAGS] |= FLAG_OVERFLOW;
        header[H_TOTAL] = 4 * nt;  // a retry with this capacity holds the tasks
    }
}

// Tiles of task k in the order both passes enumerate them, one tile row at a time:
// row(row_base, xa, xb, blocks) for the row's tiles x in [xa, xb) (tile index row_base + x),
// blocks(x) giving the warp blocks of tile x that the in-slice ellipse reaches (each 4-row
// band's exact pixel-centre x-range tested against the block's columns: the same conservative
// bound as the tile cull, so a pixel that passes the chi-square test always lies in a marked
// block); 0xff without WANT_BLOCKS or a cull. Returns the number of tiles.
template <bool WANT_BLOCKS, typename Row>
__device__ __forceinline__ int task_tiles(const int4 r, const Geo& geo, const float4 a, const float4 b,
                                          const float4 c, float chi2, float beta, const unsigned* frame_dev, Row row) {
    SliceEllipse E;
    E.ok = 0;
    if (frame_dev) {
        SliceQuad S;
        slice_setup(a, b, c, geo, beta, S);
        if (!slice_ellipse(S, r, geo, chi2, __uint_as_float(frame_dev[geo.tile_off]), E)) return 0;
    }
    int n = 0;
    for (int y = r.y; y < r.w; ++y) {
        int xa = r.x, xb = r.z;
        double bl[TILE / SUB], br[TILE / SUB];
        if (E.ok) {
            double xl, xr;
            if (!ellipse_row_range(E, y * TILE, min(y * TILE + TILE - 1, geo.H - 1), xl, xr)) continue;
            if (!(xl <= xr)) continue;  // NaN guard
            xa = max(xa, (int)floor(fmax(xl, -1e9) / TILE));
            xb = min(xb, (int)floor(fmin(xr, 1e9) / TILE) + 1);
            if (WANT_BLOCKS && xa < xb) {
#pragma unroll
                for (int sb = 0; sb < TILE / SUB; ++sb) {
                    const int ya = y * TILE + sb * SUB;
                    double u = 1e300, v = -1e300;  // empty band
                    if (ya <= geo.H - 1 && ellipse_row_range(E, ya, min(ya + SUB - 1, geo.H - 1), u, v) &&
                        !(u <= v)) {
                        u = -1e300;  // NaN: keep the whole band
                        v = 1e300;
                    }
                    bl[sb] = u;
                    br[sb] = v;
                }
            }
        }
        if (xa >= xb) continue;
        const bool ell = E.ok != 0;
        row(geo.tile_off + y * geo.tx, xa, xb, n, [&](int x) -> unsigned {
            unsigned blocks = FULL_MASK;
            if (WANT_BLOCKS && ell) {
                blocks = 0u;
#pragma unroll
                for (int sb = 0; sb < TILE / SUB; ++sb)
#pragma unroll
                    for (int qx = 0; qx < TILE / SUB; ++qx) {
                        const double c0 = (double)(x * TILE + qx * SUB), c1 = c0 + (SUB - 1);
                        if (bl[sb] <= c1 && br[sb] >= c0) blocks |= 1u << (sb * (TILE / SUB) + qx);
                    }
            }
            return blocks;
        });
        n += xb - xa;
    }
    return n;
}

__global__ void __launch_bounds__(128)
task_count_kernel(const long long* __restrict__ header, const us3d_slice_frame* __restrict__ frames,
                  const float4* __restrict__ pack, float chi2, float beta, const unsigned* __restrict__ frame_dev,
                  const int4* __restrict__ task_rect, const int2* __restrict__ task_gf, int* __restrict__ task_ntiles,
                  int* __restrict__ tile_count) {
    if (header[H_FLAGS] != 0) return;
    const long long nt = header[H_NTASK];
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += (long long)gridDim.x * blockDim.x) {
        const int2 gf = task_gf[k];
        const float4 a = pack[3 * (int64_t)gf.x], b = pack[3 * (int64_t)gf.x + 1], c = pack[3 * (int64_t)gf.x + 2];
        const Geo geo = load_geo(frames + gf.y);
        task_ntiles[k] = task_tiles<false>(task_rect[k], geo, a, b, c, chi2, beta, frame_dev,
                                           [&](int base, int xa, int xb, int, auto) {
                                               for (int x = xa; x < xb; ++x) atomicAdd(&tile_count[base + x], 1);
                                           });
    }
}

__global__ void inst_offset_kernel(int64_t G, const int* __restrict__ task_offset, const int* __restrict__ task_inst,
                                   const long long* __restrict__ header, int* __restrict__ inst_offset) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g > G) return;
    inst_offset[g] = header[H_FLAGS] != 0 ? 0 : task_inst[task_offset[g]];
}

__global__ void __launch_bounds__(128)
task_scatter_kernel(const long long* __restrict__ header, const us3d_slice_frame* __restrict__ frames,
                    const float4* __restrict__ pack, float chi2, float beta, int sort_by_depth,
                    const unsigned* __restrict__ frame_dev, const int4* __restrict__ task_rect,
                    const int2* __restrict__ task_gf, const float* __restrict__ task_v,
                    const int* __restrict__ task_inst, const int* __restrict__ tile_start, int* __restrict__ tile_cursor,
                    unsigned long long* __restrict__ keys, int* __restrict__ slot_inst,
                    blockmask_t* __restrict__ slot_mask) {
    if (header[H_FLAGS] != 0) return;
    const long long nt = header[H_NTASK];
    for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < nt; k += (long long)gridDim.x * blockDim.x) {
        const int2 gf = task_gf[k];
        const float4 a = pack[3 * (int64_t)gf.x], b = pack[3 * (int64_t)gf.x + 1], c = pack[3 * (int64_t)gf.x + 2];
        const Geo geo = load_geo(frames + gf.y);
        const unsigned long long key =
            ((unsigned long long)depth_key(task_v[k], sort_by_depth) << 32) | (unsigned long long)(uint32_t)gf.x;
        const int i0 = task_inst[k];
        // Slots are reserved four tiles at a time, so that the atomics' round trips overlap.
        task_tiles<true>(task_rect[k], geo, a, b, c, chi2, beta, frame_dev,
                         [&](int base, int xa, int xb, int i, auto blocks_of) {
                             for (int x0 = xa; x0 < xb; x0 += 4) {
                                 int within[4];
#pragma unroll
                                 for (int u = 0; u < 4; ++u)
                                     if (x0 + u < xb) within[u] = atomicAdd(&tile_cursor[base + x0 + u], 1);
#pragma unroll
                                 for (int u = 0; u < 4; ++u) {
                                     if (x0 + u >= xb) break;
                                     const int t = base + x0 + u;
                                     const int slot = tile_start[t] + within[u];
                                     // never outside the bucket (verify_kernel flags it)
                                     if (slot >= tile_start[t + 1]) continue;
                                     keys[slot] = key;
                                     slot_inst[slot] = i0 + i + (x0 - xa) + u;
                                     slot_mask[slot] = (blockmask_t)blocks_of(x0 + u);
                                 }
                             }
                         });
    }
}

// Every bucket must have been filled exactly as counted; otherwise later kernels see a flag.
__global__ void verify_kernel(int64_t T, const int* __restrict__ tile_count, const int* __restrict__ tile_cursor,
                              long long* __restrict__ header) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T || header[H_FLAGS] != 0) return;
    if (tile_cursor[t] != tile_count[t])
        atomicOr(reinterpret_cast<unsigned long long*>(header + H_FLAGS), (unsigned long long)FLAG_TABLE);
}

__global__ void check_kernel(long long* __restrict__ header, int64_t cap) {
    const long long tg = header[H_SCAN_G], tt = header[H_SCAN_T];
    long long flags = header[H_FLAGS];
    if (tg != tt) flags |= FLAG_TABLE;
    if (tg > cap || tg > 0x7fffffffLL) flags |= FLAG_OVERFLOW;
    header[H_TOTAL] = tg > header[H_TOTAL] ? tg : header[H_TOTAL];
    header[H_FLAGS] = flags;
}

// ------------------------------------------------------------------------------------
// Shading
// ------------------------------------------------------------------------------------

// Precision Lambda = L L^T from the raw factor (reference include/shader/shared.cuh:4-25):
// q1 = (L00, L01, L02, L11), s12 = L12, s22 = L22.
__device__ __forceinline__ void precision_from_raw(float t0, float t1, float t2, float t3, float t4,
                                                   float t5, float beta, float4& q1, float& s12,
                                                   float& s22) {
    const float l11 = t0 * t0 + beta;
    const float l12 = t1;
    const float l13 = t2;
    const float l22 = t3 * t3 + beta;
    const float l23 = t4;
    const float l33 = t5 * t5 + beta;
    q1.x = l11 * l11;
    q1.y = l11 * l12;
    q1.z = l11 * l13;
    q1.w = l12 * l12 + l22 * l22;
    s12 = l12 * l13 + l22 * l23;
    s22 = l13 * l13 + l23 * l23 + l33 * l33;
}

// Reference window test (src/mapper/core.cu:166-182): |(p-m).lat| <= r_lat && |(p-m).ax| <= r_ax.
__device__ __forceinline__ bool window_hit(const float3 d, const float3 lat, const float3 ax, float r_lat,
                                           float r_ax) {
    const float dl = fabsf(f3_dot(d, lat));
    const float da = fabsf(f3_dot(d, ax));
    return dl <= r_lat && da <= r_ax;
}

// Quadratic form d^T Lambda d in the reference's term order (include/shader/shared.cuh:41-52),
// which its forward and backward both use: every kernel here takes the same q <= chi2 decision
// for a (pixel, Gaussian) pair as the reference.
__device__ __forceinline__ float quad_form(const float3 d, const float4 q1, const float s12, const float s22) {
    return (q1.x * d.x + q1.y * d.y + q1.z * d.z) * d.x + (q1.y * d.x + q1.w * d.y + s12 * d.z) * d.y +
           (q1.z * d.x + s12 * d.y + s22 * d.z) * d.z;
}

constexpr float kNegHalfLog2e = -0.72134752044448170f;  // -log2(e) / 2

// When the diagonal of L is at least 1e-10 (beta >= 1e-10), the lateral/axial window of the
// reference is the bounding box of the chi-square ellipsoid (the clamps inside window_radii only
// widen it), so q <= chi2 implies the window test up to float rounding and the test can be left
// out; below that the clamp can cut the ellipsoid and the window is applied.
__host__ __device__ __forceinline__ bool window_implied(float beta) { return beta >= 1e-10f; }

__device__ __forceinline__ int find_tile_coords(const Geo& geo, int64_t t, int& tx, int& ty) {
    const int lt = (int)(t - geo.tile_off);
    tx = lt % geo.tx;
    ty = lt / geo.tx;
    return lt;
}

// Pixel (column, row) within its tile of thread / slot k: warp-block-major order.
__device__ __forceinline__ int block_col(int k) { return ((k >> 5) & 1) * BLK_W + (k & (BLK_W - 1)); }
__device__ __forceinline__ int block_row(int k) { return (k >> 6) * BLK_H + ((k & 31) >> 3); }

// One block per tile, one thread per pixel; warp w owns warp block w of the tile and visits
// only the staged Gaussians whose block mask has bit w (the others reach none of its pixels;
// without a slice cull every mask is full and all staged Gaussians are visited in list order).
// A staged Gaussian is three float4: mean + opacity, the precision Lambda, intensity + depth term;
// a fourth holds the window radii, which are computed and tested only when the window is not implied by the
// chi-square test (WINDOWED, chosen by the host from beta). Both binnings therefore run the same
// arithmetic per pair (bit-identical results); the reference's candidate counts come from
// pixel_csr_kernel<true>.
template <int BATCH, bool WINDOWED>
__global__ void __launch_bounds__(TILE_PIX, US3D_UG_FWD_MIN_CTAS)
forward_kernel(int64_t T, int64_t P, const us3d_slice_frame* __restrict__ frames, const int* __restrict__ tile_frame,
               const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
               const blockmask_t* __restrict__ sorted_mask, const long long* __restrict__ header,
               const float4* __restrict__ pack, const float* __restrict__ pixels, float chi2, float beta,
               float bg_alpha, float bg_intensity, float* __restrict__ out_image, float* __restrict__ out_alpha,
               float* __restrict__ out_depth, float2* __restrict__ pixel_aux) {
    constexpr int STRIDE = WINDOWED ? 4 : 3;
    __shared__ float4 s_st[STRIDE * BATCH];
    __shared__ blockmask_t s_blocks[BATCH];
    // per warp: byte offsets into s_st of the staged Gaussians reaching its block
    __shared__ unsigned short s_list[TILE_PIX / 32][BATCH];
    static_assert((BATCH - 1) * STRIDE * 16 <= 0xffff, "staged offsets must fit 16 bits");
    const int64_t t = blockIdx.x;
    if (t >= T || header[H_FLAGS] != 0 || tile_frame[t] < 0) return;
    const Geo geo = load_geo(frames + tile_frame[t]);
    int tx, ty;
    find_tile_coords(geo, t, tx, ty);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int px = tx * TILE + block_col(threadIdx.x);
    const int py = ty * TILE + block_row(threadIdx.x);
    const int64_t p = (int64_t)geo.pix_off + (int64_t)py * geo.W + px;
    const bool valid = px < geo.W && py < geo.H && p < P;
    float3 pv = make_float3(0.f, 0.f, 0.f);
    if (valid) pv = make_float3(pixels[3 * p], pixels[3 * p + 1], pixels[3 * p + 2]);
    const int s0 = tile_start[t];
    const int n = tile_start[t + 1] - s0;
    const bool culled = header[H_MODE] != 0;

    // sums over the contributing pairs; kc, kd: the pairs the reference leaves out of the image
    // (alpha-hat <= 1e-8) but keeps in the backward's numerator / depth sums. Such a pair needs
    // a Gaussian whose alpha-hat can fall to 1e-8 inside the chi-square region; when no staged
    // Gaussian of a batch can (TINY false), the batch runs without that test.
    float sa = 0.f, sc = 0.f, sd = 0.f, kc = 0.f, kd = 0.f;
    auto shade = [&](int off, auto tiny) {  // off: byte offset of the staged Gaussian in s_st
        constexpr bool TINY = decltype(tiny)::value;
        const float4* f = reinterpret_cast<const float4*>(reinterpret_cast<const char*>(s_st) + off);
        const float4 f0 = f[0], f1 = f[1], f2 = f[2];
        const float3 d = make_float3(pv.x - f0.x, pv.y - f0.y, pv.z - f0.z);
        if constexpr (WINDOWED) {
            const float4 f3 = f[3];
            if (!window_hit(d, geo.lat, geo.ax, f3.x, f3.y)) return;
        }
        // The exponential is evaluated for every pair and the sums are predicated: the lanes of
        // a warp (one 8x4 block) run the pair together anyway.
        const float q = quad_form(d, f1, f2.x, f2.y);
        const float ah = f0.w * exp2f(q * kNegHalfLog2e);  // exp(-q/2), as in the backward
        const bool pass = q <= chi2;
        const bool keep = pass && (!TINY || ah > 1e-8f);
        if (keep) {
            sa += ah;
            sc += ah * f2.z;
            sd += ah * f2.w;
        }
        if (TINY && pass && !keep) {
            kc += ah * f2.z;
            kd += ah * f2.w;
        }
    };
    // alpha-hat of a passing pair is at least o * exp2(chi2 * (-log2(e)/2)) up to the rounding
    // of the product and the exponential, which the factor 0.99999 covers
    const float ah_floor = exp2f(chi2 * kNegHalfLog2e) * 0.99999f;
    for (int b0 = 0; b0 < n; b0 += BATCH) {
        const int nb = min(BATCH, n - b0);
        __syncthreads();
        int tiny = 0;
        for (int j = threadIdx.x; j < nb; j += blockDim.x) {
            const int g = sorted_gid[s0 + b0 + j];
            const float4 a = pack[3 * g], b = pack[3 * g + 1], c = pack[3 * g + 2];
            tiny |= !(a.w * ah_floor > 1e-8f);
            const float dterm = f3_dot(f3_sub(make_float3(a.x, a.y, a.z), geo.o), geo.ele);
            float4 q1;
            float s12, s22;
            precision_from_raw(b.x, b.y, b.z, b.w, c.x, c.y, beta, q1, s12, s22);
            s_st[STRIDE * j] = a;
            s_st[STRIDE * j + 1] = q1;
            s_st[STRIDE * j + 2] = make_float4(s12, s22, c.z, dterm);
            if constexpr (WINDOWED) {
                float r_lat, r_ax, r_ele;
                window_radii(b.x, b.y, b.z, b.w, c.x, c.y, chi2, beta, geo.lat, geo.ax, geo.ele, r_lat, r_ax,
                             r_ele);
                s_st[STRIDE * j + 3] = make_float4(r_lat, r_ax, 0.f, 0.f);
            }
            s_blocks[j] = sorted_mask[s0 + b0 + j];
        }
        const bool any_tiny = __syncthreads_or(tiny) != 0;
        // Lanes of an invalid pixel run along (their sums are never stored).
        if (!culled) {
            if (any_tiny)
                for (int j = 0; j < nb; ++j) shade(j * (STRIDE * 16), std::true_type{});
            else
                for (int j = 0; j < nb; ++j) shade(j * (STRIDE * 16), std::false_type{});
            continue;
        }
        // Each warp lists, in staging order, the Gaussians whose mask marks one of its two
        // sub-blocks, then shades them.
        int n_w = 0;
        for (int jc = 0; jc < nb; jc += 32) {
            const int jl = jc + lane;
            const bool mine = jl < nb && ((s_blocks[jl] >> (2 * warp)) & 3u);
            const unsigned bits = __ballot_sync(0xffffffffu, mine);
            if (mine) s_list[warp][n_w + __popc(bits & ((1u << lane) - 1u))] = (unsigned short)(jl * (STRIDE * 16));
            n_w += __popc(bits);
        }
        __syncwarp();
        if (any_tiny)
            for (int k = 0; k < n_w; ++k) shade(s_list[warp][k], std::true_type{});
        else
            for (int k = 0; k < n_w; ++k) shade(s_list[warp][k], std::false_type{});
    }
    if (!valid) return;
    const float alpha_total = sa + bg_alpha;
    const float num = sc + bg_alpha * bg_intensity;
    const float img = num / fmaxf(alpha_total, 1e-8f);
    out_alpha[p] = alpha_total;
    out_image[p] = fmaxf(0.0f, fminf(1.0f, img));
    out_depth[p] = sd / fmaxf(sa, 1e-8f);
    pixel_aux[p] = make_float2(sc + kc, sd + kd);
}

// One block per tile; each thread owns one instance of the tile list at a time and sweeps the
// pixels of the 4x4 sub-blocks its mask marks (pixels and their upstream coefficients sit in
// shared memory in sub-block-major order). Instances are regrouped by the number of marked
// sub-blocks so that the lanes of a warp do similar amounts of work; every instance's sums run
// over its sub-blocks in ascending order, pixel order within sub-block c rotated by c (lanes in
// different sub-blocks mostly read different banks), so its partial does not depend on the
// grouping, and sub-blocks without a contributing pixel add nothing.
// LOSS: dL/dimage comes from the fused per-frame loss (L1 + global SSIM of image against
// target, coefficients per frame in loss_coef; see us3d_ug_loss) and dL/dalpha = dL/ddepth =
// 0; otherwise from d_image, d_alpha, d_depth.
// A pair contributes when q = quad_form <= chi2 (and, WINDOWED, the window is hit): the forward's
// selection, pair for pair.
template <bool LOSS, int THREADS, bool WINDOWED>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)
backward_kernel(int64_t T, int64_t P, const us3d_slice_frame* __restrict__ frames, const int* __restrict__ tile_frame,
                const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
                const int* __restrict__ sorted_inst, const blockmask_t* __restrict__ sorted_mask,
                const long long* __restrict__ header, const float4* __restrict__ pack,
                const float* __restrict__ pixels, const float* __restrict__ d_image, const float* __restrict__ d_alpha,
                const float* __restrict__ d_depth, const float* __restrict__ saved_alpha,
                const float2* __restrict__ pixel_aux, float chi2, float beta, float bg_alpha,
                float bg_intensity, const float* __restrict__ loss_image, const float* __restrict__ loss_target,
                const float4* __restrict__ loss_coef, float4* __restrict__ partial) {
    // Per sub-block c, entries [32 c, 32 c + 32) hold its 16 pixels twice, so that the sweep
    // rotated by c reads 16 consecutive entries from 33 c.
    __shared__ float4 s_pa[2 * TILE_PIX];  // pixel position, dL/dnum
    __shared__ float2 s_pb[2 * TILE_PIX];  // dL/dalpha_total + dL/dsum_alpha (depth), dL/ddepth_weighted
    __shared__ short s_perm[BWD_CHUNK];
    __shared__ int s_class[NSUB + 1];
    const int64_t t = blockIdx.x;
    if (t >= T || header[H_FLAGS] != 0) return;
    const int s0 = tile_start[t];
    const int n = tile_start[t + 1] - s0;
    if (n <= 0 || tile_frame[t] < 0) return;
    const Geo geo = load_geo(frames + tile_frame[t]);
    int tx, ty;
    find_tile_coords(geo, t, tx, ty);
    for (int slot = threadIdx.x; slot < TILE_PIX; slot += THREADS) {
        const int sc = slot / SUB_PIX, within = slot % SUB_PIX;  // sub-block, pixel in it
        const int r = (sc / (TILE / SUB)) * SUB + within / SUB, c = (sc % (TILE / SUB)) * SUB + within % SUB;
        const int e0 = sc * (2 * SUB_PIX) + within, e1 = e0 + SUB_PIX;
        const int64_t p = (int64_t)geo.pix_off + (int64_t)(ty * TILE + r) * geo.W + (tx * TILE + c);
        if (ty * TILE + r < geo.H && tx * TILE + c < geo.W && p < P) {
            // Per-pixel adjoint coefficients (reference src/shader/backward.cu:175-197).
            const float sum_alpha = saved_alpha[p] - bg_alpha;
            const float2 aux = pixel_aux[p];
            const float alpha_total = sum_alpha + bg_alpha;
            const float inv_alpha = 1.0f / fmaxf(alpha_total, 1e-8f);
            const float num = aux.x + bg_alpha * bg_intensity;
            float gI, gA, gD;
            if (LOSS) {
                const float x = loss_image[p], y = loss_target[p];
                const float4 k = loss_coef[tile_frame[t]];
                gI = k.x * (float)((x > y) - (x < y)) + k.y + k.z * x + k.w * y;
                gA = 0.f;
                gD = 0.f;
            } else {
                gI = d_image[p];
                gA = d_alpha[p];
                gD = d_depth[p];
            }
            const float dnum = gI * inv_alpha;
            const float dtot = gA - gI * num * inv_alpha * inv_alpha;
            const float inv_sa = 1.0f / fmaxf(sum_alpha, 1e-8f);
            const float ddw = gD * inv_sa;
            const float dsad = -gD * aux.y * inv_sa * inv_sa;
            s_pa[e0] = s_pa[e1] = make_float4(pixels[3 * p], pixels[3 * p + 1], pixels[3 * p + 2], dnum);
            s_pb[e0] = s_pb[e1] = make_float2(dtot + dsad, ddw);
        } else {
            // outside the frame: zero coefficients make every term of this slot vanish
            s_pa[e0] = s_pa[e1] = make_float4(0.f, 0.f, 0.f, 0.f);
            s_pb[e0] = s_pb[e1] = make_float2(0.f, 0.f);
        }
    }
    const bool culled = header[H_MODE] != 0;  // otherwise every mask is full: no regrouping

    for (int c0 = 0; c0 < n; c0 += BWD_CHUNK) {
        const int nc = min(BWD_CHUNK, n - c0);
        if (threadIdx.x <= NSUB) s_class[threadIdx.x] = 0;
        __syncthreads();
        if (culled) {
            for (int k = threadIdx.x; k < nc; k += blockDim.x)
                atomicAdd(&s_class[NSUB - __popc((unsigned)sorted_mask[s0 + c0 + k])], 1);
            __syncthreads();
            if (threadIdx.x == 0) {
                int acc = 0;
                for (int i = 0; i <= NSUB; ++i) {
                    const int v = s_class[i];
                    s_class[i] = acc;
                    acc += v;
                }
            }
            __syncthreads();
            for (int k = threadIdx.x; k < nc; k += blockDim.x)
                s_perm[atomicAdd(&s_class[NSUB - __popc((unsigned)sorted_mask[s0 + c0 + k])], 1)] = (short)k;
            __syncthreads();
        }

        // Rounds of THREADS instances; the regrouped order runs from the most marked sub-blocks
        // to the fewest, so odd rounds hand the warps their slices in reverse (serpentine) and
        // no warp takes the heaviest slice of every round.
        for (int r0 = 0; r0 < nc; r0 += THREADS) {
            const int wi = threadIdx.x >> 5;
            const int i = r0 + (((r0 / THREADS) & 1) ? (THREADS / 32 - 1 - wi) * 32 + (threadIdx.x & 31)
                                                     : (int)threadIdx.x);
            if (i >= nc) continue;
            const int k = s0 + c0 + (culled ? (int)s_perm[i] : i);
            const int g = sorted_gid[k];
            const int inst = sorted_inst[k];
            const unsigned blocks = sorted_mask[k];
            const float4 a = pack[3 * g], b = pack[3 * g + 1], c = pack[3 * g + 2];
            float4 q1;
            float s12, s22;
            precision_from_raw(b.x, b.y, b.z, b.w, c.x, c.y, beta, q1, s12, s22);
            const float3 m = make_float3(a.x, a.y, a.z);
            const float dterm = f3_dot(f3_sub(m, geo.o), geo.ele);
            const float o = a.w, ci = c.z;
            float r_lat = 0.f, r_ax = 0.f, r_ele;
            if (WINDOWED)
                window_radii(b.x, b.y, b.z, b.w, c.x, c.y, chi2, beta, geo.lat, geo.ax, geo.ele, r_lat, r_ax, r_ele);
            float acc_c = 0.f, acc_o = 0.f, acc_e = 0.f;
            float sdx = 0.f, sdy = 0.f, sdz = 0.f;
            float sxx = 0.f, sxy = 0.f, sxz = 0.f, syy = 0.f, syz = 0.f, szz = 0.f;
            for (unsigned mb = blocks; mb != 0u; mb &= mb - 1u) {
                const int blk = __ffs(mb) - 1;
                const float4* pa_b = s_pa + blk * (2 * SUB_PIX + 1);
                const float2* pb_b = s_pb + blk * (2 * SUB_PIX + 1);
#pragma unroll
                for (int jj = 0; jj < SUB_PIX; ++jj) {
                    const float4 pa = pa_b[jj];
                    const float3 d = make_float3(pa.x - m.x, pa.y - m.y, pa.z - m.z);
                    if constexpr (WINDOWED) {
                        if (!window_hit(d, geo.lat, geo.ax, r_lat, r_ax)) continue;
                    }
                    // A pair failing the chi-square test gets w = 0, so that every term it adds is
                    // an exact zero: no branch in the unrolled sweep. exp(-q/2) = 2^(q c) with
                    // c = -log2(e)/2.
                    const float q = quad_form(d, q1, s12, s22);
                    const float2 pb = pb_b[jj];
                    const float w = q <= chi2 ? exp2f(q * kNegHalfLog2e) : 0.0f;
                    const float dah = pa.w * ci + pb.x + pb.y * dterm;
                    const float dw = dah * w;  // dL/dopacity term; dL/dq = -o dw / 2 (o, -1/2 applied below)
                    acc_c += pa.w * w;
                    acc_o += dw;
                    acc_e += pb.y * w;
                    const float ux = dw * d.x, uy = dw * d.y, uz = dw * d.z;
                    sdx += ux;
                    sdy += uy;
                    sdz += uz;
                    sxx += ux * d.x;
                    sxy += ux * d.y;
                    sxz += ux * d.z;
                    syy += uy * d.y;
                    syz += uy * d.z;
                    szz += uz * d.z;
                }
            }
            // The pairs' common factors, applied once per instance: -o/2 of dL/dq, o of the
            // alpha-hat sums.
            const float nh = -0.5f * o;
            sdx *= nh; sdy *= nh; sdz *= nh;
            sxx *= nh; sxy *= nh; sxz *= nh; syy *= nh; syz *= nh; szz *= nh;
            acc_c *= o;
            acc_e *= o;
            // d/dmean = -2 Lambda sum(dq d) + sum(ddw * ah) * ele (reference backward.cu:218-228).
            const float vx = q1.x * sdx + q1.y * sdy + q1.z * sdz;
            const float vy = q1.y * sdx + q1.w * sdy + s12 * sdz;
            const float vz = q1.z * sdx + s12 * sdy + s22 * sdz;
            // dL/dL (lower triangle) from dL/dLambda = sum(dq d d^T) (reference backward.cu:230-255).
            const float l11 = b.x * b.x + beta, l12 = b.y, l13 = b.z;
            const float l22 = b.w * b.w + beta, l23 = c.x, l33 = c.y * c.y + beta;
            const float dl11 = 2.0f * (sxx * l11 + sxy * l12 + sxz * l13);
            const float dl12 = 2.0f * (sxy * l11 + syy * l12 + syz * l13);
            const float dl13 = 2.0f * (sxz * l11 + syz * l12 + szz * l13);
            const float dl22 = 2.0f * (syy * l22 + syz * l23);
            const float dl23 = 2.0f * (syz * l22 + szz * l23);
            const float dl33 = 2.0f * (szz * l33);
            float4* out = partial + 3 * (int64_t)inst;
            out[0] = make_float4(-2.0f * vx + acc_e * geo.ele.x, -2.0f * vy + acc_e * geo.ele.y,
                                 -2.0f * vz + acc_e * geo.ele.z, acc_o);
            out[1] = make_float4(dl11 * (2.0f * b.x), dl12, dl13, dl22 * (2.0f * b.w));
            out[2] = make_float4(dl23, dl33 * (2.0f * c.y), acc_c, 0.f);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------
// Backward with packed FP32 pairs (sm_100 f32x2): two pixels per instruction
// ------------------------------------------------------------------------------------
//
// Same work split and pair selection as backward_kernel (window implied by the chi-square
// test), but each thread sweeps the two horizontally adjacent pixels of a sub-block row pair
// at once: the pixels' positions and adjoint coefficients are staged as lane pairs, the
// instance's constants are broadcast into pairs, and the quadratic form, the adjoint products
// and the twelve gradient sums run as fma/mul/add.rn.ftz.f32x2, each lane rounding exactly as
// the scalar instruction. The quadratic form keeps the reference's term order with the
// contractions of the compiled scalar expression (QUAD_ORDER), so each lane's q, and hence the
// q <= chi2 decision, is bit-identical to the forward's. The sums of even and odd pixels are
// kept apart and added once per instance (deterministic; a different but fixed summation
// order from backward_kernel's).

// The compiled scalar a*b + c*d + e*f rounds as fma(e, f, fma(a, b, c*d)) (order 2; checked
// on B200 against the scalar expression, zero differences in 6.7e7 random quadratic forms).
#ifndef US3D_UG_QUAD_ORDER
#define US3D_UG_QUAD_ORDER 2
#endif

typedef unsigned long long f32x2;

__device__ __forceinline__ f32x2 pk2(float lo, float hi) {
    f32x2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void up2(f32x2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("add.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
    f32x2 r;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
    f32x2 r;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}
// a*b + c*d + e*f with the compiled scalar expression's contractions
__device__ __forceinline__ f32x2 tri2(f32x2 a, f32x2 b, f32x2 c, f32x2 d, f32x2 e, f32x2 f) {
#if US3D_UG_QUAD_ORDER == 1
    return fma2(e, f, fma2(c, d, mul2(a, b)));
#else
    return fma2(e, f, fma2(a, b, mul2(c, d)));
#endif
}

// Forward with two pixels per thread in FP32x2 arithmetic. One 128-thread block per tile; warp
// W (0..3) owns the 8x8 quadrant (column 8 (W & 1), row 8 (W >> 1)), i.e. 4x4 sub-blocks of
// bands 2 (W >> 1) and 2 (W >> 1) + 1 and quarters 2 (W & 1) and 2 (W & 1) + 1, and visits a
// staged Gaussian when its mask marks any of those four. Lane l shades pixels (x, y) and
// (x, y + 4) of the quadrant, x = l & 7, y = l >> 3. Staged values are stored twice, {v, v},
// so that one float4 load gives two operand pairs. Every lane rounds as forward_kernel does:
// d, the quadratic form (the reference's term order with the contractions of the compiled
// scalar expression, tri2), q * (-log2(e)/2), the exponential (scalar ex2), ah = o * e and the
// sums, where a pair that does not contribute adds an exact zero (fma(0, v, s) = s); a Gaussian
// visited because it marks another sub-block of the quadrant fails the chi-square test on
// every pixel of this one and adds zeros too. Images, alpha, depth and the no-skip sums are
// therefore bit-identical to forward_kernel's. (Not for the windowed case, beta < 1e-10.)
template <int BATCH>
__global__ void __launch_bounds__(128, 8)
forward_packed_kernel(int64_t T, int64_t P, const us3d_slice_frame* __restrict__ frames,
                      const int* __restrict__ tile_frame, const int* __restrict__ tile_start,
                      const int* __restrict__ sorted_gid, const blockmask_t* __restrict__ sorted_mask,
                      const long long* __restrict__ header, const float4* __restrict__ pack,
                      const float* __restrict__ pixels, float chi2, float beta, float bg_alpha, float bg_intensity,
                      float* __restrict__ out_image, float* __restrict__ out_alpha, float* __restrict__ out_depth,
                      float2* __restrict__ pixel_aux) {
    constexpr int REC = 6;  // float4 per staged Gaussian: {mx,mx,my,my} {mz,mz,o,o} {q0,q0,q1,q1}
                            // {q2,q2,q3,q3} {s12,s12,s22,s22} {c,c,dt,dt}
    __shared__ float4 s_st[REC * BATCH];
    __shared__ blockmask_t s_blocks[BATCH];
    __shared__ unsigned short s_list[4][BATCH];
    static_assert((BATCH - 1) * REC * 16 <= 0xffff, "staged offsets must fit 16 bits");
    const int64_t t = blockIdx.x;
    if (t >= T || header[H_FLAGS] != 0 || tile_frame[t] < 0) return;
    const Geo geo = load_geo(frames + tile_frame[t]);
    int tx, ty;
    find_tile_coords(geo, t, tx, ty);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int qc = warp & 1, qr = warp >> 1;
    const int px = tx * TILE + 8 * qc + (lane & 7);
    const int py0 = ty * TILE + 8 * qr + (lane >> 3), py1 = py0 + 4;
    const int64_t p0 = (int64_t)geo.pix_off + (int64_t)py0 * geo.W + px;
    const int64_t p1 = (int64_t)geo.pix_off + (int64_t)py1 * geo.W + px;
    const bool valid0 = px < geo.W && py0 < geo.H && p0 < P;
    const bool valid1 = px < geo.W && py1 < geo.H && p1 < P;
    float3 pa = make_float3(0.f, 0.f, 0.f), pb = make_float3(0.f, 0.f, 0.f);
    if (valid0) pa = make_float3(pixels[3 * p0], pixels[3 * p0 + 1], pixels[3 * p0 + 2]);
    if (valid1) pb = make_float3(pixels[3 * p1], pixels[3 * p1 + 1], pixels[3 * p1 + 2]);
    const f32x2 PX = pk2(pa.x, pb.x), PY = pk2(pa.y, pb.y), PZ = pk2(pa.z, pb.z);
    const f32x2 CE = pk2(kNegHalfLog2e, kNegHalfLog2e);
    const int s0 = tile_start[t];
    const int n = tile_start[t + 1] - s0;
    const bool culled = header[H_MODE] != 0;
    const unsigned qmask = 0x33u << (8 * qr + 2 * qc);  // the quadrant's four sub-blocks

    f32x2 sa = pk2(0.f, 0.f), sc = sa, sd = sa, kc = sa, kd = sa;
    auto shade = [&](int off) {  // off: byte offset of the staged Gaussian in s_st
        const float4* f = reinterpret_cast<const float4*>(reinterpret_cast<const char*>(s_st) + off);
        const float4 f0 = f[0], f1 = f[1], f2 = f[2], f3 = f[3], f4 = f[4], f5 = f[5];
        const f32x2 dx = sub2(PX, pk2(f0.x, f0.y)), dy = sub2(PY, pk2(f0.z, f0.w)), dz = sub2(PZ, pk2(f1.x, f1.y));
        const f32x2 Q0 = pk2(f2.x, f2.y), Q1 = pk2(f2.z, f2.w), Q2 = pk2(f3.x, f3.y), Q3 = pk2(f3.z, f3.w);
        const f32x2 S12 = pk2(f4.x, f4.y), S22 = pk2(f4.z, f4.w);
        const f32x2 t0 = tri2(Q0, dx, Q1, dy, Q2, dz);
        const f32x2 t1 = tri2(Q1, dx, Q3, dy, S12, dz);
        const f32x2 t2 = tri2(Q2, dx, S12, dy, S22, dz);
        const f32x2 q = tri2(t0, dx, t1, dy, t2, dz);
        float q0, q1, e0, e1;
        up2(q, q0, q1);
        up2(mul2(q, CE), e0, e1);
        float ah0, ah1;
        up2(mul2(pk2(f1.z, f1.w), pk2(exp2f(e0), exp2f(e1))), ah0, ah1);  // o * exp(-q/2)
        const bool pass0 = q0 <= chi2, pass1 = q1 <= chi2;
        const bool keep0 = pass0 && ah0 > 1e-8f, keep1 = pass1 && ah1 > 1e-8f;
        const f32x2 ak = pk2(keep0 ? ah0 : 0.f, keep1 ? ah1 : 0.f);
        const f32x2 C = pk2(f5.x, f5.y), D = pk2(f5.z, f5.w);
        sa = add2(sa, ak);
        sc = fma2(ak, C, sc);
        sd = fma2(ak, D, sd);
        if (pass0 != keep0 || pass1 != keep1) {  // the reference's alpha-hat <= 1e-8 pairs (rare)
            const f32x2 ap = pk2(pass0 && !keep0 ? ah0 : 0.f, pass1 && !keep1 ? ah1 : 0.f);
            kc = fma2(ap, C, kc);
            kd = fma2(ap, D, kd);
        }
    };
    for (int b0 = 0; b0 < n; b0 += BATCH) {
        const int nb = min(BATCH, n - b0);
        __syncthreads();
        for (int j = threadIdx.x; j < nb; j += blockDim.x) {
            const int g = sorted_gid[s0 + b0 + j];
            const float4 a = pack[3 * g], b = pack[3 * g + 1], c = pack[3 * g + 2];
            const float dterm = f3_dot(f3_sub(make_float3(a.x, a.y, a.z), geo.o), geo.ele);
            float4 q1;
            float s12, s22;
            precision_from_raw(b.x, b.y, b.z, b.w, c.x, c.y, beta, q1, s12, s22);
            float4* d = s_st + REC * j;
            d[0] = make_float4(a.x, a.x, a.y, a.y);
            d[1] = make_float4(a.z, a.z, a.w, a.w);
            d[2] = make_float4(q1.x, q1.x, q1.y, q1.y);
            d[3] = make_float4(q1.z, q1.z, q1.w, q1.w);
            d[4] = make_float4(s12, s12, s22, s22);
            d[5] = make_float4(c.z, c.z, dterm, dterm);
            s_blocks[j] = sorted_mask[s0 + b0 + j];
        }
        __syncthreads();
        if (!culled) {
            for (int j = 0; j < nb; ++j) shade(j * (REC * 16));
            continue;
        }
        int n_w = 0;
        for (int jc = 0; jc < nb; jc += 32) {
            const int jl = jc + lane;
            const bool mine = jl < nb && (s_blocks[jl] & qmask);
            const unsigned bits = __ballot_sync(0xffffffffu, mine);
            if (mine) s_list[warp][n_w + __popc(bits & ((1u << lane) - 1u))] = (unsigned short)(jl * (REC * 16));
            n_w += __popc(bits);
        }
        __syncwarp();
        for (int k = 0; k < n_w; ++k) shade(s_list[warp][k]);
    }
    float a0, a1, c0, c1, d0, d1, kc0, kc1, kd0, kd1;
    up2(sa, a0, a1);
    up2(sc, c0, c1);
    up2(sd, d0, d1);
    up2(kc, kc0, kc1);
    up2(kd, kd0, kd1);
    auto store = [&](int64_t p, float s_a, float s_c, float s_d, float k_c, float k_d) {
        const float alpha_total = s_a + bg_alpha;
        const float num = s_c + bg_alpha * bg_intensity;
        const float img = num / fmaxf(alpha_total, 1e-8f);
        out_alpha[p] = alpha_total;
        out_image[p] = fmaxf(0.0f, fminf(1.0f, img));
        out_depth[p] = s_d / fmaxf(s_a, 1e-8f);
        pixel_aux[p] = make_float2(s_c + k_c, s_d + k_d);
    };
    if (valid0) store(p0, a0, c0, d0, kc0, kd0);
    if (valid1) store(p1, a1, c1, d1, kc1, kd1);
}

template <bool LOSS, int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS)
backward_packed_kernel(int64_t T, int64_t P, const us3d_slice_frame* __restrict__ frames,
                       const int* __restrict__ tile_frame, const int* __restrict__ tile_start,
                       const int* __restrict__ sorted_gid, const int* __restrict__ sorted_inst,
                       const blockmask_t* __restrict__ sorted_mask, const long long* __restrict__ header,
                       const float4* __restrict__ pack, const float* __restrict__ pixels,
                       const float* __restrict__ d_image, const float* __restrict__ d_alpha,
                       const float* __restrict__ d_depth, const float* __restrict__ saved_alpha,
                       const float2* __restrict__ pixel_aux, float chi2, float beta, float bg_alpha,
                       float bg_intensity, const float* __restrict__ loss_image, const float* __restrict__ loss_target,
                       const float4* __restrict__ loss_coef, float4* __restrict__ partial) {
    constexpr int PAIRS = TILE_PIX / 2;       // 128 pixel pairs per tile
    constexpr int SUB_PAIRS = SUB_PIX / 2;    // 8 per sub-block
    // Per sub-block c, entries [16 c, 16 c + 16) hold its 8 pairs twice, so that the sweep
    // rotated by c mod 8 reads 8 consecutive entries from 16 c + (c mod 8).
    __shared__ float4 s_a[2 * PAIRS];  // (x0, x1, y0, y1)
    __shared__ float4 s_b[2 * PAIRS];  // (z0, z1, dnum0, dnum1)
    __shared__ float4 s_c[2 * PAIRS];  // (dtot0, dtot1, ddw0, ddw1)
    __shared__ short s_perm[BWD_CHUNK];
    __shared__ int s_class[NSUB + 1];
    const int64_t t = blockIdx.x;
    if (t >= T || header[H_FLAGS] != 0) return;
    const int s0 = tile_start[t];
    const int n = tile_start[t + 1] - s0;
    if (n <= 0 || tile_frame[t] < 0) return;
    const Geo geo = load_geo(frames + tile_frame[t]);
    int tx, ty;
    find_tile_coords(geo, t, tx, ty);
    for (int ps = threadIdx.x; ps < PAIRS; ps += THREADS) {
        const int sc = ps / SUB_PAIRS, wp = ps % SUB_PAIRS;
        float px[2], py[2], pz[2], dn[2], dt[2], dd[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int within = 2 * wp + h;
            const int r = (sc / (TILE / SUB)) * SUB + within / SUB, c = (sc % (TILE / SUB)) * SUB + within % SUB;
            const int64_t p = (int64_t)geo.pix_off + (int64_t)(ty * TILE + r) * geo.W + (tx * TILE + c);
            px[h] = py[h] = pz[h] = dn[h] = dt[h] = dd[h] = 0.f;  // outside the frame: every term vanishes
            if (ty * TILE + r < geo.H && tx * TILE + c < geo.W && p < P) {
                // Per-pixel adjoint coefficients (reference src/shader/backward.cu:175-197).
                const float sum_alpha = saved_alpha[p] - bg_alpha;
                const float2 aux = pixel_aux[p];
                const float alpha_total = sum_alpha + bg_alpha;
                const float inv_alpha = 1.0f / fmaxf(alpha_total, 1e-8f);
                const float num = aux.x + bg_alpha * bg_intensity;
                float gI, gA, gD;
                if (LOSS) {
                    const float x = loss_image[p], y = loss_target[p];
                    const float4 k = loss_coef[tile_frame[t]];
                    gI = k.x * (float)((x > y) - (x < y)) + k.y + k.z * x + k.w * y;
                    gA = 0.f;
                    gD = 0.f;
                } else {
                    gI = d_image[p];
                    gA = d_alpha[p];
                    gD = d_depth[p];
                }
                const float inv_sa = 1.0f / fmaxf(sum_alpha, 1e-8f);
                px[h] = pixels[3 * p];
                py[h] = pixels[3 * p + 1];
                pz[h] = pixels[3 * p + 2];
                dn[h] = gI * inv_alpha;
                dt[h] = (gA - gI * num * inv_alpha * inv_alpha) + (-gD * aux.y * inv_sa * inv_sa);
                dd[h] = gD * inv_sa;
            }
        }
        const int e0 = sc * (2 * SUB_PAIRS) + wp, e1 = e0 + SUB_PAIRS;
        s_a[e0] = s_a[e1] = make_float4(px[0], px[1], py[0], py[1]);
        s_b[e0] = s_b[e1] = make_float4(pz[0], pz[1], dn[0], dn[1]);
        s_c[e0] = s_c[e1] = make_float4(dt[0], dt[1], dd[0], dd[1]);
    }
    const bool culled = header[H_MODE] != 0;
    const f32x2 zero2 = pk2(0.f, 0.f);

    for (int c0 = 0; c0 < n; c0 += BWD_CHUNK) {
        const int nc = min(BWD_CHUNK, n - c0);
        if (threadIdx.x <= NSUB) s_class[threadIdx.x] = 0;
        __syncthreads();
        if (culled) {
            for (int k = threadIdx.x; k < nc; k += blockDim.x)
                atomicAdd(&s_class[NSUB - __popc((unsigned)sorted_mask[s0 + c0 + k])], 1);
            __syncthreads();
            if (threadIdx.x == 0) {
                int acc = 0;
                for (int i = 0; i <= NSUB; ++i) {
                    const int v = s_class[i];
                    s_class[i] = acc;
                    acc += v;
                }
            }
            __syncthreads();
            for (int k = threadIdx.x; k < nc; k += blockDim.x)
                s_perm[atomicAdd(&s_class[NSUB - __popc((unsigned)sorted_mask[s0 + c0 + k])], 1)] = (short)k;
            __syncthreads();
        }
        for (int r0 = 0; r0 < nc; r0 += THREADS) {
            const int wi = threadIdx.x >> 5;
            const int i = r0 + (((r0 / THREADS) & 1) ? (THREADS / 32 - 1 - wi) * 32 + (threadIdx.x & 31)
                                                     : (int)threadIdx.x);
            if (i >= nc) continue;
            const int k = s0 + c0 + (culled ? (int)s_perm[i] : i);
            const int g = sorted_gid[k];
            const int inst = sorted_inst[k];
            const unsigned blocks = sorted_mask[k];
            const float4 a = pack[3 * g], b = pack[3 * g + 1], c = pack[3 * g + 2];
            float4 q1;
            float s12, s22;
            precision_from_raw(b.x, b.y, b.z, b.w, c.x, c.y, beta, q1, s12, s22);
            const float dterm = f3_dot(f3_sub(make_float3(a.x, a.y, a.z), geo.o), geo.ele);
            const float o = a.w, ci = c.z;
            const f32x2 MX = pk2(a.x, a.x), MY = pk2(a.y, a.y), MZ = pk2(a.z, a.z);
            const f32x2 Q0 = pk2(q1.x, q1.x), Q1 = pk2(q1.y, q1.y), Q2 = pk2(q1.z, q1.z), Q3 = pk2(q1.w, q1.w);
            const f32x2 S12 = pk2(s12, s12), S22 = pk2(s22, s22), CI = pk2(ci, ci), DT = pk2(dterm, dterm);
            f32x2 acc_c = zero2, acc_o = zero2, acc_e = zero2, sdx = zero2, sdy = zero2, sdz = zero2;
            f32x2 sxx = zero2, sxy = zero2, sxz = zero2, syy = zero2, syz = zero2, szz = zero2;
            for (unsigned mb = blocks; mb != 0u; mb &= mb - 1u) {
                const int blk = __ffs(mb) - 1;
                const int base = blk * (2 * SUB_PAIRS) + (blk & (SUB_PAIRS - 1));
#pragma unroll
                for (int jj = 0; jj < SUB_PAIRS; ++jj) {
                    const float4 va = s_a[base + jj], vb = s_b[base + jj], vc = s_c[base + jj];
                    const f32x2 dx = sub2(pk2(va.x, va.y), MX), dy = sub2(pk2(va.z, va.w), MY),
                                dz = sub2(pk2(vb.x, vb.y), MZ);
                    const f32x2 dn = pk2(vb.z, vb.w), gx = pk2(vc.x, vc.y), gy = pk2(vc.z, vc.w);
                    // quadratic form in the reference's term order (quad_form), per lane
                    const f32x2 t0 = tri2(Q0, dx, Q1, dy, Q2, dz);
                    const f32x2 t1 = tri2(Q1, dx, Q3, dy, S12, dz);
                    const f32x2 t2 = tri2(Q2, dx, S12, dy, S22, dz);
                    const f32x2 q = tri2(t0, dx, t1, dy, t2, dz);
                    float q0, q1v;
                    up2(q, q0, q1v);
                    const float w0 = q0 <= chi2 ? exp2f(q0 * kNegHalfLog2e) : 0.0f;
                    const float w1 = q1v <= chi2 ? exp2f(q1v * kNegHalfLog2e) : 0.0f;
                    const f32x2 w = pk2(w0, w1);
                    const f32x2 dah = fma2(gy, DT, fma2(dn, CI, gx));
                    const f32x2 dw = mul2(dah, w);
                    acc_c = fma2(dn, w, acc_c);
                    acc_o = add2(acc_o, dw);
                    acc_e = fma2(gy, w, acc_e);
                    const f32x2 ux = mul2(dw, dx), uy = mul2(dw, dy), uz = mul2(dw, dz);
                    sdx = add2(sdx, ux);
                    sdy = add2(sdy, uy);
                    sdz = add2(sdz, uz);
                    sxx = fma2(ux, dx, sxx);
                    sxy = fma2(ux, dy, sxy);
                    sxz = fma2(ux, dz, sxz);
                    syy = fma2(uy, dy, syy);
                    syz = fma2(uy, dz, syz);
                    szz = fma2(uz, dz, szz);
                }
            }
            auto fold = [](f32x2 v) {
                float lo, hi;
                up2(v, lo, hi);
                return lo + hi;
            };
            // The pairs' common factors, applied once per instance: -o/2 of dL/dq, o of the
            // alpha-hat sums.
            const float nh = -0.5f * o;
            const float Sdx = fold(sdx) * nh, Sdy = fold(sdy) * nh, Sdz = fold(sdz) * nh;
            const float Sxx = fold(sxx) * nh, Sxy = fold(sxy) * nh, Sxz = fold(sxz) * nh;
            const float Syy = fold(syy) * nh, Syz = fold(syz) * nh, Szz = fold(szz) * nh;
            const float Ac = fold(acc_c) * o, Ao = fold(acc_o), Ae = fold(acc_e) * o;
            const float vx = q1.x * Sdx + q1.y * Sdy + q1.z * Sdz;
            const float vy = q1.y * Sdx + q1.w * Sdy + s12 * Sdz;
            const float vz = q1.z * Sdx + s12 * Sdy + s22 * Sdz;
            const float l11 = b.x * b.x + beta, l12 = b.y, l13 = b.z;
            const float l22 = b.w * b.w + beta, l23 = c.x, l33 = c.y * c.y + beta;
            const float dl11 = 2.0f * (Sxx * l11 + Sxy * l12 + Sxz * l13);
            const float dl12 = 2.0f * (Sxy * l11 + Syy * l12 + Syz * l13);
            const float dl13 = 2.0f * (Sxz * l11 + Syz * l12 + Szz * l13);
            const float dl22 = 2.0f * (Syy * l22 + Syz * l23);
            const float dl23 = 2.0f * (Syz * l22 + Szz * l23);
            const float dl33 = 2.0f * (Szz * l33);
            float4* out = partial + 3 * (int64_t)inst;
            out[0] = make_float4(-2.0f * vx + Ae * geo.ele.x, -2.0f * vy + Ae * geo.ele.y,
                                 -2.0f * vz + Ae * geo.ele.z, Ao);
            out[1] = make_float4(dl11 * (2.0f * b.x), dl12, dl13, dl22 * (2.0f * b.w));
            out[2] = make_float4(dl23, dl33 * (2.0f * c.y), Ac, 0.f);
        }
        __syncthreads();
    }
}

// Per-Gaussian gradient: the sum of its instances' 48-byte partials in instance order.
// REDUCE_COLS threads per Gaussian, thread f summing float4 column f, so that a Gaussian's
// threads read each partial together and many Gaussians' loads are in flight; the sums are the
// ones a thread summing all columns would form.
constexpr int REDUCE_COLS = 3;                      // float4 columns of a partial record
constexpr int REDUCE_THREADS = 64 * REDUCE_COLS;     // 64 Gaussians per block
__global__ void __launch_bounds__(REDUCE_THREADS)
reduce_kernel(int64_t G, const int* __restrict__ inst_offset, const long long* __restrict__ header,
              const float4* __restrict__ partial, float* __restrict__ d_means, float* __restrict__ d_tril,
              float* __restrict__ d_opac, float* __restrict__ d_inten) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t g = t / REDUCE_COLS;
    const int f = (int)(t % REDUCE_COLS);
    if (g >= G) return;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    if (header[H_FLAGS] == 0) {
        const int i1 = inst_offset[g + 1];
        int i = inst_offset[g];
        // four instances' loads in flight at a time; the sums keep instance order
        for (; i + 4 <= i1; i += 4) {
            float4 v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = partial[3 * (int64_t)(i + u) + f];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a.x += v[u].x;
                a.y += v[u].y;
                a.z += v[u].z;
                a.w += v[u].w;
            }
        }
        for (; i < i1; ++i) {
            const float4 v = partial[3 * (int64_t)i + f];
            a.x += v.x;
            a.y += v.y;
            a.z += v.z;
            a.w += v.w;
        }
    }
    if (f == 0) {
        d_means[3 * g + 0] = a.x;
        d_means[3 * g + 1] = a.y;
        d_means[3 * g + 2] = a.z;
        d_opac[g] = a.w;
    } else if (f == 1) {
        d_tril[6 * g + 0] = a.x;
        d_tril[6 * g + 1] = a.y;
        d_tril[6 * g + 2] = a.z;
        d_tril[6 * g + 3] = a.w;
    } else {
        d_tril[6 * g + 4] = a.x;
        d_tril[6 * g + 5] = a.y;
        d_inten[g] = a.z;
    }
}

// Per-pixel candidates of a full (reference) binning in tile-list order: the pixels' window
// hits (reference src/mapper/core.cu:166-182). COUNT: their number per pixel into out_counts;
// otherwise their Gaussian indices from offsets[p] on (src/mapper/core.cu:237-287).
template <bool COUNT>
__global__ void __launch_bounds__(TILE_PIX)
pixel_csr_kernel(int64_t T, int64_t P, const us3d_slice_frame* __restrict__ frames, const int* __restrict__ tile_frame,
                 const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
                 const long long* __restrict__ header, const float4* __restrict__ pack,
                 const float* __restrict__ pixels, float chi2, float beta, const int* __restrict__ offsets,
                 int* __restrict__ out_indices, int* __restrict__ out_counts) {
    __shared__ float4 s_m[FWD_BATCH];   // mean, gaussian index (as float bits)
    __shared__ float2 s_r[FWD_BATCH];   // r_lat, r_ax
    const int64_t t = blockIdx.x;
    // candidate lists exist only for a full (reference) binning
    if (t >= T || header[H_FLAGS] != 0 || header[H_MODE] != 0 || tile_frame[t] < 0) return;
    const Geo geo = load_geo(frames + tile_frame[t]);
    int tx, ty;
    find_tile_coords(geo, t, tx, ty);
    const int px = tx * TILE + (threadIdx.x & (TILE - 1));
    const int py = ty * TILE + (threadIdx.x / TILE);
    const int64_t p = (int64_t)geo.pix_off + (int64_t)py * geo.W + px;
    const bool valid = px < geo.W && py < geo.H && p < P;
    float3 pv = make_float3(0.f, 0.f, 0.f);
    int wp = 0;
    if (valid) {
        pv = make_float3(pixels[3 * p], pixels[3 * p + 1], pixels[3 * p + 2]);
        if (!COUNT) wp = offsets[p];
    }
    const int s0 = tile_start[t];
    const int n = tile_start[t + 1] - s0;
    for (int b0 = 0; b0 < n; b0 += FWD_BATCH) {
        const int nb = min(FWD_BATCH, n - b0);
        __syncthreads();
        for (int j = threadIdx.x; j < nb; j += blockDim.x) {
            const int g = sorted_gid[s0 + b0 + j];
            const float4 a = pack[3 * g], b = pack[3 * g + 1], c = pack[3 * g + 2];
            float r_lat, r_ax, r_ele;
            window_radii(b.x, b.y, b.z, b.w, c.x, c.y, chi2, beta, geo.lat, geo.ax, geo.ele, r_lat, r_ax, r_ele);
            s_m[j] = make_float4(a.x, a.y, a.z, __int_as_float(g));
            s_r[j] = make_float2(r_lat, r_ax);
        }
        __syncthreads();
        if (valid) {
            for (int j = 0; j < nb; ++j) {
                const float4 m = s_m[j];
                const float2 r = s_r[j];
                const float3 d = make_float3(pv.x - m.x, pv.y - m.y, pv.z - m.z);
                if (window_hit(d, geo.lat, geo.ax, r.x, r.y)) {
                    if (!COUNT) out_indices[wp] = __float_as_int(m.w);
                    ++wp;
                }
            }
        }
    }
    if (COUNT && valid) out_counts[p] = wp;
}

__global__ void export_kernel(int tile_off, int n_tiles_frame, const int* __restrict__ tile_start,
                              const unsigned long long* __restrict__ keys, const int* __restrict__ sorted_gid,
                              int64_t* __restrict__ out_keys, int* __restrict__ out_values,
                              int* __restrict__ rs, int* __restrict__ re) {
    const int lt = blockIdx.x;
    if (lt >= n_tiles_frame) return;
    const int base = tile_start[tile_off];
    const int s0 = tile_start[tile_off + lt];
    const int s1 = tile_start[tile_off + lt + 1];
    if (threadIdx.x == 0) {
        rs[lt] = (s1 > s0) ? s0 - base : -1;
        re[lt] = (s1 > s0) ? s1 - base : -1;
    }
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) {
        out_keys[s - base] = (int64_t)(((unsigned long long)(uint32_t)lt << 32) | (keys[s] >> 32));
        out_values[s - base] = sorted_gid[s];
    }
}

}  // namespace ug
}  // namespace us3d

using namespace us3d;
using namespace us3d::ug;

// Per-device flag: the large-bucket sort kernel's shared-memory limit has been raised.
static bool g_sort_attr_done[128];

// Launch shapes of the shading kernels (process-wide; read at every launch).
static std::atomic<int> g_fwd_batch{FWD_BATCH};
static std::atomic<int> g_bwd_threads{BWD_THREADS};
// Backward kernel variant: 0 scalar FP32, 1 packed FP32 pairs (backward_packed_kernel).
static std::atomic<int> g_bwd_variant{0};
static std::atomic<int> g_fwd_variant{0};

extern "C" int us3d_ug_set_launch_config(int32_t forward_batch, int32_t backward_threads) {
    US3D_CHECK_ARG(forward_batch == 128 || forward_batch == 256 || forward_batch == 512,
                   "forward_batch must be 128, 256 or 512 (got %d)", forward_batch);
    US3D_CHECK_ARG(backward_threads == 128 || backward_threads == 256,
                   "backward_threads must be 128 or 256 (got %d)", backward_threads);
    g_fwd_batch.store(forward_batch);
    g_bwd_threads.store(backward_threads);
    return US3D_OK;
}

extern "C" int us3d_ug_get_launch_config(int32_t* forward_batch, int32_t* backward_threads) {
    if (forward_batch) *forward_batch = g_fwd_batch.load();
    if (backward_threads) *backward_threads = g_bwd_threads.load();
    return US3D_OK;
}

extern "C" int us3d_ug_set_backward_variant(int32_t variant) {
    US3D_CHECK_ARG(variant == 0 || variant == 1, "backward variant must be 0 (scalar) or 1 (packed pairs), got %d",
                   variant);
    g_bwd_variant.store(variant);
    return US3D_OK;
}

extern "C" int us3d_ug_get_backward_variant(int32_t* variant) {
    US3D_CHECK_ARG(variant != nullptr, "variant is NULL");
    *variant = g_bwd_variant.load();
    return US3D_OK;
}

extern "C" int us3d_ug_set_forward_variant(int32_t variant) {
    US3D_CHECK_ARG(variant == 0 || variant == 1, "forward variant must be 0 (scalar) or 1 (packed pairs), got %d",
                   variant);
    g_fwd_variant.store(variant);
    return US3D_OK;
}

extern "C" int us3d_ug_get_forward_variant(int32_t* variant) {
    US3D_CHECK_ARG(variant != nullptr, "variant is NULL");
    *variant = g_fwd_variant.load();
    return US3D_OK;
}

extern "C" size_t us3d_ug_workspace_bytes(int64_t n_gauss, int32_t n_frames, int64_t n_tiles,
                                          int64_t n_pixels, int64_t instance_capacity) {
    (void)n_frames;
    if (n_gauss < 0 || n_tiles < 0 || n_pixels < 0 || instance_capacity < 0) return 0;
    return carve(nullptr, n_gauss, n_tiles, n_pixels, instance_capacity).bytes;
}

extern "C" size_t us3d_ug_backward_scratch_bytes(int64_t instance_capacity) {
    if (instance_capacity < 0) return 0;
    return (size_t)instance_capacity * 3 * sizeof(float4);
}

static int check_common(const us3d_slice_frame* frames, int32_t n_frames, int64_t n_tiles, int64_t n_pixels,
                        int64_t n_gauss) {
    US3D_CHECK_ARG(frames != nullptr || n_frames == 0, "frames table is NULL");
    US3D_CHECK_ARG(n_frames >= 0 && n_tiles >= 0 && n_pixels >= 0 && n_gauss >= 0, "negative size");
    US3D_CHECK_ARG(n_gauss <= 0x7fffffffLL, "n_gauss must fit in int32");
    US3D_CHECK_ARG(n_pixels <= 0x7fffffffLL && n_tiles <= 0x7fffffffLL, "pixel/tile count must fit in int32");
    return US3D_OK;
}

// Reads the header of a binned workspace (synchronises the stream).
static int read_header(const void* workspace, long long hdr[H_WORDS], cudaStream_t stream) {
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    US3D_CHECK_CUDA(cudaMemcpyAsync(hdr, workspace, sizeof(long long) * H_WORDS, cudaMemcpyDeviceToHost, stream));
    US3D_CHECK_CUDA(cudaStreamSynchronize(stream));
    return US3D_OK;
}

namespace us3d {
namespace ug {

// Workspace bytes with an explicit (Gaussian, frame) task capacity (internal to the library).
size_t workspace_bytes_with_tasks(int64_t n_gauss, int64_t n_tiles, int64_t n_pixels, int64_t cap, int64_t tc) {
    if (n_gauss < 0 || n_tiles < 0 || n_pixels < 0 || cap < 0 || tc < 0) return 0;
    return carve(nullptr, n_gauss, n_tiles, n_pixels, cap, tc).bytes;
}

// Number of (Gaussian, frame) tasks the last binning of `workspace` found (synchronises).
int read_task_count(const void* workspace, int64_t* n_tasks, void* stream);

// us3d_ug_bin_ex with an explicit task capacity (tc < 0: task_capacity(cap)). The shading
// entry points take the same workspace whatever tc was.
int bin_with_task_capacity(void* workspace, size_t workspace_bytes, const us3d_slice_frame* frames, int32_t n_frames,
                           int64_t n_tiles, int64_t n_pixels, int64_t n_gauss, const float* means, const float* tril,
                           const float* opac, const float* inten, float chi2, float beta, int32_t sort_by_depth,
                           int64_t cap, int64_t task_cap, const float* pixels, int32_t flags, void* stream_);

}  // namespace ug
}  // namespace us3d

extern "C" int us3d_ug_bin_ex(void* workspace, size_t workspace_bytes, const us3d_slice_frame* frames,
                              int32_t n_frames, int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
                              const float* means, const float* tril, const float* opac, const float* inten,
                              float chi2, float beta, int32_t sort_by_depth, int64_t cap, const float* pixels,
                              int32_t flags, void* stream_) {
    return bin_with_task_capacity(workspace, workspace_bytes, frames, n_frames, n_tiles, n_pixels, n_gauss, means,
                                  tril, opac, inten, chi2, beta, sort_by_depth, cap, -1, pixels, flags, stream_);
}

int us3d::ug::read_task_count(const void* workspace, int64_t* n_tasks, void* stream) {
    long long hdr[H_WORDS];
    int st = read_header(workspace, hdr, (cudaStream_t)stream);
    if (st != US3D_OK) return st;
    *n_tasks = hdr[H_NTASK];
    return US3D_OK;
}

int us3d::ug::bin_with_task_capacity(void* workspace, size_t workspace_bytes, const us3d_slice_frame* frames,
                                     int32_t n_frames, int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
                                     const float* means, const float* tril, const float* opac, const float* inten,
                                     float chi2, float beta, int32_t sort_by_depth, int64_t cap, int64_t task_cap,
                                     const float* pixels, int32_t flags, void* stream_) {
    int st = check_common(frames, n_frames, n_tiles, n_pixels, n_gauss);
    const int slice_cull = (flags & US3D_UG_BIN_SLICE_CULL) ? 1 : 0;
    US3D_CHECK_ARG((flags & ~(US3D_UG_BIN_SLICE_CULL | US3D_UG_BIN_LOGIT_ATTRIBUTES | US3D_UG_BIN_GAUSSIAN_SETS)) == 0,
                   "unknown binning flags 0x%x", (unsigned)flags);
    const int sets = (flags & US3D_UG_BIN_GAUSSIAN_SETS) ? 1 : 0;
    US3D_CHECK_ARG(!slice_cull || n_pixels == 0 || pixels != nullptr, "slice cull needs the pixel positions");
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    US3D_CHECK_ARG(n_gauss == 0 || (means && tril && opac && inten), "Gaussian parameter pointer is NULL");
    US3D_CHECK_ARG((reinterpret_cast<uintptr_t>(tril) & 7) == 0, "precision_tril must be 8-byte aligned");
    US3D_CHECK_ARG(chi2 > 0.f && beta > 0.f, "chi2_threshold and diag_beta must be > 0");
    US3D_CHECK_ARG(task_cap <= 0x7fffffffLL, "task capacity must be below 2^31");
    const int64_t tc = task_cap < 0 ? task_capacity(cap) : task_cap;
    const Workspace w = carve(workspace, n_gauss, n_tiles, n_pixels, cap, tc);
    US3D_CHECK_ARG(workspace_bytes >= w.bytes, "workspace too small: %zu < %zu bytes", workspace_bytes, w.bytes);
    cudaStream_t stream = (cudaStream_t)stream_;

    const int prof = prof_begin("ug_bin", stream);
    init_tiles_kernel<<<(unsigned)((n_tiles + 255) / 256 > 0 ? (n_tiles + 255) / 256 : 1), 256, 0, stream>>>(
        n_tiles, w.tile_count, w.tile_cursor, w.tile_frame, w.frame_dev, w.header, cap, n_gauss, n_pixels, slice_cull);
    if (n_frames > 0)
        setup_kernel<<<n_frames, 256, 0, stream>>>(frames, n_frames, n_tiles, n_pixels, w.tile_frame, w.header);
    US3D_CHECK_LAUNCH("ug setup");
    if (slice_cull && n_tiles > 0)
        tile_dev_kernel<<<(unsigned)n_tiles, TILE_PIX, 0, stream>>>(n_tiles, n_pixels, frames, w.tile_frame, pixels,
                                                                    w.tile_dev, w.frame_dev);
    const unsigned* tdev = slice_cull ? w.frame_dev : nullptr;
    const int gb = (int)((n_gauss + 255) / 256);
    const unsigned tb = (unsigned)std::min<int64_t>((tc + 127) / 128, 148 * 16);
    if (n_gauss > 0) {
        pack_kernel<<<gb, 256, 0, stream>>>(n_gauss, means, tril, opac, inten,
                                            (flags & US3D_UG_BIN_LOGIT_ATTRIBUTES) ? 1 : 0, w.pack);
        cull_kernel<<<gb, 256, 0, stream>>>(n_gauss, n_tiles, n_pixels, frames, n_frames, sets, w.pack, chi2, beta, nullptr,
                                            tc, w.gtasks, w.task_rect, w.task_gf, w.task_v);
        US3D_CHECK_LAUNCH("ug cull");
    }
    US3D_CHECK_CUDA(exclusive_scan(w.gtasks, n_gauss, w.task_offset, w.bs_g, w.header + H_NTASK, stream));
    task_check_kernel<<<1, 1, 0, stream>>>(w.header, tc);
    US3D_CHECK_CUDA(cudaMemsetAsync(w.task_ntiles, 0, sizeof(int) * (size_t)tc, stream));
    if (n_gauss > 0) {
        cull_kernel<<<gb, 256, 0, stream>>>(n_gauss, n_tiles, n_pixels, frames, n_frames, sets, w.pack, chi2, beta,
                                            w.task_offset, tc, w.gtasks, w.task_rect, w.task_gf, w.task_v);
        task_count_kernel<<<tb, 128, 0, stream>>>(w.header, frames, w.pack, chi2, beta, tdev, w.task_rect, w.task_gf,
                                                  w.task_ntiles, w.tile_count);
        US3D_CHECK_LAUNCH("ug task count");
    }
    US3D_CHECK_CUDA(exclusive_scan(w.task_ntiles, tc, w.task_inst, w.bs_k, w.header + H_SCAN_G, stream));
    inst_offset_kernel<<<(unsigned)((n_gauss + 256) / 256), 256, 0, stream>>>(n_gauss, w.task_offset, w.task_inst,
                                                                             w.header, w.inst_offset);
    US3D_CHECK_CUDA(exclusive_scan(w.tile_count, n_tiles, w.tile_start, w.bs_t, w.header + H_SCAN_T, stream));
    check_kernel<<<1, 1, 0, stream>>>(w.header, cap);
    if (n_gauss > 0) {
        task_scatter_kernel<<<tb, 128, 0, stream>>>(w.header, frames, w.pack, chi2, beta, sort_by_depth, tdev,
                                                    w.task_rect, w.task_gf, w.task_v, w.task_inst, w.tile_start,
                                                    w.tile_cursor, w.keys, w.slot_inst, w.slot_mask);
        US3D_CHECK_LAUNCH("ug scatter");
    }
    if (n_tiles > 0)
        verify_kernel<<<(unsigned)((n_tiles + 255) / 256), 256, 0, stream>>>(n_tiles, w.tile_count, w.tile_cursor,
                                                                              w.header);
    if (n_tiles > 0) {
        US3D_CHECK_CUDA(launch_tile_sort(n_tiles, n_gauss, w.tile_start, w.header, w.keys, w.slot_inst, w.sorted_gid,
                                         w.sorted_inst, g_sort_attr_done, stream, w.slot_mask, w.sorted_mask));
    }
    prof_end(prof, stream);
    count_launches(1 + (n_frames > 0) + (slice_cull && n_tiles > 0) + 4 * (n_gauss > 0) + 9 + 3 + (n_gauss > 0) +
                   (1 + tile_sort_launches(n_gauss)) * (n_tiles > 0));
    return US3D_OK;
}

extern "C" int us3d_ug_bin(void* workspace, size_t workspace_bytes, const us3d_slice_frame* frames,
                           int32_t n_frames, int64_t n_tiles, int64_t n_pixels, int64_t n_gauss,
                           const float* means, const float* tril, const float* opac, const float* inten,
                           float chi2, float beta, int32_t sort_by_depth, int64_t cap, void* stream) {
    return us3d_ug_bin_ex(workspace, workspace_bytes, frames, n_frames, n_tiles, n_pixels, n_gauss, means, tril, opac,
                          inten, chi2, beta, sort_by_depth, cap, nullptr, 0, stream);
}

extern "C" int us3d_ug_read_status(const void* workspace, int64_t* total, int32_t* overflow, void* stream_) {
    long long hdr[H_WORDS];
    int st = read_header(workspace, hdr, (cudaStream_t)stream_);
    if (st != US3D_OK) return st;
    if (total) *total = hdr[H_TOTAL];
    if (overflow) *overflow = (int32_t)hdr[H_FLAGS];
    return US3D_OK;
}

extern "C" int us3d_ug_forward(void* workspace, const us3d_slice_frame* frames, int32_t n_frames, int64_t n_tiles,
                               int64_t n_pixels, int64_t n_gauss, int64_t cap, const float* pixels, float chi2,
                               float beta, float bg_alpha, float bg_intensity, float* out_image, float* out_alpha,
                               float* out_depth, int32_t* out_counts, void* stream_) {
    int st = check_common(frames, n_frames, n_tiles, n_pixels, n_gauss);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    US3D_CHECK_ARG(n_pixels == 0 || (pixels && out_image && out_alpha && out_depth), "output pointer is NULL");
    const Workspace w = carve(workspace, n_gauss, n_tiles, n_pixels, cap);
    if (n_tiles == 0) return US3D_OK;
    cudaStream_t stream = (cudaStream_t)stream_;
    const int prof = prof_begin("ug_forward", stream);
    auto launch = [&](auto kernel) {
        kernel<<<(unsigned)n_tiles, TILE_PIX, 0, stream>>>(
            n_tiles, n_pixels, frames, w.tile_frame, w.tile_start, w.sorted_gid, w.sorted_mask, w.header, w.pack,
            pixels, chi2, beta, bg_alpha, bg_intensity, out_image, out_alpha, out_depth, w.pixel_aux);
    };
    auto launch_packed = [&](auto kernel) {
        kernel<<<(unsigned)n_tiles, 128, 0, stream>>>(
            n_tiles, n_pixels, frames, w.tile_frame, w.tile_start, w.sorted_gid, w.sorted_mask, w.header, w.pack,
            pixels, chi2, beta, bg_alpha, bg_intensity, out_image, out_alpha, out_depth, w.pixel_aux);
    };
    if (!window_implied(beta)) {
        launch(forward_kernel<256, true>);
    } else if (g_fwd_variant.load() == 1) {
        // at most 256 staged Gaussians (96 bytes each) fit the static shared memory
        if (g_fwd_batch.load() == 128)
            launch_packed(forward_packed_kernel<128>);
        else
            launch_packed(forward_packed_kernel<256>);
    } else {
        switch (g_fwd_batch.load()) {
            case 128: launch(forward_kernel<128, false>); break;
            case 256: launch(forward_kernel<256, false>); break;
            default: launch(forward_kernel<512, false>); break;
        }
    }
    US3D_CHECK_LAUNCH("ug forward");
    if (out_counts) {  // the reference's per-pixel candidate counts (full binning only)
        pixel_csr_kernel<true><<<(unsigned)n_tiles, TILE_PIX, 0, stream>>>(
            n_tiles, n_pixels, frames, w.tile_frame, w.tile_start, w.sorted_gid, w.header, w.pack, pixels, chi2, beta,
            nullptr, nullptr, out_counts);
        US3D_CHECK_LAUNCH("ug counts");
    }
    prof_end(prof, stream);
    count_launches(1 + (out_counts != nullptr));
    return US3D_OK;
}

static int ug_backward_impl(void* workspace, const us3d_slice_frame* frames, int32_t n_frames, int64_t n_tiles,
                            int64_t n_pixels, int64_t n_gauss, int64_t cap, const float* pixels,
                            const float* d_image, const float* d_alpha, const float* d_depth,
                            const float* loss_image, const float* loss_target, const float4* loss_coef,
                            const float* saved_alpha, float chi2, float beta, float bg_alpha, float bg_intensity,
                            void* scratch, size_t scratch_bytes, float* d_means, float* d_tril, float* d_opac,
                            float* d_inten, cudaStream_t stream) {
    const bool fused = loss_coef != nullptr;
    int st = check_common(frames, n_frames, n_tiles, n_pixels, n_gauss);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    US3D_CHECK_ARG(scratch != nullptr || cap == 0, "backward scratch is NULL");
    US3D_CHECK_ARG(scratch_bytes >= us3d_ug_backward_scratch_bytes(cap), "backward scratch too small: %zu < %zu",
                   scratch_bytes, us3d_ug_backward_scratch_bytes(cap));
    US3D_CHECK_ARG(n_gauss == 0 || (d_means && d_tril && d_opac && d_inten), "gradient pointer is NULL");
    if (fused)
        US3D_CHECK_ARG(n_pixels == 0 || (pixels && loss_image && loss_target && saved_alpha), "input pointer is NULL");
    else
        US3D_CHECK_ARG(n_pixels == 0 || (pixels && d_image && d_alpha && d_depth && saved_alpha),
                       "input pointer is NULL");
    const Workspace w = carve(workspace, n_gauss, n_tiles, n_pixels, cap);
    float4* partial = reinterpret_cast<float4*>(scratch);
    const int prof = prof_begin("ug_backward", stream);
    if (n_tiles > 0) {
        const int threads = g_bwd_threads.load();
        auto launch = [&](auto kernel, int nthreads) {
            kernel<<<(unsigned)n_tiles, nthreads, 0, stream>>>(
                n_tiles, n_pixels, frames, w.tile_frame, w.tile_start, w.sorted_gid, w.sorted_inst, w.sorted_mask,
                w.header, w.pack, pixels, d_image, d_alpha, d_depth, saved_alpha, w.pixel_aux, chi2, beta, bg_alpha,
                bg_intensity, loss_image, loss_target, loss_coef, partial);
        };
        const bool packed = g_bwd_variant.load() == 1;
        if (!window_implied(beta))
            fused ? launch(backward_kernel<true, 256, true>, 256) : launch(backward_kernel<false, 256, true>, 256);
        else if (packed && fused)
            threads == 128 ? launch(backward_packed_kernel<true, 128>, 128)
                           : launch(backward_packed_kernel<true, 256>, 256);
        else if (packed)
            threads == 128 ? launch(backward_packed_kernel<false, 128>, 128)
                           : launch(backward_packed_kernel<false, 256>, 256);
        else if (fused)
            threads == 128 ? launch(backward_kernel<true, 128, false>, 128)
                           : launch(backward_kernel<true, 256, false>, 256);
        else
            threads == 128 ? launch(backward_kernel<false, 128, false>, 128)
                           : launch(backward_kernel<false, 256, false>, 256);
        US3D_CHECK_LAUNCH("ug backward");
    }
    if (n_gauss > 0) {
        reduce_kernel<<<(unsigned)((n_gauss * REDUCE_COLS + REDUCE_THREADS - 1) / REDUCE_THREADS), REDUCE_THREADS, 0,
                        stream>>>(n_gauss, w.inst_offset, w.header, partial, d_means, d_tril, d_opac, d_inten);
        US3D_CHECK_LAUNCH("ug reduce");
    }
    prof_end(prof, stream);
    count_launches((n_tiles > 0) + (n_gauss > 0));
    return US3D_OK;
}

extern "C" int us3d_ug_backward(void* workspace, const us3d_slice_frame* frames, int32_t n_frames, int64_t n_tiles,
                                int64_t n_pixels, int64_t n_gauss, int64_t cap, const float* pixels,
                                const float* d_image, const float* d_alpha, const float* d_depth,
                                const float* saved_alpha, float chi2, float beta, float bg_alpha,
                                float bg_intensity, void* scratch, size_t scratch_bytes, float* d_means,
                                float* d_tril, float* d_opac, float* d_inten, void* stream_) {
    return ug_backward_impl(workspace, frames, n_frames, n_tiles, n_pixels, n_gauss, cap, pixels, d_image, d_alpha,
                            d_depth, nullptr, nullptr, nullptr, saved_alpha, chi2, beta, bg_alpha, bg_intensity,
                            scratch, scratch_bytes, d_means, d_tril, d_opac, d_inten, (cudaStream_t)stream_);
}

extern "C" int us3d_ug_backward_loss(void* workspace, const us3d_slice_frame* frames, int32_t n_frames,
                                     int64_t n_tiles, int64_t n_pixels, int64_t n_gauss, int64_t cap,
                                     const float* pixels, const float* image, const float* target,
                                     const float* loss_coef, const float* saved_alpha, float chi2, float beta,
                                     float bg_alpha, float bg_intensity, void* scratch, size_t scratch_bytes,
                                     float* d_means, float* d_tril, float* d_opac, float* d_inten, void* stream_) {
    US3D_CHECK_ARG(loss_coef != nullptr || n_frames == 0, "loss coefficients are NULL");
    US3D_CHECK_ARG((reinterpret_cast<uintptr_t>(loss_coef) & 15) == 0, "loss coefficients must be 16-byte aligned");
    return ug_backward_impl(workspace, frames, n_frames, n_tiles, n_pixels, n_gauss, cap, pixels, nullptr, nullptr,
                            nullptr, image, target, reinterpret_cast<const float4*>(loss_coef), saved_alpha, chi2,
                            beta, bg_alpha, bg_intensity, scratch, scratch_bytes, d_means, d_tril, d_opac, d_inten,
                            (cudaStream_t)stream_);
}

extern "C" int us3d_ug_pixel_csr(void* workspace, const us3d_slice_frame* frames, int32_t n_frames, int64_t n_tiles,
                                 int64_t n_pixels, int64_t n_gauss, int64_t cap, const float* pixels, float chi2,
                                 float beta, const int32_t* offsets, int32_t* out_indices, void* stream_) {
    int st = check_common(frames, n_frames, n_tiles, n_pixels, n_gauss);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    US3D_CHECK_ARG(n_pixels == 0 || (pixels && offsets), "input pointer is NULL");
    const Workspace w = carve(workspace, n_gauss, n_tiles, n_pixels, cap);
    if (n_tiles == 0) return US3D_OK;
    cudaStream_t stream = (cudaStream_t)stream_;
    pixel_csr_kernel<false><<<(unsigned)n_tiles, TILE_PIX, 0, stream>>>(n_tiles, n_pixels, frames, w.tile_frame,
                                                                         w.tile_start, w.sorted_gid, w.header, w.pack,
                                                                         pixels, chi2, beta, offsets, out_indices,
                                                                         nullptr);
    US3D_CHECK_LAUNCH("ug pixel csr");
    count_launches(1);
    return US3D_OK;
}

extern "C" int us3d_ug_export_bins(const void* workspace, int64_t n_tiles, int32_t frame_tile_offset,
                                   int32_t frame_n_tiles, int64_t* out_keys, int32_t* out_values,
                                   int32_t* out_range_start, int32_t* out_range_end, void* stream_) {
    cudaStream_t stream = (cudaStream_t)stream_;
    long long hdr[H_WORDS];
    int st = read_header(workspace, hdr, stream);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(hdr[H_T] == n_tiles, "n_tiles does not match the binned workspace");
    US3D_CHECK_ARG(frame_tile_offset >= 0 && frame_n_tiles >= 0 && frame_tile_offset + (int64_t)frame_n_tiles <= n_tiles,
                   "frame tile range out of bounds");
    if (hdr[H_FLAGS] != 0) {
        us3d::set_error("workspace binning overflowed (flags=%lld)", hdr[H_FLAGS]);
        return US3D_CAPACITY_OVERFLOW;
    }
    const Workspace w = carve(const_cast<void*>(workspace), hdr[H_G], hdr[H_T], hdr[H_P], hdr[H_CAP]);
    if (frame_n_tiles == 0) return US3D_OK;
    export_kernel<<<frame_n_tiles, 256, 0, stream>>>(frame_tile_offset, frame_n_tiles, w.tile_start, w.keys,
                                                     w.sorted_gid, out_keys, out_values, out_range_start,
                                                     out_range_end);
    US3D_CHECK_LAUNCH("ug export");
    count_launches(1);
    return US3D_OK;
}

extern "C" int us3d_ug_frame_instances(const void* workspace, int64_t n_tiles, int32_t frame_tile_offset,
                                       int32_t frame_n_tiles, int64_t* first, int64_t* count, void* stream_) {
    cudaStream_t stream = (cudaStream_t)stream_;
    long long hdr[H_WORDS];
    int st = read_header(workspace, hdr, stream);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(hdr[H_T] == n_tiles, "n_tiles does not match the binned workspace");
    US3D_CHECK_ARG(frame_tile_offset >= 0 && frame_n_tiles >= 0 && frame_tile_offset + (int64_t)frame_n_tiles <= n_tiles,
                   "frame tile range out of bounds");
    const Workspace w = carve(const_cast<void*>(workspace), hdr[H_G], hdr[H_T], hdr[H_P], hdr[H_CAP]);
    int se[2];
    US3D_CHECK_CUDA(cudaMemcpyAsync(&se[0], w.tile_start + frame_tile_offset, sizeof(int), cudaMemcpyDeviceToHost, stream));
    US3D_CHECK_CUDA(cudaMemcpyAsync(&se[1], w.tile_start + frame_tile_offset + frame_n_tiles, sizeof(int),
                                    cudaMemcpyDeviceToHost, stream));
    US3D_CHECK_CUDA(cudaStreamSynchronize(stream));
    if (first) *first = se[0];
    if (count) *count = se[1] - se[0];
    return US3D_OK;
}
