// slice-adapted 3DGS: bounded additive splatting of projected 2D Gaussians (RGB + alpha).
//
// Reference behaviour restated here (paths inside KevinWCCC/ultrasound-3d-reconstruction,
// ops/slice_adapted_3dgs_renderer/src/render.cu):
//   :158-198   pixel <-> slice-plane mm mapping, per-Gaussian pixel bounding box
//   :199-259   per-pair weight: q <= r^2, power = -q/2 clamped to [-50, 0], w = e^power * weight
//   :261-352   16x16 tile rectangles, keys (tile << 32), ranges
//   :354-515   per-pixel forward over the tile list, per-pair backward
//
// B200 design: the reference switches between per-Gaussian atomic scatter (fewer than
// 16384 Gaussians) and tile binning; here every size is tile-binned through the shared
// bucket + per-tile sort, the forward stages each tile's Gaussians in shared memory (one
// pixel per thread, tile-list order = Gaussian order), and the backward gives each thread
// one (tile, Gaussian) instance whose bounding box it sweeps inside the tile, accumulating
// the ten parameter gradients in registers; per-instance partials are reduced per Gaussian
// in a fixed order (the reference issues up to 10 float atomics per pair).
#include "us3d_common.cuh"
#include "scan.cuh"
#include "binning.cuh"

namespace us3d {
namespace sa {

constexpr int TILE = 16;  // reference SLICE_3DGS_TILE_SIZE (render.cu:14)
constexpr int FWD_BATCH = 256;
constexpr int PARTIAL_F4 = 3;  // 12 floats per instance
constexpr int BWD_CHUNK = 1024;  // instances a backward block orders by box area at a time
constexpr int AREA_BINS = 32;    // area classes of 8 pixels (a box inside one tile covers 1..256)

struct Workspace {
    long long* header;
    int4* rects;       // N tile rectangles
    int4* bbox;        // N pixel bounding boxes (xmin, ymin, xmax, ymax), inclusive
    int* touched;      // N
    int* inst_offset;  // N + 1
    long long* bs_g;
    int* tile_count;
    int* tile_start;
    int* tile_cursor;
    long long* bs_t;
    unsigned long long* keys;
    int* slot_inst;
    int* sorted_gid;
    int* sorted_inst;
    float4* fwd_part;  // list-range sums of the forward when it splits tiles (frame_split(T) x T x 256)
    size_t bytes;
};

// Blocks that share one tile in the splat kernels: frames with fewer tiles than four per SM split
// each tile four ways (a 256x256 slice has 256 tiles, under two blocks per SM).
static inline int frame_split(int64_t T) { return T < 4 * 148 ? 4 : 1; }

static Workspace carve(void* base, int64_t N, int64_t T, int64_t cap) {
    Carver c(base);
    Workspace w;
    w.header = c.take<long long>(H_WORDS);
    w.rects = c.take<int4>((size_t)N);
    w.bbox = c.take<int4>((size_t)N);
    w.touched = c.take<int>((size_t)N);
    w.inst_offset = c.take<int>((size_t)N + 1);
    w.bs_g = c.take<long long>((size_t)scan_num_blocks(N) + 1);
    w.tile_count = c.take<int>((size_t)T);
    w.tile_start = c.take<int>((size_t)T + 1);
    w.tile_cursor = c.take<int>((size_t)T);
    w.bs_t = c.take<long long>((size_t)scan_num_blocks(T) + 1);
    w.keys = c.take<unsigned long long>((size_t)cap);
    w.slot_inst = c.take<int>((size_t)cap);
    w.sorted_gid = c.take<int>((size_t)cap);
    w.sorted_inst = c.take<int>((size_t)cap);
    w.fwd_part = c.take<float4>(frame_split(T) > 1 ? (size_t)frame_split(T) * T * TILE * TILE : 0);
    w.bytes = align_up(c.off, 256);
    return w;
}

// Pixel centre in slice-plane mm: -h + 2h * i / (n - 1) (reference render.cu:158-170).
__device__ __forceinline__ float plane_x(int x, int W, float hw) {
    return (W <= 1) ? 0.0f : -hw + (2.0f * hw) * float(x) / float(W - 1);
}
__device__ __forceinline__ float plane_y(int y, int H, float hh) {
    return (H <= 1) ? 0.0f : -hh + (2.0f * hh) * float(y) / float(H - 1);
}

// Pixel bounding box of the radius_sigma ellipse (reference render.cu:172-198).
__device__ __forceinline__ void pixel_bbox(const float4 inv, float mx, float my, int H, int W, float hw, float hh,
                                           float rs, int& xmin, int& xmax, int& ymin, int& ymax) {
    float det = inv.x * inv.w - inv.y * inv.z;
    det = fmaxf(det, 1.0e-8f);
    const float sigx = sqrtf(fmaxf(inv.w / det, 1.0e-8f));
    const float sigy = sqrtf(fmaxf(inv.x / det, 1.0e-8f));
    const float rx = rs * sigx, ry = rs * sigy;
    const float sx = (W > 1) ? float(W - 1) / (2.0f * hw) : 0.0f;
    const float sy = (H > 1) ? float(H - 1) / (2.0f * hh) : 0.0f;
    xmin = max(0, int(floorf((mx - rx + hw) * sx)));
    xmax = min(W - 1, int(ceilf((mx + rx + hw) * sx)));
    ymin = max(0, int(floorf((my - ry + hh) * sy)));
    ymax = min(H - 1, int(ceilf((my + ry + hh) * sy)));
}

__global__ void init_kernel(int64_t T, int* __restrict__ tile_count, int* __restrict__ tile_cursor,
                            long long* __restrict__ header, int64_t cap, int64_t N) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (blockIdx.x == 0 && threadIdx.x < H_WORDS) {
        long long v = 0;
        if (threadIdx.x == H_CAP) v = cap;
        if (threadIdx.x == H_G) v = N;
        if (threadIdx.x == H_T) v = T;
        header[threadIdx.x] = v;
    }
    if (t >= T) return;
    tile_count[t] = 0;
    tile_cursor[t] = 0;
}

__global__ void __launch_bounds__(256)
preprocess_kernel(int64_t N, int H, int W, int gw, int gh, float hw, float hh, float rs,
                  const float2* __restrict__ means, const float4* __restrict__ invs, int4* __restrict__ rects,
                  int4* __restrict__ bbox, int* __restrict__ touched, int* __restrict__ tile_count) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= N) return;
    const float2 m = means[g];
    int xmin, xmax, ymin, ymax;
    pixel_bbox(invs[g], m.x, m.y, H, W, hw, hh, rs, xmin, xmax, ymin, ymax);
    rects[g] = make_int4(0, 0, 0, 0);
    bbox[g] = make_int4(xmin, ymin, xmax, ymax);
    touched[g] = 0;
    if (xmax < xmin || ymax < ymin) return;
    const int x0 = max(0, xmin / TILE), y0 = max(0, ymin / TILE);
    const int x1 = min(gw, xmax / TILE + 1), y1 = min(gh, ymax / TILE + 1);
    if (x0 >= x1 || y0 >= y1) return;
    rects[g] = make_int4(x0, y0, x1, y1);
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


// One block of 16x16 threads per tile and list range, staged Gaussians, per-pixel sums in
// tile-list order (reference render.cu:354-426). With split > 1 the tile's list is cut into
// `split` contiguous ranges, block (tile, part) sums range `part` into part_out, and
// combine_kernel adds the ranges in order.
__global__ void __launch_bounds__(TILE * TILE)
forward_kernel(int split, int H, int W, int gw, float hw, float hh, float rs, const float2* __restrict__ means,
               const float4* __restrict__ invs, const float* __restrict__ weights, const float* __restrict__ colors,
               const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
               const long long* __restrict__ header, float* __restrict__ image, float* __restrict__ alpha,
               float4* __restrict__ part_out) {
    __shared__ float4 s_inv[FWD_BATCH];
    __shared__ float4 s_mw[FWD_BATCH];   // mx, my, weight, c0
    __shared__ float2 s_c12[FWD_BATCH];  // c1, c2
    if (header[H_FLAGS] != 0) return;
    const int t = blockIdx.x / split, part = blockIdx.x % split;
    const int x = (t % gw) * TILE + (threadIdx.x % TILE);
    const int y = (t / gw) * TILE + (threadIdx.x / TILE);
    const bool valid = x < W && y < H;
    const float px = plane_x(x, W, hw), py = plane_y(y, H, hh);
    const float r2 = rs * rs;
    const int l0 = tile_start[t], ln = tile_start[t + 1] - l0;
    const int lo = (int)((int64_t)ln * part / split), hi = (int)((int64_t)ln * (part + 1) / split);
    const int s0 = l0 + lo, n = hi - lo;
    float o0 = 0.f, o1 = 0.f, o2 = 0.f, ao = 0.f;
    for (int b0 = 0; b0 < n; b0 += FWD_BATCH) {
        const int nb = min(FWD_BATCH, n - b0);
        __syncthreads();
        for (int j = threadIdx.x; j < nb; j += blockDim.x) {
            const int g = sorted_gid[s0 + b0 + j];
            const float2 m = means[g];
            s_inv[j] = invs[g];
            s_mw[j] = make_float4(m.x, m.y, weights[g], colors[3 * g]);
            s_c12[j] = make_float2(colors[3 * g + 1], colors[3 * g + 2]);
        }
        __syncthreads();
        if (valid) {
            for (int j = 0; j < nb; ++j) {
                const float4 mw = s_mw[j];
                const float4 inv = s_inv[j];
                const float dx = px - mw.x, dy = py - mw.y;
                const float qx = inv.x * dx + inv.y * dy;
                const float qy = inv.z * dx + inv.w * dy;
                const float quad = dx * qx + dy * qy;
                if (quad > r2) continue;
                float power = -0.5f * quad;
                if (power < -50.0f) continue;
                if (power > 0.0f) power = 0.0f;
                const float w = __expf(power) * mw.z;
                const float2 c12 = s_c12[j];
                o0 += w * mw.w;
                o1 += w * c12.x;
                o2 += w * c12.y;
                ao += w;
            }
        }
    }
    if (split > 1) {
        part_out[((int64_t)part * (gridDim.x / split) + t) * (TILE * TILE) + threadIdx.x] = make_float4(o0, o1, o2, ao);
        return;
    }
    if (!valid) return;
    const int64_t p = (int64_t)y * W + x;
    image[3 * p + 0] = o0;
    image[3 * p + 1] = o1;
    image[3 * p + 2] = o2;
    alpha[p] = ao;
}

// Sum of a pixel's list-range sums, in range order (thread per pixel of the tile grid).
__global__ void __launch_bounds__(256)
combine_kernel(int split, int T, int H, int W, int gw, const long long* __restrict__ header,
               const float4* __restrict__ part_in, float* __restrict__ image, float* __restrict__ alpha) {
    if (header[H_FLAGS] != 0) return;
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // tile * 256 + pixel in tile
    if (i >= (int64_t)T * TILE * TILE) return;
    const int t = (int)(i / (TILE * TILE)), l = (int)(i % (TILE * TILE));
    const int x = (t % gw) * TILE + (l % TILE), y = (t / gw) * TILE + (l / TILE);
    if (x >= W || y >= H) return;
    float4 a = part_in[i];
    for (int k = 1; k < split; ++k) {
        const float4 b = part_in[(int64_t)k * T * TILE * TILE + i];
        a.x += b.x;
        a.y += b.y;
        a.z += b.z;
        a.w += b.w;
    }
    const int64_t p = (int64_t)y * W + x;
    image[3 * p + 0] = a.x;
    image[3 * p + 1] = a.y;
    image[3 * p + 2] = a.z;
    alpha[p] = a.w;
}

// One block per tile, or `split` blocks per tile that share its instances (frames with few
// tiles: a 256x256 slice has 256, under two blocks per SM); a thread owns one instance at a time
// and sweeps the part of its pixel bounding box inside the tile (reference render.cu:428-515 and
// :517-600 for the per-pair terms), so the partials do not depend on the split.
__global__ void __launch_bounds__(256)
backward_kernel(int split, int H, int W, int gw, float hw, float hh, float rs, const float2* __restrict__ means,
                const float4* __restrict__ invs, const float* __restrict__ weights, const float* __restrict__ colors,
                const float* __restrict__ grad_image, const float* __restrict__ grad_alpha,
                const int4* __restrict__ bbox, const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
                const int* __restrict__ sorted_inst, const long long* __restrict__ header,
                float4* __restrict__ partial) {
    __shared__ float4 s_go[TILE * TILE];  // grad_image rgb, grad_alpha
    __shared__ int s_key[BWD_CHUNK];      // area class << 16 | rank within the class
    __shared__ int s_ord[BWD_CHUNK];      // chunk positions ordered by area class
    __shared__ int s_bin[AREA_BINS];
    if (header[H_FLAGS] != 0) return;
    const int t = blockIdx.x / split, part = blockIdx.x % split;
    const int s0 = tile_start[t], n = tile_start[t + 1] - s0;
    const int cs = min(BWD_CHUNK, (n + split - 1) / split);  // chunk: the split shares a tile evenly
    if (n <= part * cs) return;
    const int tx0 = (t % gw) * TILE, ty0 = (t / gw) * TILE;
    {
        const int x = tx0 + (threadIdx.x % TILE), y = ty0 + (threadIdx.x / TILE);
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (threadIdx.x < TILE * TILE && x < W && y < H) {
            const int64_t p = (int64_t)y * W + x;
            v = make_float4(grad_image[3 * p], grad_image[3 * p + 1], grad_image[3 * p + 2], grad_alpha[p]);
        }
        if (threadIdx.x < TILE * TILE) s_go[threadIdx.x] = v;
    }
    __syncthreads();
    const float r2 = rs * rs;
    const int xe = min(tx0 + TILE - 1, W - 1), ye = min(ty0 + TILE - 1, H - 1);
    // The tile's instances go out in chunks; inside a chunk, positions are handed to threads in
    // order of the box-in-tile area (a counting sort on area classes), so that the 32 lanes of a
    // warp sweep similar pixel counts. Which thread computes an instance does not change its sums.
    for (int q0 = part * cs; q0 < n; q0 += split * cs) {
        const int nc = min(cs, n - q0);
        __syncthreads();  // the previous chunk's s_ord is read to the end
        if (threadIdx.x < AREA_BINS) s_bin[threadIdx.x] = 0;
        __syncthreads();
        for (int j = threadIdx.x; j < nc; j += blockDim.x) {
            const int4 bb = bbox[sorted_gid[s0 + q0 + j]];
            const int area = max(0, min(bb.z, xe) - max(bb.x, tx0) + 1) * max(0, min(bb.w, ye) - max(bb.y, ty0) + 1);
            const int bin = min(AREA_BINS - 1, max(area - 1, 0) >> 3);
            s_key[j] = (bin << 16) | atomicAdd(&s_bin[bin], 1);
        }
        __syncthreads();
        if (threadIdx.x < 32) {  // exclusive scan of the class counts in one warp
            const int v = s_bin[threadIdx.x];
            int incl = v;
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, incl, o);
                if ((int)threadIdx.x >= o) incl += u;
            }
            s_bin[threadIdx.x] = incl - v;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < nc; j += blockDim.x) {
            const int key = s_key[j];
            s_ord[s_bin[key >> 16] + (key & 0xffff)] = j;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nc; i += blockDim.x) {
            const int k = q0 + s_ord[i];
            const int g = sorted_gid[s0 + k];
            const int4 bb = bbox[g];
            const int x0 = max(bb.x, tx0), x1 = min(bb.z, xe);
            const int y0 = max(bb.y, ty0), y1 = min(bb.w, ye);
            const float2 m = means[g];
            const float4 inv = invs[g];
            const float weight = weights[g];
            const float c0 = colors[3 * g], c1 = colors[3 * g + 1], c2 = colors[3 * g + 2];
            float gm0 = 0.f, gm1 = 0.f, gi0 = 0.f, gi1 = 0.f, gi2 = 0.f, gi3 = 0.f, gwt = 0.f, gc0 = 0.f, gc1 = 0.f,
                  gc2 = 0.f;
            // Row-major sweep of the box in one loop (the same pixel order as rows then columns), so
            // that lanes with equal areas but different box shapes run in step.
            const int bw = x1 - x0 + 1;
            const int cnt = (x1 >= x0 && y1 >= y0) ? bw * (y1 - y0 + 1) : 0;
            int x = x0 - 1, y = y0;
            float py = plane_y(y0, H, hh);
            for (int q = 0; q < cnt; ++q) {
                if (++x > x1) {
                    x = x0;
                    py = plane_y(++y, H, hh);
                }
                const float px = plane_x(x, W, hw);
                const float dx = px - m.x, dy = py - m.y;
                const float qx = inv.x * dx + inv.y * dy;
                const float qy = inv.z * dx + inv.w * dy;
                const float quad = dx * qx + dy * qy;
                if (quad > r2) continue;
                float power = -0.5f * quad;
                if (power < -50.0f) continue;
                if (power > 0.0f) power = 0.0f;
                const float e = __expf(power);
                const float4 go = s_go[(y - ty0) * TILE + (x - tx0)];
                const float dot = go.x * c0 + go.y * c1 + go.z * c2;
                gwt += e * (dot + go.w);
                const float ew = e * weight;
                gc0 += ew * go.x;
                gc1 += ew * go.y;
                gc2 += ew * go.z;
                const float dpow = weight * (dot + go.w) * e;
                const float cm = -0.5f * dpow;
                gi0 += cm * dx * dx;
                gi1 += cm * dx * dy;
                gi2 += cm * dy * dx;
                gi3 += cm * dy * dy;
                gm0 += 0.5f * dpow * ((inv.x + inv.x) * dx + (inv.y + inv.z) * dy);
                gm1 += 0.5f * dpow * ((inv.z + inv.y) * dx + (inv.w + inv.w) * dy);
            }
            float4* out = partial + (int64_t)PARTIAL_F4 * sorted_inst[s0 + k];
            out[0] = make_float4(gm0, gm1, gi0, gi1);
            out[1] = make_float4(gi2, gi3, gwt, gc0);
            out[2] = make_float4(gc1, gc2, 0.f, 0.f);
        }
    }
}

// Per-Gaussian gradient: the sum of its instances' 48-byte partials in instance order.
// REDUCE_COLS threads per Gaussian, thread f summing float4 column f, so that a Gaussian's
// threads read each partial together; the sums are the ones a thread summing all columns would
// form.
constexpr int REDUCE_COLS = 3;
constexpr int REDUCE_THREADS = 64 * REDUCE_COLS;  // 64 Gaussians per block
__global__ void __launch_bounds__(REDUCE_THREADS)
reduce_kernel(int64_t N, const int* __restrict__ inst_offset, const long long* __restrict__ header,
              const float4* __restrict__ partial, float* __restrict__ d_means, float* __restrict__ d_inv,
              float* __restrict__ d_w, float* __restrict__ d_c) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t g = t / REDUCE_COLS;
    const int f = (int)(t % REDUCE_COLS);
    if (g >= N) return;
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
    if (header[H_FLAGS] == 0) {
        const int i1 = inst_offset[g + 1];
        int i = inst_offset[g];
        for (; i + 4 <= i1; i += 4) {  // four instances' loads in flight, summed in order
            float4 v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) v[u] = partial[(int64_t)PARTIAL_F4 * (i + u) + f];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a.x += v[u].x; a.y += v[u].y; a.z += v[u].z; a.w += v[u].w;
            }
        }
        for (; i < i1; ++i) {
            const float4 v = partial[(int64_t)PARTIAL_F4 * i + f];
            a.x += v.x; a.y += v.y; a.z += v.z; a.w += v.w;
        }
    }
    if (f == 0) {
        d_means[2 * g] = a.x;
        d_means[2 * g + 1] = a.y;
        d_inv[4 * g] = a.z;
        d_inv[4 * g + 1] = a.w;
    } else if (f == 1) {
        d_inv[4 * g + 2] = a.x;
        d_inv[4 * g + 3] = a.y;
        d_w[g] = a.z;
        d_c[3 * g] = a.w;
    } else {
        d_c[3 * g + 1] = a.x;
        d_c[3 * g + 2] = a.y;
    }
}

__global__ void export_kernel(int T, const int* __restrict__ tile_start, const int* __restrict__ sorted_gid,
                              int* __restrict__ out_ids, int* __restrict__ rs, int* __restrict__ re) {
    const int t = blockIdx.x;
    if (t >= T) return;
    const int s0 = tile_start[t], s1 = tile_start[t + 1];
    if (threadIdx.x == 0) {
        rs[t] = (s1 > s0) ? s0 : -1;
        re[t] = (s1 > s0) ? s1 : -1;
    }
    for (int s = s0 + threadIdx.x; s < s1; s += blockDim.x) out_ids[s] = sorted_gid[s];
}

// Dense splat over arbitrary pixel coordinates (the package's unbounded additive_splat;
// reference render.cu:41-153): every pixel sums all Gaussians with power >= -50.
__global__ void __launch_bounds__(256)
dense_forward_kernel(int64_t P, int64_t N, const float2* __restrict__ pixels, const float2* __restrict__ means,
                     const float4* __restrict__ invs, const float* __restrict__ weights,
                     const float* __restrict__ colors, float* __restrict__ image, float* __restrict__ alpha) {
    __shared__ float4 s_inv[256];
    __shared__ float4 s_mw[256];
    __shared__ float2 s_c12[256];
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = p < P;
    const float2 px = valid ? pixels[p] : make_float2(0.f, 0.f);
    float o0 = 0.f, o1 = 0.f, o2 = 0.f, ao = 0.f;
    for (int64_t b0 = 0; b0 < N; b0 += 256) {
        const int nb = (int)min((int64_t)256, N - b0);
        __syncthreads();
        if (threadIdx.x < nb) {
            const int64_t g = b0 + threadIdx.x;
            s_inv[threadIdx.x] = invs[g];
            s_mw[threadIdx.x] = make_float4(means[g].x, means[g].y, weights[g], colors[3 * g]);
            s_c12[threadIdx.x] = make_float2(colors[3 * g + 1], colors[3 * g + 2]);
        }
        __syncthreads();
        if (!valid) continue;
        for (int j = 0; j < nb; ++j) {
            const float4 mw = s_mw[j], inv = s_inv[j];
            const float dx = px.x - mw.x, dy = px.y - mw.y;
            const float qx = inv.x * dx + inv.y * dy;
            const float qy = inv.z * dx + inv.w * dy;
            float power = -0.5f * (dx * qx + dy * qy);
            if (power < -50.0f) continue;
            if (power > 0.0f) power = 0.0f;
            const float w = __expf(power) * mw.z;
            const float2 c12 = s_c12[j];
            o0 += w * mw.w;
            o1 += w * c12.x;
            o2 += w * c12.y;
            ao += w;
        }
    }
    if (!valid) return;
    image[3 * p] = o0;
    image[3 * p + 1] = o1;
    image[3 * p + 2] = o2;
    alpha[p] = ao;
}

// Backward of the dense splat: one thread per Gaussian over all pixels (no atomics).
__global__ void __launch_bounds__(128)
dense_backward_kernel(int64_t P, int64_t N, const float2* __restrict__ pixels, const float2* __restrict__ means,
                      const float4* __restrict__ invs, const float* __restrict__ weights,
                      const float* __restrict__ colors, const float* __restrict__ grad_image,
                      const float* __restrict__ grad_alpha, float* __restrict__ d_means, float* __restrict__ d_inv,
                      float* __restrict__ d_w, float* __restrict__ d_c) {
    const int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= N) return;
    const float2 m = means[g];
    const float4 inv = invs[g];
    const float weight = weights[g], c0 = colors[3 * g], c1 = colors[3 * g + 1], c2 = colors[3 * g + 2];
    float gm0 = 0.f, gm1 = 0.f, gi0 = 0.f, gi1 = 0.f, gi2 = 0.f, gi3 = 0.f, gwt = 0.f, gc0 = 0.f, gc1 = 0.f, gc2 = 0.f;
    for (int64_t p = 0; p < P; ++p) {
        const float2 px = pixels[p];
        const float dx = px.x - m.x, dy = px.y - m.y;
        const float qx = inv.x * dx + inv.y * dy, qy = inv.z * dx + inv.w * dy;
        float power = -0.5f * (dx * qx + dy * qy);
        if (power < -50.0f) continue;
        if (power > 0.0f) power = 0.0f;
        const float e = __expf(power);
        const float go0 = grad_image[3 * p], go1 = grad_image[3 * p + 1], go2 = grad_image[3 * p + 2];
        const float ga = grad_alpha[p];
        const float dot = go0 * c0 + go1 * c1 + go2 * c2;
        gwt += e * (dot + ga);
        gc0 += e * weight * go0;
        gc1 += e * weight * go1;
        gc2 += e * weight * go2;
        const float dpow = weight * (dot + ga) * e;
        const float cm = -0.5f * dpow;
        gi0 += cm * dx * dx;
        gi1 += cm * dx * dy;
        gi2 += cm * dy * dx;
        gi3 += cm * dy * dy;
        gm0 += 0.5f * dpow * ((inv.x + inv.x) * dx + (inv.y + inv.z) * dy);
        gm1 += 0.5f * dpow * ((inv.z + inv.y) * dx + (inv.w + inv.w) * dy);
    }
    d_means[2 * g] = gm0; d_means[2 * g + 1] = gm1;
    d_inv[4 * g] = gi0; d_inv[4 * g + 1] = gi1; d_inv[4 * g + 2] = gi2; d_inv[4 * g + 3] = gi3;
    d_w[g] = gwt;
    d_c[3 * g] = gc0; d_c[3 * g + 1] = gc1; d_c[3 * g + 2] = gc2;
}

}  // namespace sa
}  // namespace us3d

using namespace us3d;
using namespace us3d::sa;

static bool g_sa_sort_attr[128];

static int sa_check(int H, int W, float hw, float hh, float rs, int64_t N, int64_t cap) {
    US3D_CHECK_ARG(H > 0 && W > 0, "image dimensions must be positive");
    US3D_CHECK_ARG(hw > 0.f && hh > 0.f, "physical half extents must be positive");
    US3D_CHECK_ARG(rs > 0.f, "radius_sigma must be positive");
    US3D_CHECK_ARG(N >= 0 && N <= 0x7fffffffLL, "Gaussian count out of range");
    US3D_CHECK_ARG(cap >= 0 && cap <= 0x7fffffffLL, "instance capacity must be in [0, 2^31)");
    return US3D_OK;
}

extern "C" size_t us3d_sa_workspace_bytes(int64_t n, int32_t H, int32_t W, int64_t cap) {
    if (n < 0 || H <= 0 || W <= 0 || cap < 0) return 0;
    const int64_t T = (int64_t)((W + TILE - 1) / TILE) * ((H + TILE - 1) / TILE);
    return carve(nullptr, n, T, cap).bytes;
}

extern "C" size_t us3d_sa_backward_scratch_bytes(int64_t cap) {
    return cap < 0 ? 0 : (size_t)cap * PARTIAL_F4 * sizeof(float4);
}

extern "C" int us3d_sa_bounded_forward(void* workspace, size_t workspace_bytes, int64_t n, int32_t H, int32_t W,
                                       float half_width, float half_height, const float* means2d, const float* inv2d,
                                       const float* weights, const float* colors, float radius_sigma, int64_t cap,
                                       float* out_image, float* out_alpha, void* stream_) {
    int st = sa_check(H, W, half_width, half_height, radius_sigma, n, cap);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace && out_image && out_alpha, "NULL pointer argument");
    US3D_CHECK_ARG(n == 0 || (means2d && inv2d && weights && colors), "NULL input pointer");
    US3D_CHECK_ARG((reinterpret_cast<uintptr_t>(means2d) & 7) == 0 && (reinterpret_cast<uintptr_t>(inv2d) & 15) == 0,
                   "means2d must be 8-byte and inv2d 16-byte aligned");
    const int gw = (W + TILE - 1) / TILE, gh = (H + TILE - 1) / TILE;
    const int64_t T = (int64_t)gw * gh;
    const Workspace w = carve(workspace, n, T, cap);
    US3D_CHECK_ARG(workspace_bytes >= w.bytes, "workspace too small: %zu < %zu", workspace_bytes, w.bytes);
    cudaStream_t stream = (cudaStream_t)stream_;
    const int prof = prof_begin("sa_forward", stream);
    init_kernel<<<(unsigned)((T + 255) / 256), 256, 0, stream>>>(T, w.tile_count, w.tile_cursor, w.header, cap, n);
    const unsigned gb = (unsigned)((n + 255) / 256);
    const float2* m2 = reinterpret_cast<const float2*>(means2d);
    const float4* iv = reinterpret_cast<const float4*>(inv2d);
    if (n > 0)
        preprocess_kernel<<<gb, 256, 0, stream>>>(n, H, W, gw, gh, half_width, half_height, radius_sigma, m2, iv,
                                                  w.rects, w.bbox, w.touched, w.tile_count);
    US3D_CHECK_CUDA(launch_rect_count(n, gw, T, RectOf4{w.rects}, w.tile_count, stream));
    US3D_CHECK_CUDA(exclusive_scan(w.touched, n, w.inst_offset, w.bs_g, w.header + H_SCAN_G, stream));
    US3D_CHECK_CUDA(exclusive_scan(w.tile_count, T, w.tile_start, w.bs_t, w.header + H_SCAN_T, stream));
    check_kernel<<<1, 1, 0, stream>>>(w.header, cap);
    US3D_CHECK_CUDA(launch_rect_scatter(n, gw, T, RectOf4{w.rects}, nullptr, w.inst_offset, w.tile_start,
                                        w.tile_cursor, w.header, w.keys, w.slot_inst, stream));
    US3D_CHECK_CUDA(launch_tile_sort(T, n, w.tile_start, w.header, w.keys, w.slot_inst, w.sorted_gid, w.sorted_inst,
                                     g_sa_sort_attr, stream));
    const int split = frame_split(T);
    forward_kernel<<<(unsigned)(T * split), TILE * TILE, 0, stream>>>(
        split, H, W, gw, half_width, half_height, radius_sigma, m2, iv, weights, colors, w.tile_start, w.sorted_gid,
        w.header, out_image, out_alpha, w.fwd_part);
    US3D_CHECK_LAUNCH("sa forward");
    if (split > 1) {
        combine_kernel<<<(unsigned)((T * TILE * TILE + 255) / 256), 256, 0, stream>>>(split, (int)T, H, W, gw, w.header,
                                                                                   w.fwd_part, out_image, out_alpha);
        US3D_CHECK_LAUNCH("sa forward combine");
    }
    prof_end(prof, stream);
    count_launches(1 + 3 * (n > 0) + 6 + 1 + tile_sort_launches(n) + 1 + (split > 1));
    return US3D_OK;
}

extern "C" int us3d_sa_read_status(const void* workspace, int64_t* total, int32_t* flags, void* stream_) {
    US3D_CHECK_ARG(workspace != nullptr, "workspace is NULL");
    long long hdr[H_WORDS];
    cudaStream_t stream = (cudaStream_t)stream_;
    US3D_CHECK_CUDA(cudaMemcpyAsync(hdr, workspace, sizeof(hdr), cudaMemcpyDeviceToHost, stream));
    US3D_CHECK_CUDA(cudaStreamSynchronize(stream));
    if (total) *total = hdr[H_TOTAL];
    if (flags) *flags = (int32_t)hdr[H_FLAGS];
    return US3D_OK;
}

extern "C" int us3d_sa_bounded_backward(void* workspace, int64_t n, int32_t H, int32_t W, float half_width,
                                        float half_height, const float* means2d, const float* inv2d,
                                        const float* weights, const float* colors, const float* grad_image,
                                        const float* grad_alpha, float radius_sigma, int64_t cap, void* scratch,
                                        size_t scratch_bytes, float* d_means, float* d_inv, float* d_weights,
                                        float* d_colors, void* stream_) {
    int st = sa_check(H, W, half_width, half_height, radius_sigma, n, cap);
    if (st != US3D_OK) return st;
    US3D_CHECK_ARG(workspace && grad_image && grad_alpha, "NULL pointer argument");
    US3D_CHECK_ARG(scratch_bytes >= us3d_sa_backward_scratch_bytes(cap), "backward scratch too small");
    US3D_CHECK_ARG(n == 0 || (d_means && d_inv && d_weights && d_colors), "NULL gradient pointer");
    const int gw = (W + TILE - 1) / TILE, gh = (H + TILE - 1) / TILE;
    const int64_t T = (int64_t)gw * gh;
    const Workspace w = carve(workspace, n, T, cap);
    cudaStream_t stream = (cudaStream_t)stream_;
    float4* partial = reinterpret_cast<float4*>(scratch);
    const int prof = prof_begin("sa_backward", stream);
    const int split = frame_split(T);
    backward_kernel<<<(unsigned)(T * split), 256, 0, stream>>>(split, H, W, gw, half_width, half_height, radius_sigma,
                                                     reinterpret_cast<const float2*>(means2d),
                                                     reinterpret_cast<const float4*>(inv2d), weights, colors,
                                                     grad_image, grad_alpha, w.bbox, w.tile_start, w.sorted_gid,
                                                     w.sorted_inst, w.header, partial);
    if (n > 0)
        reduce_kernel<<<(unsigned)((n * REDUCE_COLS + REDUCE_THREADS - 1) / REDUCE_THREADS), REDUCE_THREADS, 0,
                        stream>>>(n, w.inst_offset, w.header, partial, d_means, d_inv, d_weights, d_colors);
    US3D_CHECK_LAUNCH("sa backward");
    prof_end(prof, stream);
    count_launches(1 + (n > 0));
    return US3D_OK;
}

extern "C" int us3d_sa_export_bins(const void* workspace, int64_t n, int32_t H, int32_t W, int64_t cap,
                                   int32_t* out_sorted_ids, int32_t* out_range_start, int32_t* out_range_end,
                                   void* stream_) {
    US3D_CHECK_ARG(workspace && out_range_start && out_range_end && H > 0 && W > 0, "bad argument");
    const int gw = (W + TILE - 1) / TILE, gh = (H + TILE - 1) / TILE;
    const int64_t T = (int64_t)gw * gh;
    const Workspace w = carve(const_cast<void*>(workspace), n, T, cap);
    export_kernel<<<(unsigned)T, 256, 0, (cudaStream_t)stream_>>>((int)T, w.tile_start, w.sorted_gid, out_sorted_ids,
                                                                  out_range_start, out_range_end);
    US3D_CHECK_LAUNCH("sa export");
    count_launches(1);
    return US3D_OK;
}

extern "C" int us3d_sa_dense_forward(int64_t n_pixels, int64_t n, const float* pixels, const float* means2d,
                                     const float* inv2d, const float* weights, const float* colors, float* out_image,
                                     float* out_alpha, void* stream_) {
    US3D_CHECK_ARG(n_pixels >= 0 && n >= 0, "negative size");
    US3D_CHECK_ARG(n_pixels == 0 || (pixels && out_image && out_alpha), "NULL pointer argument");
    if (n_pixels == 0) return US3D_OK;
    dense_forward_kernel<<<(unsigned)((n_pixels + 255) / 256), 256, 0, (cudaStream_t)stream_>>>(
        n_pixels, n, reinterpret_cast<const float2*>(pixels), reinterpret_cast<const float2*>(means2d),
        reinterpret_cast<const float4*>(inv2d), weights, colors, out_image, out_alpha);
    US3D_CHECK_LAUNCH("sa dense forward");
    count_launches(1);
    return US3D_OK;
}

extern "C" int us3d_sa_dense_backward(int64_t n_pixels, int64_t n, const float* pixels, const float* means2d,
                                      const float* inv2d, const float* weights, const float* colors,
                                      const float* grad_image, const float* grad_alpha, float* d_means, float* d_inv,
                                      float* d_weights, float* d_colors, void* stream_) {
    US3D_CHECK_ARG(n_pixels >= 0 && n >= 0, "negative size");
    if (n == 0) return US3D_OK;
    dense_backward_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream_>>>(
        n_pixels, n, reinterpret_cast<const float2*>(pixels), reinterpret_cast<const float2*>(means2d),
        reinterpret_cast<const float4*>(inv2d), weights, colors, grad_image, grad_alpha, d_means, d_inv, d_weights,
        d_colors);
    US3D_CHECK_LAUNCH("sa dense backward");
    count_launches(1);
    return US3D_OK;
}
