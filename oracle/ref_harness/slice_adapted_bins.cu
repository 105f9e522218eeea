// TEST INFRASTRUCTURE ONLY. Compiles the reference's slice-adapted splat source
// (ops/slice_adapted_3dgs_renderer/src/render.cu, included unmodified) together with one
// binding that returns what its internal build_tile_binning computes for N >= 16384
// Gaussians (render.cu:624-754): sorted Gaussian ids and per-tile ranges.
#include "render.cu"

std::vector<torch::Tensor> RefTileBinning(int64_t H, int64_t W, double half_width, double half_height,
                                          torch::Tensor means2d, torch::Tensor inv2d, double radius_sigma) {
    TileBinning b = build_tile_binning((int)H, (int)W, (float)half_width, (float)half_height, means2d.contiguous(),
                                       inv2d.contiguous(), means2d.size(0), (float)radius_sigma,
                                       at::cuda::getCurrentCUDAStream());
    cudaStreamSynchronize(at::cuda::getCurrentCUDAStream());
    return {b.sorted_gauss_ids, b.tile_range_starts, b.tile_range_ends};
}

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) { m.def("RefTileBinning", &RefTileBinning); }
