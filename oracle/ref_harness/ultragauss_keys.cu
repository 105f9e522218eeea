// TEST INFRASTRUCTURE ONLY. Drives the reference's own UltraGauss mapper kernels
// (compiled from ops/ultragauss_renderer/src/mapper/core.cu) and CUB exactly as the
// reference's MapperForwardCUDA does up to the tile ranges
// (ops/ultragauss_renderer/src/mapper/wrapper_mapper.cu:64-151), and returns the
// intermediate arrays that MapperForwardCUDA keeps private: per-Gaussian tile counts,
// rectangles and depths, the sorted keys and values, and the tile ranges.
#include <torch/extension.h>
#include <ATen/cuda/CUDAContext.h>
#include <cub/cub.cuh>

#include "mapper/core.cuh"

std::vector<torch::Tensor> RefBinning(const torch::Tensor& means_packed, const torch::Tensor& tril,
                                      const torch::Tensor& org, const torch::Tensor& lat, const torch::Tensor& ax,
                                      const torch::Tensor& ele, int H, int W, float dlat, float dax, float near_mm,
                                      float coloff, float chi2, bool sort_by_depth, float beta) {
    const int G = means_packed.size(0);
    auto oi = torch::TensorOptions().dtype(torch::kInt32).device(torch::kCUDA);
    auto of = torch::TensorOptions().dtype(torch::kFloat32).device(torch::kCUDA);
    auto ol = torch::TensorOptions().dtype(torch::kInt64).device(torch::kCUDA);
    cudaStream_t stream = at::cuda::getCurrentCUDAStream();
    const int block = 256, grid = (G + block - 1) / block;
    torch::Tensor touched = torch::zeros({G + 1}, oi);
    torch::Tensor rects = torch::zeros({G, 4}, oi);
    torch::Tensor depths = torch::zeros({G}, of);
    kernel_project_gauss_and_compute_tile_rects<<<grid, block, 0, stream>>>(
        G, reinterpret_cast<float4*>(means_packed.data_ptr<float>()), tril.data_ptr<float>(), H, W, near_mm, dlat,
        dax, coloff, chi2, beta, org.data_ptr<float>(), lat.data_ptr<float>(), ele.data_ptr<float>(),
        ax.data_ptr<float>(), touched.data_ptr<int>(), reinterpret_cast<int4*>(rects.data_ptr<int>()),
        depths.data_ptr<float>());
    torch::Tensor offsets = torch::empty({G + 1}, oi);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, touched.data_ptr<int>(), offsets.data_ptr<int>(), G + 1, stream);
    torch::Tensor temp = torch::empty({(long)tb}, torch::TensorOptions().dtype(torch::kByte).device(torch::kCUDA));
    cub::DeviceScan::ExclusiveSum(temp.data_ptr(), tb, touched.data_ptr<int>(), offsets.data_ptr<int>(), G + 1,
                                  stream);
    const int n = offsets[G].item<int>();
    const int gw = (W + SLICE_TILE_SIZE - 1) / SLICE_TILE_SIZE, gh = (H + SLICE_TILE_SIZE - 1) / SLICE_TILE_SIZE;
    torch::Tensor rs = torch::full({gw * gh}, -1, oi), re = torch::full({gw * gh}, -1, oi);
    torch::Tensor k1 = torch::empty({n}, ol), k2 = torch::empty({n}, ol);
    torch::Tensor v1 = torch::empty({n}, oi), v2 = torch::empty({n}, oi);
    if (n > 0) {
        kernel_generate_tile_depth_keys<<<grid, block, 0, stream>>>(
            G, gw, sort_by_depth, reinterpret_cast<int4*>(rects.data_ptr<int>()), depths.data_ptr<float>(),
            offsets.data_ptr<int>(), (uint64_t*)k1.data_ptr<int64_t>(), v1.data_ptr<int>());
        cub::DoubleBuffer<uint64_t> dk((uint64_t*)k1.data_ptr<int64_t>(), (uint64_t*)k2.data_ptr<int64_t>());
        cub::DoubleBuffer<int> dv(v1.data_ptr<int>(), v2.data_ptr<int>());
        tb = 0;
        const int b0 = sort_by_depth ? 0 : 32;
        cub::DeviceRadixSort::SortPairs(nullptr, tb, dk, dv, n, b0, 64, stream);
        torch::Tensor t2 = torch::empty({(long)tb}, torch::TensorOptions().dtype(torch::kByte).device(torch::kCUDA));
        cub::DeviceRadixSort::SortPairs(t2.data_ptr(), tb, dk, dv, n, b0, 64, stream);
        kernel_identify_tile_ranges<<<(n + block - 1) / block, block, 0, stream>>>(n, dk.Current(), rs.data_ptr<int>(),
                                                                                  re.data_ptr<int>());
        torch::Tensor ks = dk.Current() == (uint64_t*)k1.data_ptr<int64_t>() ? k1 : k2;
        torch::Tensor vs = dv.Current() == v1.data_ptr<int>() ? v1 : v2;
        cudaStreamSynchronize(stream);
        return {touched.narrow(0, 0, G), rects, depths, ks, vs, rs, re};
    }
    return {touched.narrow(0, 0, G), rects, depths, k1, v1, rs, re};
}

PYBIND11_MODULE(TORCH_EXTENSION_NAME, m) { m.def("RefBinning", &RefBinning); }
