// iq_tile_r3.cu -- instantiation of the tile-pass kernel with R = 3 register
// slots (8 amplitudes per thread), 256 threads per CTA, 2 CTAs per SM (<= 128
// registers per thread: twice the resident warps of R = 4).  Kept in
// its own translation unit so the instantiations compile in parallel.
#include "iq_tile.cuh"

namespace iqb {

cudaError_t launch_tile_r3(const CUtensorMap& tm, const PassDesc& d, const double2* mats, int* dev_status, int nbuf,
                          unsigned grid, size_t smem, cudaStream_t st, double* grad_partials) {
  auto kern = tile_pass_kernel<3, tile_pass_threads(3), 2>;
  static std::atomic<uint64_t> smem_set{0};
  cudaError_t r = allow_full_dynamic_smem(kern, smem_set);
  if (r != cudaSuccess) return r;
  kern<<<grid, tile_pass_threads(3), smem, st>>>(tm, d, mats, dev_status, nbuf, grad_partials);
  return cudaGetLastError();
}

}  // namespace iqb
