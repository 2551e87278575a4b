// iq_tile_r5.cu -- instantiation of the tile-pass kernel with R = 5 register
// slots (32 amplitudes per thread), 128 threads per CTA, 1 CTA(s) per SM.  Kept in
// its own translation unit so the instantiations compile in parallel.
#include "iq_tile.cuh"

namespace iqb {

cudaError_t launch_tile_r5(const CUtensorMap& tm, const PassDesc& d, const double2* mats, int* dev_status, int nbuf,
                          unsigned grid, size_t smem, cudaStream_t st, double* grad_partials) {
  auto kern = tile_pass_kernel<5, tile_pass_threads(5), 1>;
  static std::atomic<uint64_t> smem_set{0};
  cudaError_t r = allow_full_dynamic_smem(kern, smem_set);
  if (r != cudaSuccess) return r;
  kern<<<grid, tile_pass_threads(5), smem, st>>>(tm, d, mats, dev_status, nbuf, grad_partials);
  return cudaGetLastError();
}

}  // namespace iqb
