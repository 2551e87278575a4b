// iq_tile_r4.cu -- instantiation of the tile-pass kernel with R = 4 register
// slots (16 amplitudes per thread), 128 threads per CTA, 2 CTA(s) per SM.  Kept in
// its own translation unit so the instantiations compile in parallel.
#include "iq_tile.cuh"

namespace iqb {

cudaError_t launch_tile_r4(const CUtensorMap& tm, const PassDesc& d, const double2* mats, int* dev_status, int nbuf,
                          unsigned grid, size_t smem, cudaStream_t st, double* grad_partials) {
  auto kern = tile_pass_kernel<4, tile_pass_threads(4), 2>;
  static std::atomic<uint64_t> smem_set{0};
  cudaError_t r = allow_full_dynamic_smem(kern, smem_set);
  if (r != cudaSuccess) return r;
  kern<<<grid, tile_pass_threads(4), smem, st>>>(tm, d, mats, dev_status, nbuf, grad_partials);
  return cudaGetLastError();
}

}  // namespace iqb
