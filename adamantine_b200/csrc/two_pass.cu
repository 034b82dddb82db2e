// Launcher of the two-pass schedule's gather pass (two_pass_gather_kernel in
// tile_kernel.cuh) for FE degrees 1 and 2.
#include "thermal.hpp"
#include "tile_kernel.cuh"

namespace adm
{
void launch_two_pass_gather(int deg, KernelArgs const &a, int n_members, cudaStream_t stream)
{
  // one CTA per (tile, member)
  dim3 const grid((unsigned)(a.nt[0] * a.nt[1] * a.nt[2]), (unsigned)n_members);
  if (deg == 1)
    two_pass_gather_kernel<1><<<grid, 128, 0, stream>>>(a);
  else
    two_pass_gather_kernel<2><<<grid, 128, 0, stream>>>(a);
  ADM_CK(cudaGetLastError());
}

size_t two_pass_halo_size(int deg)
{
  return deg == 1 ? (size_t)HaloOf<1>::SIZE : (size_t)HaloOf<2>::SIZE;
}
} // namespace adm
