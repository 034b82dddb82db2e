// Instantiations of the fused tile kernel for FE degree 2, 3 material
// state(s) and polynomial properties up to degree 4, in the three launch
// schedules; one translation unit per (degree, states, degree) so the build
// runs in parallel.
#include "tile_kernel.cuh"

namespace adm
{
void launch_tile_d2_s3_p4(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  launch_tile_t<2, 3, 4>(map, a, n_items, stream);
}
} // namespace adm
