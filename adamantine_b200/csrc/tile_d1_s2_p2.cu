// Instantiations of the FE_Q(1) cell kernel (one thread per cell), 2 material
// state(s) and polynomial properties up to degree 2, in the three launch
// schedules; one translation unit per (degree, states, degree) so the build
// runs in parallel.
#include "cell_kernel_q1.cuh"

namespace adm
{
void launch_tile_d1_s2_p2(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  launch_cell_q1<2, 2>(map, a, n_items, stream);
}
} // namespace adm
