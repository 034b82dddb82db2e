// One instantiation of the fused tile kernel (FE degree 1, 2 material
// state(s), polynomial properties up to degree 4); one translation unit
// per instantiation so the build runs in parallel.
#include "tile_kernel.cuh"

namespace adm
{
// Launches the persistent tile kernel over n_items work items with at most
// the number of CTAs that are resident at once on the device.
void launch_tile_d1_s2_p4(CUtensorMap const &map, KernelArgs const &a, int n_items,
                            cudaStream_t stream)
{
  static int grid_cap = 0;
  if (grid_cap == 0)
  {
    cudaFuncSetAttribute(tile_kernel<1, 2, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)TD<1>::SMEM);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_kernel<1, 2, 4>, TD<1>::NT,
                                                  TD<1>::SMEM);
    grid_cap = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }
  int const grid = n_items < grid_cap ? n_items : grid_cap;
  tile_kernel<1, 2, 4><<<grid, TD<1>::NT, TD<1>::SMEM, stream>>>(map, a, n_items);
}
} // namespace adm
