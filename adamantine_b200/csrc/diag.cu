// Diagnostic kernels of include/adamantine_b200_diag.h.
#include "../../include/adamantine_b200.h"
#include "../../include/adamantine_b200_diag.h"
#include "tile_kernel.cuh"

namespace
{
__global__ void reciprocal_kernel(double const *x, double *y, double *y_ref, int64_t n)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n)
  {
    y[i] = adm::recip(x[i]);
    y_ref[i] = 1.0 / x[i];
  }
}
} // namespace

extern "C" int adm_diag_reciprocal(double const *x, double *y, double *y_ref, int64_t n)
{
  if (!x || !y || !y_ref || n < 0)
    return ADM_ERR_INVALID;
  if (n == 0)
    return ADM_OK;
  reciprocal_kernel<<<(unsigned)((n + 255) / 256), 256>>>(x, y, y_ref, n);
  if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
    return ADM_ERR_CUDA;
  return ADM_OK;
}
