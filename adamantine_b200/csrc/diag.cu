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

namespace
{
// Eight independent FMA chains per thread, so that the FP64 pipe, not the
// dependent-issue latency, bounds the rate.
__global__ void __launch_bounds__(256) fma_rate_kernel(double b, double c, int iters, double *out)
{
  double a[8];
#pragma unroll
  for (int k = 0; k < 8; ++k)
    a[k] = threadIdx.x * 1e-3 + k;
  for (int it = 0; it < iters; ++it)
  {
#pragma unroll
    for (int k = 0; k < 8; ++k)
      a[k] = fma(a[k], b, c);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k)
    s += a[k];
  out[blockIdx.x * (int64_t)blockDim.x + threadIdx.x] = s;
}
} // namespace

extern "C" int adm_diag_fp64_fma_rate(int device, double *tflops)
{
  if (!tflops)
    return ADM_ERR_INVALID;
  *tflops = 0.0;
  if (cudaSetDevice(device) != cudaSuccess)
    return ADM_ERR_CUDA;
  int n_sm = 0;
  if (cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return ADM_ERR_CUDA;
  int const blocks = n_sm * 8, threads = 256, iters = 4096;
  double *out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * blocks * threads) != cudaSuccess)
    return ADM_ERR_ALLOC;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 0.f;
  int rc = ADM_OK;
  for (int rep = 0; rep < 6 && rc == ADM_OK; ++rep)
  {
    cudaEventRecord(e0);
    fma_rate_kernel<<<blocks, threads>>>(0.999999, 1e-6, iters, out);
    cudaEventRecord(e1);
    if (cudaGetLastError() != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess)
      rc = ADM_ERR_CUDA;
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0 && (best == 0.f || ms < best))
      best = ms;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (rc == ADM_OK && best > 0.f)
    *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (best * 1e-3) / 1e12;
  return rc;
}

namespace
{
// The bounded mbarrier wait of the tile kernels on a barrier that nothing
// arrives at: the wait must give up after `limit_ns` nanoseconds and report
// it.
__global__ void wait_timeout_kernel(long long limit_ns, int *status)
{
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0)
  {
    adm::mbar_init(&bar, 1);
    adm::fence_mbar_init();
  }
  __syncthreads();
  bool const arrived = adm::mbar_wait(&bar, 0u, limit_ns);
  if (__syncthreads_or(!arrived) && threadIdx.x == 0)
    *status = 1;
}
} // namespace

extern "C" int adm_diag_wait_timeout(long long limit_us, int32_t *timed_out)
{
  if (!timed_out || limit_us < 1 || limit_us > 1000000)
    return ADM_ERR_INVALID;
  *timed_out = 0;
  int *d = nullptr;
  if (cudaMalloc(&d, sizeof(int)) != cudaSuccess)
    return ADM_ERR_ALLOC;
  int rc = ADM_OK;
  if (cudaMemset(d, 0, sizeof(int)) != cudaSuccess)
    rc = ADM_ERR_CUDA;
  if (rc == ADM_OK)
  {
    wait_timeout_kernel<<<1, 64>>>(limit_us * 1000, d);
    if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess)
      rc = ADM_ERR_CUDA;
  }
  int h = 0;
  if (rc == ADM_OK && cudaMemcpy(&h, d, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = ADM_ERR_CUDA;
  cudaFree(d);
  *timed_out = h;
  return rc;
}
