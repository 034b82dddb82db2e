// EnKF analysis of a batched ensemble on the GPU, FP64 throughout.
//
// Restates DataAssimilator::update_ensemble (source/DataAssimilator.cc:95-189)
// with localization "none": the perturbed-observation update
//   x_k += P H^T (H P H^T + R)^-1 (y + e_k - H x_k),   P = A A^T / (N - 1),
// A the anomalies of the augmented states [x_k; p_k] about the ensemble
// mean (calc_sample_covariance_sparse, :690-752), H picking one state entry
// per observation (calc_Hx, :614-628), R the observation covariance. The
// reference forms the sparse P and solves with GMRES per member
// (apply_kalman_gain, :403-476); here P is never formed:
//   HA  = H A                        (m x N)
//   C   = HA HA^T / (N - 1) + R      (m x m, lower triangle)
//   C   = L L^T                      (blocked Cholesky, own kernels)
//   Z   = C^-1 D,  D_k = y + e_k - H x_k   (triangular solves, N columns)
//   W   = HA^T Z / (N - 1)           (N x N)
//   x_k += A W[:, k]                 (one pass over the states)
// which is the same matrix product evaluated in a different order.
#include "capi_common.hpp"
#include "../../include/adamantine_b200_ensemble.h"

#include <cmath>
#include <cstring>

namespace adm
{
namespace
{
constexpr int kNB = 64;        // Cholesky block size
constexpr int kMaxN = 64;      // members per analysis
constexpr int kMaxObs = 16384; // observations (the solve keeps one column in shared memory)
constexpr int kMaxGain = 256;  // members of a sharded analysis (all GPUs)

enum EnkfError
{
  EERR_NONE = 0,
  EERR_NOT_SPD = 1,   // a Cholesky pivot was not positive and finite
  EERR_BAD_INDEX = 2  // an observation index outside [0, n_state)
};

// HA[k][j] = x_k[idx_k[j]] - mean_k(...), D[k][j] = y_j + e_k[j] - x_k[idx_k[j]].
__global__ void hx_kernel(double const *states, int64_t stride, int n_members, int64_t n_state,
                          int64_t const *idx, int m, double const *obs, double const *pert,
                          double *HA, double *D, int *err)
{
  int const j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m)
    return;
  double sum = 0.0;
  for (int k = 0; k < n_members; ++k)
  {
    int64_t i = idx[(int64_t)k * m + j];
    if (i < 0 || i >= n_state)
    {
      atomicCAS(err, 0, (int)EERR_BAD_INDEX);
      i = 0;
    }
    double const hx = states[(int64_t)k * stride + i];
    HA[(int64_t)k * m + j] = hx;
    D[(int64_t)k * m + j] = obs[j] + pert[(int64_t)k * m + j] - hx;
    sum += hx;
  }
  double const mean = sum / n_members;
  for (int k = 0; k < n_members; ++k)
    HA[(int64_t)k * m + j] -= mean;
}

// Lower triangle of C = HA^T HA * scale + R (R diagonal var, or dense cov).
// 32 x 32 output tile per block, 256 threads, 4 outputs per thread.
__global__ void __launch_bounds__(256) cov_kernel(double const *HA, int n_members, int m, double scale,
                                                  double const *var, double const *cov, double *C)
{
  int const bi = blockIdx.y, bj = blockIdx.x;
  if (bj > bi)
    return;
  __shared__ double si[32][33], sj[32][33]; // [k][row]
  int const tid = threadIdx.x;
  int const tr = tid / 8, tc = (tid % 8) * 4; // row tr, columns tc..tc+3
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  for (int k0 = 0; k0 < n_members; k0 += 32)
  {
    for (int e = tid; e < 32 * 32; e += 256)
    {
      int const kk = e / 32, r = e % 32;
      int const k = k0 + kk;
      int const gi = bi * 32 + r, gj = bj * 32 + r;
      si[kk][r] = (k < n_members && gi < m) ? HA[(int64_t)k * m + gi] : 0.0;
      sj[kk][r] = (k < n_members && gj < m) ? HA[(int64_t)k * m + gj] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int kk = 0; kk < 32; ++kk)
    {
      double const a = si[kk][tr];
#pragma unroll
      for (int c = 0; c < 4; ++c)
        acc[c] = fma(a, sj[kk][tc + c], acc[c]);
    }
    __syncthreads();
  }
  int const gi = bi * 32 + tr;
  if (gi >= m)
    return;
#pragma unroll
  for (int c = 0; c < 4; ++c)
  {
    int const gj = bj * 32 + tc + c;
    if (gj > gi || gj >= m)
      continue;
    double v = acc[c] * scale;
    if (cov)
      v += cov[(int64_t)gi * m + gj];
    else if (gi == gj)
      v += var[gi];
    C[(int64_t)gi * m + gj] = v;
  }
}

// Unblocked Cholesky of the diagonal block at (k0, k0), one CTA.
__global__ void __launch_bounds__(256) potrf_diag_kernel(double *C, int m, int k0, int *err)
{
  __shared__ double a[kNB][kNB + 1];
  int const nb = min(kNB, m - k0);
  int const tid = threadIdx.x;
  for (int e = tid; e < nb * nb; e += blockDim.x)
  {
    int const r = e / nb, c = e % nb;
    a[r][c] = c <= r ? C[(int64_t)(k0 + r) * m + k0 + c] : 0.0;
  }
  __syncthreads();
  for (int j = 0; j < nb; ++j)
  {
    if (tid == 0)
    {
      double const d = a[j][j];
      if (!(d > 0.0) || !isfinite(d))
      {
        atomicCAS(err, 0, (int)EERR_NOT_SPD);
        a[j][j] = 1.0;
      }
      else
        a[j][j] = sqrt(d);
    }
    __syncthreads();
    double const piv = a[j][j];
    for (int i = j + 1 + tid; i < nb; i += blockDim.x)
      a[i][j] /= piv;
    __syncthreads();
    int const w = nb - j - 1;
    for (int e = tid; e < w * w; e += blockDim.x)
    {
      int const i = j + 1 + e / w, l = j + 1 + e % w;
      if (l <= i)
        a[i][l] -= a[i][j] * a[l][j];
    }
    __syncthreads();
  }
  for (int e = tid; e < nb * nb; e += blockDim.x)
  {
    int const r = e / nb, c = e % nb;
    if (c <= r)
      C[(int64_t)(k0 + r) * m + k0 + c] = a[r][c];
  }
}

// Panel below the diagonal block: L[r, k0:k0+nb] = C[r, k0:k0+nb] L_kk^-T,
// one row per thread.
__global__ void __launch_bounds__(128) trsm_panel_kernel(double *C, int m, int k0)
{
  __shared__ double l[kNB][kNB + 1];
  __shared__ double inv_d[kNB];
  int const nb = min(kNB, m - k0);
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x)
  {
    int const r = e / nb, c = e % nb;
    l[r][c] = c <= r ? C[(int64_t)(k0 + r) * m + k0 + c] : 0.0;
  }
  __syncthreads();
  if (threadIdx.x < nb)
    inv_d[threadIdx.x] = 1.0 / l[threadIdx.x][threadIdx.x];
  __syncthreads();
  int const r = k0 + nb + blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m)
    return;
  double *row = C + (int64_t)r * m + k0;
  double x[kNB];
#pragma unroll
  for (int j = 0; j < kNB; ++j)
  {
    if (j < nb)
    {
      double s = row[j];
#pragma unroll
      for (int q = 0; q < j; ++q)
        s -= x[q] * l[j][q];
      x[j] = s * inv_d[j];
      row[j] = x[j];
    }
  }
}

// Trailing update of the lower triangle: C[i][j] -= L[i, panel] L[j, panel]^T
// for 64 x 64 tiles right of / below the panel.
__global__ void __launch_bounds__(256) syrk_update_kernel(double *C, int m, int k0)
{
  int const base = k0 + kNB;
  int const bi = blockIdx.y, bj = blockIdx.x;
  if (bj > bi)
    return;
  int const i0 = base + bi * 64, j0 = base + bj * 64;
  // the panel's 64 columns in two chunks of 32 (static shared memory)
  __shared__ double pi[64][33], pj[64][33];
  int const tid = threadIdx.x;
  int const tr = (tid / 16) * 4, tc = (tid % 16) * 4;
  double acc[4][4] = {};
  for (int q0 = 0; q0 < kNB; q0 += 32)
  {
    for (int e = tid; e < 64 * 32; e += 256)
    {
      int const r = e / 32, c = e % 32;
      pi[r][c] = i0 + r < m ? C[(int64_t)(i0 + r) * m + k0 + q0 + c] : 0.0;
      pj[r][c] = j0 + r < m ? C[(int64_t)(j0 + r) * m + k0 + q0 + c] : 0.0;
    }
    __syncthreads();
    for (int q = 0; q < 32; ++q)
    {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
      {
        a[u] = pi[tr + u][q];
        b[u] = pj[tc + u][q];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v)
          acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
    {
      int const gi = i0 + tr + u, gj = j0 + tc + v;
      if (gi < m && gj <= gi)
        C[(int64_t)gi * m + gj] -= acc[u][v];
    }
}

// Z_k = C^-1 D_k for one member k per CTA: forward L y = d, backward
// L^T z = y, blocked by kNB; the diagonal block is solved by warp 0 with
// shuffles, the off-diagonal updates by all threads. The column lives in
// shared memory.
__global__ void __launch_bounds__(256) solve_kernel(double const *L, int m, double const *D, double *Z)
{
  extern __shared__ double col[]; // [m]
  int const k = blockIdx.x;
  int const tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < m; i += blockDim.x)
    col[i] = D[(int64_t)k * m + i];
  __syncthreads();
  int const nblk = (m + kNB - 1) / kNB;
  // forward
  for (int b = 0; b < nblk; ++b)
  {
    int const k0 = b * kNB, nb = min(kNB, m - k0);
    if (warp == 0)
    {
      for (int j = 0; j < nb; ++j)
      {
        double s = 0.0;
        for (int q = lane; q < j; q += 32)
          s += L[(int64_t)(k0 + j) * m + k0 + q] * col[k0 + q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
          col[k0 + j] = (col[k0 + j] - s) / L[(int64_t)(k0 + j) * m + k0 + j];
        __syncwarp();
      }
    }
    __syncthreads();
    for (int i = k0 + nb + tid; i < m; i += blockDim.x)
    {
      double const *row = L + (int64_t)i * m + k0;
      double s = 0.0;
      for (int q = 0; q < nb; ++q)
        s += row[q] * col[k0 + q];
      col[i] -= s;
    }
    __syncthreads();
  }
  // backward
  for (int b = nblk - 1; b >= 0; --b)
  {
    int const k0 = b * kNB, nb = min(kNB, m - k0);
    if (warp == 0)
    {
      for (int j = nb - 1; j >= 0; --j)
      {
        double s = 0.0;
        for (int q = j + 1 + lane; q < nb; q += 32)
          s += L[(int64_t)(k0 + q) * m + k0 + j] * col[k0 + q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
          col[k0 + j] = (col[k0 + j] - s) / L[(int64_t)(k0 + j) * m + k0 + j];
        __syncwarp();
      }
    }
    __syncthreads();
    for (int i = tid; i < k0; i += blockDim.x)
    {
      double s = 0.0;
      for (int q = 0; q < nb; ++q)
        s += L[(int64_t)(k0 + q) * m + i] * col[k0 + q];
      col[i] -= s;
    }
    __syncthreads();
  }
  for (int i = tid; i < m; i += blockDim.x)
    Z[(int64_t)k * m + i] = col[i];
}

// W[a][b] = scale * sum_j HA[a][j] Z[b][j], one warp per entry.
__global__ void w_kernel(double const *HA, double const *Z, int n_members, int m, double scale, double *W)
{
  int const gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (gw >= n_members * n_members)
    return;
  int const a = gw / n_members, b = gw % n_members;
  double s = 0.0;
  for (int j = lane; j < m; j += 32)
    s += HA[(int64_t)a * m + j] * Z[(int64_t)b * m + j];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0)
    W[a * n_members + b] = s * scale;
}

// x_l[i] += sum_k (x_k[i] - mean[i]) W[k][l] for every state row i and the
// parameter rows; rows where a member's mask is 0 keep that member's value.
__global__ void __launch_bounds__(256) update_kernel(double *states, int64_t stride, int n_members,
                                                     int64_t n_state, double *params, int n_params,
                                                     uint8_t const *mask, double const *W)
{
  __shared__ double w[kMaxN * kMaxN];
  for (int e = threadIdx.x; e < n_members * n_members; e += blockDim.x)
    w[e] = W[e];
  __syncthreads();
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n_state + n_params)
    return;
  bool const is_param = i >= n_state;
  double a[kMaxN];
  double sum = 0.0;
#pragma unroll
  for (int k = 0; k < kMaxN; ++k)
  {
    a[k] = 0.0;
    if (k < n_members)
    {
      a[k] = is_param ? params[(int64_t)k * n_params + (i - n_state)] : states[(int64_t)k * stride + i];
      sum += a[k];
    }
  }
  double const mean = sum / n_members;
#pragma unroll
  for (int k = 0; k < kMaxN; ++k)
    a[k] -= mean;
  for (int l = 0; l < n_members; ++l)
  {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kMaxN; ++k)
      if (k < n_members)
        s = fma(a[k], w[k * n_members + l], s);
    if (is_param)
      params[(int64_t)l * n_params + (i - n_state)] += s;
    else if (!mask || mask[(int64_t)l * n_state + i])
      states[(int64_t)l * stride + i] += s;
  }
}
// HX[k][j] = x_k[idx_k[j]] for the local members (sharded analysis).
__global__ void observe_kernel(double const *states, int64_t stride, int n_members, int64_t n_state,
                               int64_t const *idx, int m, double *HX, int *err)
{
  int64_t const e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n_members * m)
    return;
  int const k = (int)(e / m);
  int64_t i = idx[e];
  if (i < 0 || i >= n_state)
  {
    atomicCAS(err, 0, (int)EERR_BAD_INDEX);
    i = 0;
  }
  HX[e] = states[(int64_t)k * stride + i];
}

// HA = HX - mean over members, D = y + e_k - HX (from all members' HX).
__global__ void center_kernel(double const *HX, int n_members, int m, double const *obs, double const *pert,
                              double *HA, double *D)
{
  int const j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= m)
    return;
  double sum = 0.0;
  for (int k = 0; k < n_members; ++k)
    sum += HX[(int64_t)k * m + j];
  double const mean = sum / n_members;
  for (int k = 0; k < n_members; ++k)
  {
    double const hx = HX[(int64_t)k * m + j];
    HA[(int64_t)k * m + j] = hx - mean;
    D[(int64_t)k * m + j] = obs[j] + pert[(int64_t)k * m + j] - hx;
  }
}

// U[k][i] = sum over the local members k' of (x_k'[i] - mean[i]) W[k'][k]
// for every member k of the ensemble (rows i: the states, then the
// parameters). W rows of the local members are staged in shared memory.
__global__ void __launch_bounds__(256) partial_update_kernel(double const *states, int64_t stride, int n_local,
                                                             int n_members, int64_t n_state, double const *params,
                                                             int n_params, double const *sum, double const *W,
                                                             double *U)
{
  extern __shared__ double w[]; // [n_local][n_members]
  for (int e = threadIdx.x; e < n_local * n_members; e += blockDim.x)
    w[e] = W[e];
  __syncthreads();
  int64_t const rows = n_state + n_params;
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= rows)
    return;
  bool const is_param = i >= n_state;
  double const mean = sum[i] / n_members;
  double a[kMaxN];
#pragma unroll
  for (int k = 0; k < kMaxN; ++k)
  {
    a[k] = 0.0;
    if (k < n_local)
      a[k] = (is_param ? params[(int64_t)k * n_params + (i - n_state)] : states[(int64_t)k * stride + i]) - mean;
  }
  for (int l = 0; l < n_members; ++l)
  {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < kMaxN; ++k)
      if (k < n_local)
        s = fma(a[k], w[k * n_members + l], s);
    U[(int64_t)l * rows + i] = s;
  }
}

// sum[i] = sum over the local members of the augmented state (rows: the
// states, then the parameters).
__global__ void local_sum_kernel(double const *states, int64_t stride, int n_local, int64_t n_state,
                                 double const *params, int n_params, double *sum)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n_state + n_params)
    return;
  double s = 0.0;
  for (int k = 0; k < n_local; ++k)
    s += i < n_state ? states[(int64_t)k * stride + i] : params[(int64_t)k * n_params + (i - n_state)];
  sum[i] = s;
}

// x_k[i] += U[k][i] for the local members (mask: 1 = update).
__global__ void apply_kernel(double *states, int64_t stride, int n_local, int64_t n_state, double *params,
                             int n_params, double const *U, uint8_t const *mask)
{
  int64_t const rows = n_state + n_params;
  int64_t const e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n_local * rows)
    return;
  int const k = (int)(e / rows);
  int64_t const i = e % rows;
  double const u = U[e];
  if (i >= n_state)
    params[(int64_t)k * n_params + (i - n_state)] += u;
  else if (!mask || mask[(int64_t)k * n_state + i])
    states[(int64_t)k * stride + i] += u;
}

} // namespace

// Workspace of the analysis, grown on demand.
struct Enkf
{
  int device = 0;
  cudaStream_t stream = nullptr;
  DevBuf<double> HA, D, C, Z, W;
  DevBuf<int> err;

  void analysis(int N, double *states, int64_t stride, int64_t n_state, double *params, int n_params,
                int m, int64_t const *idx, double const *obs, double const *var, double const *cov,
                double const *pert, uint8_t const *mask)
  {
    NvtxRange const nvtx_range("adm::enkf_analysis");
    if (N < 2 || N > kMaxN)
      throw Error(ADM_ERR_UNSUPPORTED, "the analysis takes 2 to 64 members");
    if (m < 1 || m > kMaxObs)
      throw Error(ADM_ERR_UNSUPPORTED, "the analysis takes 1 to 16384 observations");
    if (!states || !idx || !obs || !pert || (!var && !cov) || (n_params > 0 && !params) ||
        n_params < 0 || n_state < 1 || stride < n_state)
      throw Error(ADM_ERR_INVALID, "invalid analysis arguments");
    ADM_CK(cudaSetDevice(device));
    HA.alloc((size_t)N * m);
    D.alloc((size_t)N * m);
    Z.alloc((size_t)N * m);
    C.alloc((size_t)m * m);
    W.alloc((size_t)N * N);
    err.alloc(1);
    ADM_CK(cudaMemsetAsync(err.p, 0, sizeof(int), stream));
    hx_kernel<<<(m + 127) / 128, 128, 0, stream>>>(states, stride, N, n_state, idx, m, obs, pert, HA.p, D.p,
                                                   err.p);
    ADM_CK(cudaGetLastError());
    double const scale = 1.0 / (N - 1.0);
    int const t32 = (m + 31) / 32;
    cov_kernel<<<dim3(t32, t32), 256, 0, stream>>>(HA.p, N, m, scale, var, cov, C.p);
    ADM_CK(cudaGetLastError());
    for (int k0 = 0; k0 < m; k0 += kNB)
    {
      potrf_diag_kernel<<<1, 256, 0, stream>>>(C.p, m, k0, err.p);
      int const below = m - k0 - kNB;
      if (below > 0)
      {
        trsm_panel_kernel<<<(below + 127) / 128, 128, 0, stream>>>(C.p, m, k0);
        int const t = (below + 63) / 64;
        syrk_update_kernel<<<dim3(t, t), 256, 0, stream>>>(C.p, m, k0);
      }
      ADM_CK(cudaGetLastError());
    }
    // stop before touching the states if an index or a pivot was bad
    int h_err = 0;
    ADM_CK(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    ADM_CK(cudaStreamSynchronize(stream));
    if (h_err == EERR_BAD_INDEX)
      throw Error(ADM_ERR_INVALID, "an observation index is outside [0, n_state)");
    if (h_err == EERR_NOT_SPD)
      throw Error(ADM_ERR_DEVICE, "H P H^T + R is not positive definite (Cholesky pivot <= 0)");
    size_t const smem = (size_t)m * sizeof(double);
    ADM_CK(cudaFuncSetAttribute(solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    solve_kernel<<<N, 256, smem, stream>>>(C.p, m, D.p, Z.p);
    ADM_CK(cudaGetLastError());
    w_kernel<<<(N * N * 32 + 255) / 256, 256, 0, stream>>>(HA.p, Z.p, N, m, scale, W.p);
    ADM_CK(cudaGetLastError());
    int64_t const rows = n_state + n_params;
    update_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(states, stride, N, n_state, params,
                                                                      n_params, mask, W.p);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaStreamSynchronize(stream));
  }

  // ---- building blocks of the sharded analysis (members split over GPUs)
  void check_err()
  {
    int h_err = 0;
    ADM_CK(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    ADM_CK(cudaStreamSynchronize(stream));
    if (h_err == EERR_BAD_INDEX)
      throw Error(ADM_ERR_INVALID, "an observation index is outside [0, n_state)");
    if (h_err == EERR_NOT_SPD)
      throw Error(ADM_ERR_DEVICE, "H P H^T + R is not positive definite (Cholesky pivot <= 0)");
  }

  void observe(int N, double const *states, int64_t stride, int64_t n_state, int m, int64_t const *idx, double *hx)
  {
    if (N < 1 || m < 1 || !states || !idx || !hx || stride < n_state)
      throw Error(ADM_ERR_INVALID, "invalid observation arguments");
    ADM_CK(cudaSetDevice(device));
    err.alloc(1);
    ADM_CK(cudaMemsetAsync(err.p, 0, sizeof(int), stream));
    int64_t const total = (int64_t)N * m;
    observe_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(states, stride, N, n_state, idx, m, hx,
                                                                        err.p);
    ADM_CK(cudaGetLastError());
    check_err();
  }

  // W = HA^T (HA HA^T / (N-1) + R)^-1 D / (N-1) from every member's HX.
  void gain(int N, int m, double const *hx, double const *obs, double const *var, double const *cov,
            double const *pert, double *Wout)
  {
    NvtxRange const nvtx_range("adm::enkf_gain");
    if (N < 2 || N > kMaxGain)
      throw Error(ADM_ERR_UNSUPPORTED, "the gain takes 2 to 256 members");
    if (m < 1 || m > kMaxObs)
      throw Error(ADM_ERR_UNSUPPORTED, "the analysis takes 1 to 16384 observations");
    if (!hx || !obs || !pert || !Wout || (!var && !cov))
      throw Error(ADM_ERR_INVALID, "invalid gain arguments");
    ADM_CK(cudaSetDevice(device));
    HA.alloc((size_t)N * m);
    D.alloc((size_t)N * m);
    Z.alloc((size_t)N * m);
    C.alloc((size_t)m * m);
    err.alloc(1);
    ADM_CK(cudaMemsetAsync(err.p, 0, sizeof(int), stream));
    center_kernel<<<(m + 127) / 128, 128, 0, stream>>>(hx, N, m, obs, pert, HA.p, D.p);
    ADM_CK(cudaGetLastError());
    double const scale = 1.0 / (N - 1.0);
    factor(N, m, scale, var, cov);
    check_err();
    solve_and_w(N, m, scale, Wout);
    ADM_CK(cudaStreamSynchronize(stream));
  }

  void local_sum(int n_local, double const *states, int64_t stride, int64_t n_state, double const *params,
                 int n_params, double *sum)
  {
    if (n_local < 1 || !states || !sum || stride < n_state || n_params < 0 || (n_params > 0 && !params))
      throw Error(ADM_ERR_INVALID, "invalid local-sum arguments");
    ADM_CK(cudaSetDevice(device));
    int64_t const rows = n_state + n_params;
    local_sum_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(states, stride, n_local, n_state, params,
                                                                        n_params, sum);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaStreamSynchronize(stream));
  }

  void partial_update(int n_local, int N, double const *states, int64_t stride, int64_t n_state,
                      double const *params, int n_params, double const *sum, double const *w_rows, double *U)
  {
    if (n_local < 1 || n_local > kMaxN || N < n_local || N > kMaxGain || !states || !sum || !w_rows || !U ||
        stride < n_state || n_params < 0 || (n_params > 0 && !params))
      throw Error(ADM_ERR_INVALID, "invalid partial-update arguments (at most 64 local members)");
    ADM_CK(cudaSetDevice(device));
    int64_t const rows = n_state + n_params;
    size_t const smem = sizeof(double) * (size_t)n_local * N;
    ADM_CK(cudaFuncSetAttribute(partial_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    partial_update_kernel<<<(unsigned)((rows + 255) / 256), 256, smem, stream>>>(
        states, stride, n_local, N, n_state, params, n_params, sum, w_rows, U);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaStreamSynchronize(stream));
  }

  void apply(int n_local, double *states, int64_t stride, int64_t n_state, double *params, int n_params,
             double const *U, uint8_t const *mask)
  {
    if (n_local < 1 || !states || !U || stride < n_state || n_params < 0 || (n_params > 0 && !params))
      throw Error(ADM_ERR_INVALID, "invalid apply arguments");
    ADM_CK(cudaSetDevice(device));
    int64_t const total = (int64_t)n_local * (n_state + n_params);
    apply_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(states, stride, n_local, n_state, params,
                                                                     n_params, U, mask);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaStreamSynchronize(stream));
  }

  // C = HA HA^T scale + R and its Cholesky factor (lower, in place)
  void factor(int N, int m, double scale, double const *var, double const *cov)
  {
    int const t32 = (m + 31) / 32;
    cov_kernel<<<dim3(t32, t32), 256, 0, stream>>>(HA.p, N, m, scale, var, cov, C.p);
    ADM_CK(cudaGetLastError());
    for (int k0 = 0; k0 < m; k0 += kNB)
    {
      potrf_diag_kernel<<<1, 256, 0, stream>>>(C.p, m, k0, err.p);
      int const below = m - k0 - kNB;
      if (below > 0)
      {
        trsm_panel_kernel<<<(below + 127) / 128, 128, 0, stream>>>(C.p, m, k0);
        int const t = (below + 63) / 64;
        syrk_update_kernel<<<dim3(t, t), 256, 0, stream>>>(C.p, m, k0);
      }
      ADM_CK(cudaGetLastError());
    }
  }

  // Z = C^-1 D, W = HA^T Z scale
  void solve_and_w(int N, int m, double scale, double *Wout)
  {
    size_t const smem = (size_t)m * sizeof(double);
    ADM_CK(cudaFuncSetAttribute(solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    solve_kernel<<<N, 256, smem, stream>>>(C.p, m, D.p, Z.p);
    ADM_CK(cudaGetLastError());
    w_kernel<<<(N * N * 32 + 255) / 256, 256, 0, stream>>>(HA.p, Z.p, N, m, scale, Wout);
    ADM_CK(cudaGetLastError());
  }
};

} // namespace adm

extern "C" {

int adm_enkf_create(int device, void *stream, adm_enkf **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(out, "null argument");
    *out = nullptr;
    auto *e = new adm::Enkf;
    e->device = device;
    e->stream = reinterpret_cast<cudaStream_t>(stream);
    *out = reinterpret_cast<adm_enkf *>(e);
  });
}

int adm_enkf_destroy(adm_enkf *e)
{
  return adm::guard([&] { delete reinterpret_cast<adm::Enkf *>(e); });
}

int adm_enkf_analysis(adm_enkf *e, int32_t n_members, double *states, int64_t stride, int64_t n_state,
                      double *params, int32_t n_params, int32_t n_obs, int64_t const *obs_index,
                      double const *obs, double const *obs_var, double const *obs_cov,
                      double const *perturbations, uint8_t const *update_mask)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    reinterpret_cast<adm::Enkf *>(e)->analysis(n_members, states, stride, n_state, params, n_params, n_obs,
                                               obs_index, obs, obs_var, obs_cov, perturbations, update_mask);
  });
}

int adm_enkf_observe(adm_enkf *e, int32_t n_members, double const *states, int64_t stride, int64_t n_state,
                     int32_t n_obs, int64_t const *obs_index, double *hx)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    reinterpret_cast<adm::Enkf *>(e)->observe(n_members, states, stride, n_state, n_obs, obs_index, hx);
  });
}

int adm_enkf_gain(adm_enkf *e, int32_t n_members, int32_t n_obs, double const *hx, double const *obs,
                  double const *obs_var, double const *obs_cov, double const *perturbations, double *w)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    reinterpret_cast<adm::Enkf *>(e)->gain(n_members, n_obs, hx, obs, obs_var, obs_cov, perturbations, w);
  });
}

int adm_enkf_local_sum(adm_enkf *e, int32_t n_local, double const *states, int64_t stride, int64_t n_state,
                       double const *params, int32_t n_params, double *sum)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    reinterpret_cast<adm::Enkf *>(e)->local_sum(n_local, states, stride, n_state, params, n_params, sum);
  });
}

int adm_enkf_partial_update(adm_enkf *e, int32_t n_local, int32_t n_members, double const *states, int64_t stride,
                            int64_t n_state, double const *params, int32_t n_params, double const *sum,
                            double const *w_rows, double *u)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    reinterpret_cast<adm::Enkf *>(e)->partial_update(n_local, n_members, states, stride, n_state, params, n_params,
                                                     sum, w_rows, u);
  });
}

int adm_enkf_apply(adm_enkf *e, int32_t n_local, double *states, int64_t stride, int64_t n_state, double *params,
                   int32_t n_params, double const *u, uint8_t const *update_mask)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    reinterpret_cast<adm::Enkf *>(e)->apply(n_local, states, stride, n_state, params, n_params, u, update_mask);
  });
}

} // extern "C"
