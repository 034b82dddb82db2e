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
//
// With a diagonal R and no localization the m x m system is not formed at
// all: by the Sherman-Morrison-Woodbury identity
//   HA^T (HA HA^T / (N-1) + R)^-1 / (N-1) = ((N-1) I + G)^-1 HA^T R^-1,
//   G = HA^T R^-1 HA   (N x N),
// so W = ((N-1) I + G)^-1 E with E = HA^T R^-1 D: two N x N Gram products
// over the observations and one N x N Cholesky (the ensemble-space form of
// the same update). A non-positive variance takes the m x m path, which
// reports the indefinite C as before.
//
// With localization (the reference's sparsity pattern of pairs within the
// cutoff and its cutoff function) P is no longer A A^T / (N - 1): the
// observation block C is scaled entry by entry, the parameter rows keep
// x_k += A_p W[:, k], and each state row i takes
//   x_k[i] += sum_{j near i} rho_ij g_ij Z_k[j],
//   g_ij = sum_l A_l[i] HA_l[j] / (N - 1),
// over the observations j within the cutoff of node i, found through a
// uniform grid of observation buckets (no P, no n x m matrix).
#include "capi_common.hpp"
#include "../../include/adamantine_b200_ensemble.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace adm
{
namespace
{
constexpr int kNB = 64;        // Cholesky block size
constexpr size_t kPotrfSmem = sizeof(double) * 2 * kNB * (kNB + 1); // potrf_diag_kernel
constexpr size_t kPanelSmem = sizeof(double) * 2 * kNB * (kNB + 1); // trsm_panel_kernel
constexpr int kMaxN = 64;      // members per analysis
constexpr int kMaxObs = 16384; // observations (the solve keeps one column in shared memory)
constexpr int kMaxGain = 256;  // members of a sharded analysis (all GPUs)

enum EnkfError
{
  EERR_NONE = 0,
  EERR_NOT_SPD = 1,   // a Cholesky pivot was not positive and finite
  EERR_BAD_INDEX = 2, // an observation index outside [0, n_state)
  EERR_SINGULAR = 3   // an LU pivot was zero or not finite
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

// Geometry of a localized analysis: state entry i = a + pitch (b + nn1 c)
// sits at origin + (a, b, c) spacing; the observations are sorted into
// nb[0] x nb[1] x nb[2] buckets of size bsize from bmin.
struct LocGeom
{
  int function = ADM_LOC_NONE;
  double cutoff = 0.0, cutoff2 = 0.0;
  double origin[3] = {0, 0, 0}, spacing[3] = {0, 0, 0};
  int64_t nn[3] = {0, 0, 0}, pitch = 0;
  double bmin[3] = {0, 0, 0}, bsize[3] = {1, 1, 1};
  double bmax[3] = {0, 0, 0}; // the observation points' extent (with bmin)
  int nb[3] = {1, 1, 1};
};

// Scaling of a covariance entry between support points at squared distance
// d2: 0 outside the cutoff sphere (the sparsity pattern), else 1 or the
// Gaspari-Cohn correlation (Gaspari and Cohn 1999, eq. 4.10) of
// r = 2 d / cutoff, as gaspari_cohn_function (DataAssimilator.cc:672-688).
__device__ __forceinline__ double loc_weight(LocGeom const &g, double d2)
{
  if (!(d2 <= g.cutoff2))
    return 0.0;
  if (g.function != ADM_LOC_GASPARI_COHN)
    return 1.0;
  double const r = 2.0 * sqrt(d2) / g.cutoff;
  if (r < 1.0)
    return 1.0 + r * r * (-5.0 / 3.0 + r * (5.0 / 8.0 + r * (0.5 - 0.25 * r)));
  if (r < 2.0)
    return 4.0 - 5.0 * r + r * r * (5.0 / 3.0 + r * (5.0 / 8.0 + r * (-0.5 + r / 12.0))) - 2.0 / (3.0 * r);
  return 0.0;
}

// Lower triangle of C = HA^T HA * scale + R (R diagonal var, or dense cov);
// with oxyz (observation support points) the HA^T HA part is localized.
// 32 x 32 output tile per block, 256 threads, 4 outputs per thread.
__global__ void __launch_bounds__(256) cov_kernel(double const *HA, int n_members, int m, double scale,
                                                  double const *var, double const *cov, double *C,
                                                  double const *oxyz, LocGeom g, int full)
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
    if (oxyz)
    {
      double const dx = oxyz[3 * gi] - oxyz[3 * gj], dy = oxyz[3 * gi + 1] - oxyz[3 * gj + 1],
                   dz = oxyz[3 * gi + 2] - oxyz[3 * gj + 2];
      v *= loc_weight(g, dx * dx + dy * dy + dz * dz);
    }
    if (cov)
      v += cov[(int64_t)gi * m + gj];
    else if (gi == gj)
      v += var[gi];
    C[(int64_t)gi * m + gj] = v;
    if (full && gj != gi)
    {
      double u = acc[c] * scale;
      if (oxyz)
      {
        double const dx = oxyz[3 * gi] - oxyz[3 * gj], dy = oxyz[3 * gi + 1] - oxyz[3 * gj + 1],
                     dz = oxyz[3 * gi + 2] - oxyz[3 * gj + 2];
        u *= loc_weight(g, dx * dx + dy * dy + dz * dz);
      }
      if (cov)
        u += cov[(int64_t)gj * m + gi];
      C[(int64_t)gj * m + gi] = u;
    }
  }
}

// acc[u][v] = sum_q A[r + u][q] B[q][c + 16 v] over the kNB columns of A,
// with r = 4 (tid / 16), c = tid % 16: a 64 x 64 product, 4 x 4 outputs per
// thread of 256 (B row-major with leading dimension ldb >= 64; consecutive
// threads read consecutive entries of B, two rows of A per warp). With
// upper = true, A is upper triangular and the sum starts at q = r.
template <bool upper = false>
__device__ __forceinline__ void mm64(double const (*A)[kNB + 1], double const *B, int ldb, double acc[4][4])
{
  int const r = 4 * (threadIdx.x >> 4), c = threadIdx.x & 15;
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
      acc[u][v] = 0.0;
#pragma unroll 4
  for (int q = upper ? r : 0; q < kNB; ++q)
  {
    double x[4], y[4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
      x[u] = A[r + u][q];
#pragma unroll
    for (int v = 0; v < 4; ++v)
      y[v] = B[q * ldb + c + 16 * v];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v)
        acc[u][v] = fma(x[u], y[v], acc[u][v]);
  }
}

// Unblocked Cholesky of the diagonal block at (k0, k0), one CTA; the
// inverse of the factor goes to Linv (kNB x kNB, row-major, zero above the
// diagonal and beyond the block), for the panel solve and the triangular
// solves (products instead of substitutions). Each thread keeps a 4 x 4
// set of the block's entries in registers, (ty + 16 u, tx + 16 v); one
// barrier per column: step j reads column j (published by its owners into
// col[j & 1]), writes column j of the factor into l and updates the
// trailing triangle with a[i][c] -= (a[i][j] / sqrt(a[j][j]))
// (a[c][j] / sqrt(a[j][j])), after which the owners of column j + 1 publish
// it; the same step forms row j - 1 of the inverse, whose inputs (rows < j
// of l and of the inverse) are complete after the previous barrier:
// xi[i][c] = (delta_ic - sum_{q=c}^{i-1} l[i][q] xi[q][c]) / l[i][i]
// (four threads per column, a fixed 16-term predicated sum each).
// Dynamic shared memory kPotrfSmem: l and xi, kNB x (kNB + 1) each.
__global__ void __launch_bounds__(256) potrf_diag_kernel(double *C, int m, int k0, int *err, double *Linv)
{
  extern __shared__ double pd_sm[];
  double(*l)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(pd_sm);
  double(*xi)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(pd_sm + kNB * (kNB + 1));
  __shared__ double col[2][kNB];
  __shared__ double rdiag[kNB];
  int const nb = min(kNB, m - k0);
  int const tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  double a[4][4];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
    {
      int const r = ty + 16 * u, c = tx + 16 * v;
      a[u][v] = (r < nb && c <= r) ? C[(int64_t)(k0 + r) * m + k0 + c] : 0.0;
    }
  for (int e = tid; e < kNB * kNB; e += blockDim.x)
  {
    l[e / kNB][e % kNB] = 0.0;
    xi[e / kNB][e % kNB] = 0.0;
  }
  if (tx == 0)
#pragma unroll
    for (int u = 0; u < 4; ++u)
      col[0][ty + 16 * u] = a[u][0];
  __syncthreads();
  int const icol = tid >> 2, part = tid & 3; // inverse: four threads per column
  for (int j = 0; j <= nb; ++j)
  {
    if (j < nb)
    {
      double const *cb = col[j & 1];
      double d = cb[j];
      if (!(d > 0.0) || !isfinite(d))
      {
        if (tid == 0)
          atomicCAS(err, 0, (int)EERR_NOT_SPD);
        d = 1.0;
      }
      double const sd = sqrt(d), rs = 1.0 / sd;
      if (tid < nb - j)
        l[j + tid][j] = tid == 0 ? sd : cb[j + tid] * rs;
      if (tid == 0)
        rdiag[j] = rs;
      double li[4], lc[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
      {
        li[u] = cb[ty + 16 * u] * rs;
        lc[u] = cb[tx + 16 * u] * rs;
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v)
        {
          int const i = ty + 16 * u, c = tx + 16 * v;
          if (c > j && c <= i)
            a[u][v] -= li[u] * lc[v];
        }
      int const jn = j + 1;
#pragma unroll
      for (int v = 0; v < 4; ++v)
        if (jn < nb && tx + 16 * v == jn)
#pragma unroll
          for (int u = 0; u < 4; ++u)
            col[jn & 1][ty + 16 * u] = a[u][v];
    }
    if (j >= 1)
    {
      int const i = j - 1;
      double s = 0.0;
#pragma unroll
      for (int k = 0; k < kNB / 4; ++k)
      {
        int const q = part + 4 * k;
        if (q >= icol && q < i)
          s = fma(l[i][q], xi[q][icol], s);
      }
      s += __shfl_xor_sync(0xffffffffu, s, 1);
      s += __shfl_xor_sync(0xffffffffu, s, 2);
      if (part == 0 && icol <= i)
        xi[i][icol] = ((i == icol ? 1.0 : 0.0) - s) * rdiag[i];
    }
    __syncthreads();
  }
  for (int e = tid; e < kNB * kNB; e += blockDim.x)
  {
    int const r = e / kNB, c = e % kNB;
    if (r < nb && c <= r)
      C[(int64_t)(k0 + r) * m + k0 + c] = l[r][c];
    Linv[e] = xi[r][c];
  }
}

// Panel below the diagonal block: L[r, k0:k0+nb] = C[r, k0:k0+nb] L_kk^-T
// = rows * Linv^T, 64 rows per CTA as one 64 x 64 x 64 product (no
// substitution chain). With right-hand sides R (m x N, row-major), the
// CTAs after the row CTAs also take the forward solve's block step, 64
// columns each: R[k0 .. k0+nb] = Linv R[k0 .. k0+nb] in place (those rows
// are final once the earlier steps' trailing updates have run). Dynamic
// shared memory kPanelSmem: two kNB x (kNB + 1) tiles.
__global__ void __launch_bounds__(256) trsm_panel_kernel(double *C, int m, int k0, double const *Linv, double *R,
                                                         int N)
{
  extern __shared__ double tp_sm[];
  double(*v)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(tp_sm);
  double(*lb)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(tp_sm + kNB * (kNB + 1));
  int const nb = min(kNB, m - k0);
  int const n_row = (m - k0 - nb + kNB - 1) / kNB;
  int const tid = threadIdx.x;
  int const rr = 4 * (tid >> 4), cc = tid & 15;
  double acc[4][4];
  if ((int)blockIdx.x >= n_row)
  {
    int const n0 = 64 * ((int)blockIdx.x - n_row), nc = min(64, N - n0);
    for (int e = tid; e < kNB * kNB; e += blockDim.x)
    {
      int const q = e / kNB, n = e % kNB;
      v[q][n] = Linv[e];
      lb[q][n] = (q < nb && n < nc) ? R[(int64_t)(k0 + q) * N + n0 + n] : 0.0;
    }
    __syncthreads();
    mm64(v, &lb[0][0], kNB + 1, acc);
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int w = 0; w < 4; ++w)
      {
        int const q = rr + u, n = cc + 16 * w;
        if (q < nb && n < nc)
          R[(int64_t)(k0 + q) * N + n0 + n] = acc[u][w];
      }
    return;
  }
  int const r0 = k0 + nb + kNB * (int)blockIdx.x, nr = min(kNB, m - r0);
  for (int e = tid; e < kNB * kNB; e += blockDim.x)
  {
    int const r = e / kNB, q = e % kNB;
    v[r][q] = (r < nr && q < nb) ? C[(int64_t)(r0 + r) * m + k0 + q] : 0.0;
    lb[q][r] = Linv[e]; // lb[q][j] = Linv[j][q]
  }
  __syncthreads();
  mm64(v, &lb[0][0], kNB + 1, acc);
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int w = 0; w < 4; ++w)
    {
      int const r = rr + u, c = cc + 16 * w;
      if (r < nr && c < nb)
        C[(int64_t)(r0 + r) * m + k0 + c] = acc[u][w];
    }
}

// Trailing update of the lower triangle: C[i][j] -= L[i, panel] L[j, panel]^T
// for 64 x 64 tiles right of / below the panel (blockIdx.x < t, the tile
// columns). With right-hand sides R (m x N), the CTAs with blockIdx.x >= t
// take the forward solve's update of the rows below the block, 64 columns
// each: R[i][n] -= L[i, panel] Y[panel][n], Y being R's block rows after
// the panel kernel.
__global__ void __launch_bounds__(256) syrk_update_kernel(double *C, int m, int k0, double *R, int N)
{
  int const base = k0 + kNB;
  int const t = (m - base + 63) / 64;
  int const bi = blockIdx.y, bj = blockIdx.x;
  bool const aug = bj >= t;
  if (!aug && bj > bi)
    return;
  int const i0 = base + bi * 64, j0 = aug ? 64 * (bj - t) : base + bj * 64;
  // the panel's 64 columns in two chunks of 32 (static shared memory)
  __shared__ double pi[64][33], pj[64][33];
  int const tid = threadIdx.x;
  // rows tr + u, columns tc + 16 v (consecutive threads read consecutive
  // rows of pj: no bank conflicts at the 33-double pitch)
  int const tr = (tid / 16) * 4, tc = tid % 16;
  double acc[4][4] = {};
  for (int q0 = 0; q0 < kNB; q0 += 32)
  {
    for (int e = tid; e < 64 * 32; e += 256)
    {
      int const r = e / 32, c = e % 32;
      pi[r][c] = i0 + r < m ? C[(int64_t)(i0 + r) * m + k0 + q0 + c] : 0.0;
      if (aug)
      {
        int const n = e % 64, q = e / 64; // consecutive threads: consecutive columns of R
        pj[n][q] = j0 + n < N ? R[(int64_t)(k0 + q0 + q) * N + j0 + n] : 0.0;
      }
      else
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
        b[u] = pj[tc + 16 * u][q];
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
      int const gi = i0 + tr + u, gj = j0 + tc + 16 * v;
      if (aug)
      {
        if (gi < m && gj < N)
          R[(int64_t)gi * N + gj] -= acc[u][v];
      }
      else if (gi < m && gj <= gi)
        C[(int64_t)gi * m + gj] -= acc[u][v];
    }
}

// One block step of the backward solve L^T Z = Y for N right-hand sides
// (R and Z are m x N, row-major; R holds the forward solution Y, which the
// factorization carried along), 64 of them per blockIdx.y. Every CTA forms
// the block's solution z = Linv^T r_b from the inverse of the factor's
// diagonal block (r_b: rows k0 .. k0 + nb of R, final for this step); CTA
// 0 stores it in Z; then each CTA updates its 64-row chunk of the rows
// above, R[r] -= L[b, r]^T z. Both are 64 x 64 x 64 products (mm64; zero
// padding beyond nb, N and the chunk). Dynamic shared memory kTrsmSmem:
// r_b and z (kNB x 64 each) and one kNB x (kNB + 1) tile, first Linv^T,
// then the tile of L.
constexpr size_t kTrsmSmem = sizeof(double) * (2 * (size_t)kNB * 64 + (size_t)kNB * (kNB + 1));

__global__ void __launch_bounds__(256) trsm_back_kernel(double const *L, double const *Linv_b, int m, int N, int k0,
                                                        double *R, double *Z)
{
  extern __shared__ double ts_sm[];
  double *const rb = ts_sm;            // [kNB][64]
  double *const zb = ts_sm + kNB * 64; // [kNB][64]
  double(*lt)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(ts_sm + 2 * kNB * 64);
  int const nb = min(kNB, m - k0);
  int const n0 = 64 * (int)blockIdx.y, nc = min(64, N - n0); // the CTA's columns
  int const tid = threadIdx.x;
  int const rr = 4 * (tid >> 4), cc = tid & 15;
  for (int e = tid; e < kNB * 64; e += blockDim.x)
  {
    int const q = e / 64, n = e % 64;
    rb[e] = (q < nb && n < nc) ? R[(int64_t)(k0 + q) * N + n0 + n] : 0.0;
    lt[e % kNB][e / kNB] = Linv_b[e];
  }
  __syncthreads();
  double acc[4][4];
  mm64<true>(lt, rb, 64, acc); // Linv^T is upper triangular
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int w = 0; w < 4; ++w)
      zb[(rr + u) * 64 + cc + 16 * w] = acc[u][w];
  __syncthreads();
  if (blockIdx.x == 0)
    for (int e = tid; e < nb * nc; e += blockDim.x)
      Z[(int64_t)(k0 + e / nc) * N + n0 + e % nc] = zb[(e / nc) * 64 + e % nc];
  // the CTA's rows, above the block
  int const r0 = kNB * (int)blockIdx.x, nr = min(k0, r0 + kNB) - r0;
  if (nr <= 0)
    return;
  // the tile: lt[r][q] = L[k0 + q][r0 + r]
  for (int e = tid; e < kNB * kNB; e += blockDim.x)
  {
    int const q = e / kNB, r = e % kNB;
    lt[r][q] = (r < nr && q < nb) ? L[(int64_t)(k0 + q) * m + r0 + r] : 0.0;
  }
  __syncthreads();
  mm64(lt, zb, 64, acc);
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int w = 0; w < 4; ++w)
    {
      int const r = rr + u, n = cc + 16 * w;
      if (r < nr && n < nc)
        R[(int64_t)(r0 + r) * N + n0 + n] -= acc[u][w];
    }
}

// ---- ensemble-space solve (diagonal R, no localization)

// G[a][b] = sum_j HA[a][j] HA[b][j] / var[j] (which 0) and
// E[a][b] = sum_j HA[a][j] D[b][j] / var[j] (which 1), one warp per entry;
// *bad_var is set when a variance is not positive and finite.
__global__ void ens_gram_kernel(double const *HA, double const *D, double const *var, int n_members, int m,
                                double *G, double *E, int *bad_var)
{
  int const gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int const nn = n_members * n_members;
  if (gw >= 2 * nn)
    return;
  int const which = gw / nn, a = (gw % nn) / n_members, b = gw % n_members;
  double const *x = which == 0 ? HA : D;
  double s = 0.0;
  bool bad = false;
  for (int j = lane; j < m; j += 32)
  {
    double const v = var[j];
    bad |= !(v > 0.0) || !isfinite(v);
    s += HA[(int64_t)a * m + j] * x[(int64_t)b * m + j] / v;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_xor_sync(0xffffffffu, s, o);
  if (__any_sync(0xffffffffu, bad) && lane == 0)
    atomicExch(bad_var, 1);
  if (lane == 0)
    (which == 0 ? G : E)[a * n_members + b] = s;
}

// W = ((N-1) I + G)^-1 E for N <= kMaxN, one CTA: Cholesky of the N x N
// matrix in shared memory (the update of a column step forms the scaled
// entries it needs, so the column is scaled after it), then one right-hand
// side (column of E) per thread, forward and backward.
__global__ void __launch_bounds__(256) ens_solve_kernel(double const *G, double const *E, int n, double *W,
                                                        int *err)
{
  extern __shared__ double ens_sm[]; // M [n][n + 1], then X [n][n + 1]
  int const ld = n + 1;
  double *const Mp = ens_sm, *const Xp = ens_sm + n * ld;
#define M(a, b) Mp[(a) * ld + (b)]
#define X(a, b) Xp[(a) * ld + (b)]
  int const tid = threadIdx.x;
  for (int e = tid; e < n * n; e += blockDim.x)
  {
    int const a = e / n, b = e % n;
    M(a, b) = G[e] + (a == b ? (double)(n - 1) : 0.0);
    X(a, b) = E[e];
  }
  __syncthreads();
  // right-looking Cholesky of the lower triangle
  for (int j = 0; j < n; ++j)
  {
    double const d = M(j, j);
    bool const ok = d > 0.0 && isfinite(d);
    if (!ok && tid == 0)
      atomicCAS(err, 0, (int)EERR_NOT_SPD);
    double const r = ok ? sqrt(d) : 1.0;
    int const w = n - j - 1;
    __syncthreads(); // everyone has read M(j, j) and column j
    for (int e = tid; e < w * w; e += blockDim.x)
    {
      int const i = j + 1 + e / w, l = j + 1 + e % w;
      if (l <= i)
        M(i, l) -= (M(i, j) / r) * (M(l, j) / r);
    }
    __syncthreads();
    if (tid == 0)
      M(j, j) = r;
    for (int i = j + 1 + tid; i < n; i += blockDim.x)
      M(i, j) /= r;
    __syncthreads();
  }
  // one column of X per thread: L y = e, L^T x = y
  if (tid < n)
  {
    int const b = tid;
    for (int i = 0; i < n; ++i)
    {
      double s = X(i, b);
      for (int q = 0; q < i; ++q)
        s -= M(i, q) * X(q, b);
      X(i, b) = s / M(i, i);
    }
    for (int i = n - 1; i >= 0; --i)
    {
      double s = X(i, b);
      for (int q = i + 1; q < n; ++q)
        s -= M(q, i) * X(q, b);
      X(i, b) = s / M(i, i);
    }
  }
  __syncthreads();
  for (int e = tid; e < n * n; e += blockDim.x)
    W[e] = X(e / n, e % n);
#undef M
#undef X
}

// ---- LU with partial pivoting (C = P^T L U, row-major, in place), for a
// localized H P H^T + R that need not be positive definite (a step-function
// Schur product is not a correlation; the reference solves it with GMRES).
// Right-looking, blocked by kNB: panel, row swaps, triangular solve of the
// block row, trailing update.

// Panel k0 .. k0 + nb - 1 over rows k0 .. m - 1, one CTA: per column the
// pivot (largest magnitude, first on ties), the swap inside the panel, the
// multipliers (kept in shared memory with the pivot row) and the rank-1
// update of the rest of the panel, one element per thread, which also finds
// the next column's pivot candidates. Dynamic shared memory: m - k0 + kNB
// doubles.
__global__ void __launch_bounds__(1024) lu_panel_kernel(double *C, int m, int k0, int *piv, int *err)
{
  extern __shared__ double lsm[]; // [m - k0] multipliers, then [kNB] pivot row
  double *const urow = lsm + (m - k0);
  __shared__ double red_v[32];
  __shared__ int red_i[32];
  __shared__ int s_piv;
  __shared__ double s_d;
  int const nb = min(kNB, m - k0);
  int const tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  // candidate of this thread for the first column
  double best = -1.0;
  int bidx = m;
  for (int i = k0 + tid; i < m; i += blockDim.x)
  {
    double const v = fabs(C[(int64_t)i * m + k0]);
    if (v > best)
    {
      best = v;
      bidx = i;
    }
  }
  for (int jj = 0; jj < nb; ++jj)
  {
    int const j = k0 + jj;
    // block argmax (ties: smaller row)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
    {
      double const ov = __shfl_xor_sync(0xffffffffu, best, o);
      int const oi = __shfl_xor_sync(0xffffffffu, bidx, o);
      if (ov > best || (ov == best && oi < bidx))
      {
        best = ov;
        bidx = oi;
      }
    }
    if (lane == 0)
    {
      red_v[warp] = best;
      red_i[warp] = bidx;
    }
    __syncthreads();
    if (tid == 0)
    {
      double bv = red_v[0];
      int bi = red_i[0];
      for (int w = 1; w < nw; ++w)
        if (red_v[w] > bv || (red_v[w] == bv && red_i[w] < bi))
        {
          bv = red_v[w];
          bi = red_i[w];
        }
      if (bi >= m || !(bv > 0.0) || !isfinite(bv))
      {
        atomicCAS(err, 0, (int)EERR_SINGULAR);
        bi = j;
      }
      piv[j] = bi;
      s_piv = bi;
    }
    __syncthreads();
    int const p = s_piv;
    int const w = nb - jj - 1;
    // swap rows j and p inside the panel; the pivot row's tail to shared
    for (int c = tid; c < nb; c += blockDim.x)
    {
      double const a = C[(int64_t)j * m + k0 + c], b = C[(int64_t)p * m + k0 + c];
      if (p != j)
      {
        C[(int64_t)j * m + k0 + c] = b;
        C[(int64_t)p * m + k0 + c] = a;
      }
      double const pj = p != j ? b : a; // the new row j
      if (c == jj)
        s_d = (fabs(pj) > 0.0 && isfinite(pj)) ? pj : 1.0; // a bad pivot was flagged above
      if (c > jj)
        urow[c - jj - 1] = pj;
    }
    __syncthreads();
    double const d = s_d;
    // multipliers
    for (int i = j + 1 + tid; i < m; i += blockDim.x)
    {
      double const l = C[(int64_t)i * m + j] / d;
      C[(int64_t)i * m + j] = l;
      lsm[i - k0] = l;
    }
    __syncthreads();
    // rank-1 update of the panel's remaining columns, one element per thread
    best = -1.0;
    bidx = m;
    if (w > 0)
    {
      int64_t const total = (int64_t)(m - j - 1) * w;
      for (int64_t e = tid; e < total; e += blockDim.x)
      {
        int const i = j + 1 + (int)(e / w), c = 1 + (int)(e % w);
        double *const a = C + (int64_t)i * m + j + c;
        double const v = fma(-lsm[i - k0], urow[c - 1], *a);
        *a = v;
        if (c == 1 && fabs(v) > best)
        {
          best = fabs(v);
          bidx = i;
        }
      }
    }
    __syncthreads();
  }
}

// The panel's row swaps applied to the columns outside it, one column per
// thread.
__global__ void lu_swap_kernel(double *C, int m, int k0, int const *piv)
{
  int const nb = min(kNB, m - k0);
  int const c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m || (c >= k0 && c < k0 + nb))
    return;
  for (int j = k0; j < k0 + nb; ++j)
  {
    int const p = piv[j];
    if (p != j)
    {
      double const t = C[(int64_t)j * m + c];
      C[(int64_t)j * m + c] = C[(int64_t)p * m + c];
      C[(int64_t)p * m + c] = t;
    }
  }
}

// Block row U12 = L11^-1 A12 (L11 unit lower), one column per thread.
__global__ void __launch_bounds__(128) lu_trsm_kernel(double *C, int m, int k0)
{
  __shared__ double l[kNB][kNB + 1];
  int const nb = min(kNB, m - k0);
  for (int e = threadIdx.x; e < nb * nb; e += blockDim.x)
  {
    int const r = e / nb, c = e % nb;
    l[r][c] = c < r ? C[(int64_t)(k0 + r) * m + k0 + c] : 0.0;
  }
  __syncthreads();
  int const c = k0 + nb + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= m)
    return;
  double x[kNB];
#pragma unroll
  for (int r = 0; r < kNB; ++r)
  {
    if (r < nb)
    {
      double s = C[(int64_t)(k0 + r) * m + c];
#pragma unroll
      for (int q = 0; q < r; ++q)
        s = fma(-l[r][q], x[q], s);
      x[r] = s;
      C[(int64_t)(k0 + r) * m + c] = s;
    }
  }
}

// Trailing update A22 -= L21 U12 on 64 x 64 tiles.
__global__ void __launch_bounds__(256) lu_update_kernel(double *C, int m, int k0)
{
  int const base = k0 + kNB;
  int const i0 = base + blockIdx.y * 64, j0 = base + blockIdx.x * 64;
  __shared__ double pa[64][33], pb[32][65];
  int const tid = threadIdx.x;
  int const tr = (tid / 16) * 4, tc = (tid % 16) * 4;
  double acc[4][4] = {};
  for (int q0 = 0; q0 < kNB; q0 += 32)
  {
    for (int e = tid; e < 64 * 32; e += 256)
    {
      int const r = e / 32, c = e % 32;
      pa[r][c] = i0 + r < m ? C[(int64_t)(i0 + r) * m + k0 + q0 + c] : 0.0;
      int const br = e / 64, bc = e % 64;
      pb[br][bc] = j0 + bc < m ? C[(int64_t)(k0 + q0 + br) * m + j0 + bc] : 0.0;
    }
    __syncthreads();
    for (int q = 0; q < 32; ++q)
    {
      double a[4], b[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
      {
        a[u] = pa[tr + u][q];
        b[u] = pb[q][tc + u];
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
      if (gi < m && gj < m)
        C[(int64_t)gi * m + gj] -= acc[u][v];
    }
}

// Z_k = C^-1 D_k from the LU factors, one member per CTA: the row swaps,
// forward L y = P d (unit diagonal), backward U z = y; blocked by kNB,
// the column in shared memory.
__global__ void __launch_bounds__(256) lu_solve_kernel(double const *LU, int const *piv, int m, double const *D,
                                                       double *Z)
{
  extern __shared__ double col[]; // [m]
  int const k = blockIdx.x;
  int const tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int i = tid; i < m; i += blockDim.x)
    col[i] = D[(int64_t)k * m + i];
  __syncthreads();
  if (tid == 0)
    for (int j = 0; j < m; ++j)
    {
      int const p = piv[j];
      if (p != j)
      {
        double const t = col[j];
        col[j] = col[p];
        col[p] = t;
      }
    }
  __syncthreads();
  int const nblk = (m + kNB - 1) / kNB;
  for (int b = 0; b < nblk; ++b)
  {
    int const k0 = b * kNB, nb = min(kNB, m - k0);
    if (warp == 0)
      for (int j = 0; j < nb; ++j)
      {
        double s = 0.0;
        for (int q = lane; q < j; q += 32)
          s += LU[(int64_t)(k0 + j) * m + k0 + q] * col[k0 + q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
          col[k0 + j] -= s;
        __syncwarp();
      }
    __syncthreads();
    for (int i = k0 + nb + tid; i < m; i += blockDim.x)
    {
      double const *row = LU + (int64_t)i * m + k0;
      double s = 0.0;
      for (int q = 0; q < nb; ++q)
        s += row[q] * col[k0 + q];
      col[i] -= s;
    }
    __syncthreads();
  }
  for (int b = nblk - 1; b >= 0; --b)
  {
    int const k0 = b * kNB, nb = min(kNB, m - k0);
    if (warp == 0)
      for (int j = nb - 1; j >= 0; --j)
      {
        double s = 0.0;
        for (int q = j + 1 + lane; q < nb; q += 32)
          s += LU[(int64_t)(k0 + j) * m + k0 + q] * col[k0 + q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
          col[k0 + j] = (col[k0 + j] - s) / LU[(int64_t)(k0 + j) * m + k0 + j];
        __syncwarp();
      }
    __syncthreads();
    for (int i = tid; i < k0; i += blockDim.x)
    {
      double const *row = LU + (int64_t)i * m + k0;
      double s = 0.0;
      for (int q = 0; q < nb; ++q)
        s += row[q] * col[k0 + q];
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
                                                             double *U, int64_t row0)
{
  extern __shared__ double w[]; // [n_local][n_members]
  for (int e = threadIdx.x; e < n_local * n_members; e += blockDim.x)
    w[e] = W[e];
  __syncthreads();
  int64_t const rows = n_state + n_params;
  int64_t const i = row0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
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

// out[j][k] = in[k][j] (m x N from N x m).
__global__ void transpose_kernel(double const *in, int n, int m, double *out)
{
  int64_t const e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)n * m)
    return;
  int const k = (int)(e % n);
  int64_t const j = e / n;
  out[e] = in[(int64_t)k * m + j];
}

// Localized update of the state rows, written as U[l][i] for the n_out
// members l (the rows of Z). Block: a 32 x 4 x 2 brick of nodes, one per
// thread; blockIdx.y: 32 output members. The n_k members seen here are
// members k0 .. k0 + n_k - 1 of HA; their anomalies about sum / n_mean
// (or, with sum NULL, about their own mean) stay in registers, and the
// block walks the observation buckets that meet its brick grown by the
// cutoff (one list for all threads, so HA^T / Z^T rows are broadcast
// loads).
template <int KMAX>
__global__ void __launch_bounds__(256) loc_state_kernel(LocGeom g, double const *states, int64_t stride, int n_k,
                                                        int k0, double const *sum, int n_mean, double const *HAt,
                                                        double const *Zt, int N, int n_out, double scale,
                                                        int const *bstart, int const *perm, double const *sxyz,
                                                        double *U, int64_t rows)
{
  int const tid = threadIdx.x;
  int64_t const nbx = (g.pitch + 31) / 32, nby = (g.nn[1] + 3) / 4;
  int64_t const blk = blockIdx.x;
  int64_t const a0 = (blk % nbx) * 32, b0 = ((blk / nbx) % nby) * 4, c0 = (blk / (nbx * nby)) * 2;
  int64_t const ia = a0 + (tid & 31), ib = b0 + ((tid >> 5) & 3), ic = c0 + (tid >> 7);
  // rows of the padded layout get a result (0 in the row padding); nodes
  // get the update
  bool const in_rows = ia < g.pitch && ib < g.nn[1] && ic < g.nn[2];
  bool const valid = in_rows && ia < g.nn[0];
  int64_t const i = ia + g.pitch * (ib + g.nn[1] * ic);
  double const px = g.origin[0] + (double)ia * g.spacing[0];
  double const py = g.origin[1] + (double)ib * g.spacing[1];
  double const pz = g.origin[2] + (double)ic * g.spacing[2];

  double a[KMAX];
  double mean = 0.0;
  if (valid)
  {
    if (sum)
      mean = sum[i] / n_mean;
    else
    {
      double s = 0.0;
      for (int k = 0; k < n_k; ++k)
        s += states[(int64_t)k * stride + i];
      mean = s / n_k;
    }
  }
#pragma unroll
  for (int k = 0; k < KMAX; ++k)
    a[k] = (valid && k < n_k) ? states[(int64_t)k * stride + i] - mean : 0.0;

  // buckets meeting the brick's box grown by the cutoff
  int q0[3], q1[3];
  {
    int64_t const hi_idx[3] = {min(a0 + 31, g.nn[0] - 1), min(b0 + 3, g.nn[1] - 1), min(c0 + 1, g.nn[2] - 1)};
    int64_t const lo_idx[3] = {a0, b0, c0};
    for (int d = 0; d < 3; ++d)
    {
      double const lo = g.origin[d] + (double)lo_idx[d] * g.spacing[d] - g.cutoff;
      double const hi = g.origin[d] + (double)hi_idx[d] * g.spacing[d] + g.cutoff;
      if (g.nb[d] == 1)
      {
        // one bucket along d: none of its points is within the cutoff of
        // the brick when the grown brick misses their extent (the margin
        // keeps the test on the safe side of rounding)
        double const margin = 1e-9 * g.cutoff;
        q0[d] = 0;
        q1[d] = (hi + margin < g.bmin[d] || lo - margin > g.bmax[d]) ? -1 : 0;
        continue;
      }
      double const f0 = floor((lo - g.bmin[d]) / g.bsize[d]), f1 = floor((hi - g.bmin[d]) / g.bsize[d]);
      q0[d] = (int)fmin(fmax(f0, 0.0), (double)g.nb[d]);
      q1[d] = (int)fmin(fmax(f1, -1.0), (double)(g.nb[d] - 1));
    }
  }
  int const l0 = blockIdx.y * 32;
  double acc[32];
#pragma unroll
  for (int l = 0; l < 32; ++l)
    acc[l] = 0.0;
  for (int qz = q0[2]; qz <= q1[2]; ++qz)
    for (int qy = q0[1]; qy <= q1[1]; ++qy)
      for (int qx = q0[0]; qx <= q1[0]; ++qx)
      {
        int const bucket = qx + g.nb[0] * (qy + g.nb[1] * qz);
        int const s1 = bstart[bucket + 1];
        for (int s = bstart[bucket]; s < s1; ++s)
        {
          double const dx = sxyz[3 * s] - px, dy = sxyz[3 * s + 1] - py, dz = sxyz[3 * s + 2] - pz;
          double const w = valid ? loc_weight(g, dx * dx + dy * dy + dz * dz) : 0.0;
          if (w == 0.0)
            continue;
          int64_t const j = perm[s];
          double const *ha = HAt + j * N + k0;
          double gk = 0.0;
#pragma unroll
          for (int k = 0; k < KMAX; ++k)
            if (k < n_k)
              gk = fma(a[k], ha[k], gk);
          double const f = w * scale * gk;
          double const *z = Zt + j * N + l0;
#pragma unroll
          for (int l = 0; l < 32; ++l)
            if (l0 + l < n_out)
              acc[l] = fma(f, z[l], acc[l]);
        }
      }
  if (!in_rows)
    return;
#pragma unroll
  for (int l = 0; l < 32; ++l)
    if (l0 + l < n_out)
      U[(int64_t)(l0 + l) * rows + i] = acc[l];
}

} // namespace

// Workspace of the analysis, grown on demand.
struct Enkf
{
  int device = 0;
  cudaStream_t stream = nullptr;
  DevBuf<double> HA, D, C, Z, W;
  DevBuf<double> Linv;   // inverses of the Cholesky factor's diagonal blocks
  DevBuf<double> Rt, Yt; // m x N: the right-hand sides (then the forward solution), Z
  DevBuf<int> err;
  // localization: geometry, observation points (input order and bucket
  // order), bucket offsets, and the transposed HA / Z and the update rows
  bool loc = false;
  int loc_m = 0;
  LocGeom lg;
  DevBuf<double> oxyz, sxyz, HAt, Zt, U, sumb;
  DevBuf<int> bstart, perm, piv;
  int gain_n = 0, gain_m = 0; // shape of the last gain (HA and Z kept)

  // a step-function (or "none") localized H P H^T + R may be indefinite:
  // LU with pivoting; otherwise (SPD) Cholesky
  bool use_lu() const { return loc && lg.function != ADM_LOC_GASPARI_COHN; }
  bool factored_lu = false; // the last factor of C was LU (else Cholesky)
  DevBuf<double> G, E;
  DevBuf<int> bad_var;

  // W by the ensemble-space form when R is diagonal, there is no
  // localization and N <= kMaxN; false (nothing decided) when a variance is
  // not positive, so that the m x m path runs. Raises on a bad index.
  bool woodbury_w(int N, int m, double const *var, double const *cov, double *Wout)
  {
    if (cov || loc || N > kMaxN)
      return false;
    G.alloc((size_t)N * N);
    E.alloc((size_t)N * N);
    bad_var.alloc(1);
    ADM_CK(cudaMemsetAsync(bad_var.p, 0, sizeof(int), stream));
    int const warps = 2 * N * N;
    ens_gram_kernel<<<(warps * 32 + 255) / 256, 256, 0, stream>>>(HA.p, D.p, var, N, m, G.p, E.p, bad_var.p);
    size_t const smem = sizeof(double) * 2 * (size_t)N * (N + 1);
    ADM_CK(cudaFuncSetAttribute(ens_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    ens_solve_kernel<<<1, 256, smem, stream>>>(G.p, E.p, N, Wout, err.p);
    ADM_CK(cudaGetLastError());
    int h[2] = {0, 0};
    ADM_CK(cudaMemcpyAsync(&h[0], err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    ADM_CK(cudaMemcpyAsync(&h[1], bad_var.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    ADM_CK(cudaStreamSynchronize(stream));
    if (h[0] == EERR_BAD_INDEX)
      raise_err(h[0]);
    if (h[1] || h[0] != 0)
    {
      ADM_CK(cudaMemsetAsync(err.p, 0, sizeof(int), stream));
      return false;
    }
    return true;
  }

  void set_localization(int function, double cutoff, int m, double const *xyz, double const *origin,
                        double const *spacing, int64_t const *nodes, int64_t pitch)
  {
    if (m == 0)
    {
      loc = false;
      loc_m = 0;
      return;
    }
    if (function < ADM_LOC_NONE || function > ADM_LOC_GASPARI_COHN)
      throw Error(ADM_ERR_INVALID, "unknown localization cutoff function");
    if (!(cutoff > 0.0))
      throw Error(ADM_ERR_INVALID, "the localization cutoff distance must be positive");
    if (m < 0 || m > kMaxObs || !xyz || !origin || !spacing || !nodes)
      throw Error(ADM_ERR_INVALID, "invalid localization arguments");
    for (int d = 0; d < 3; ++d)
      if (nodes[d] < 1 || !std::isfinite(origin[d]) || !std::isfinite(spacing[d]) || spacing[d] < 0.0)
        throw Error(ADM_ERR_INVALID, "invalid localization grid");
    if (pitch < nodes[0])
      throw Error(ADM_ERR_INVALID, "pitch must be at least nodes[0]");
    LocGeom g;
    g.function = function;
    g.cutoff = cutoff;
    g.cutoff2 = cutoff * cutoff;
    g.pitch = pitch;
    double omin[3], omax[3], lo[3], hi[3];
    for (int d = 0; d < 3; ++d)
    {
      g.origin[d] = origin[d];
      g.spacing[d] = spacing[d];
      g.nn[d] = nodes[d];
      omin[d] = omax[d] = xyz[d];
    }
    for (int j = 0; j < m; ++j)
      for (int d = 0; d < 3; ++d)
      {
        double const v = xyz[3 * j + d];
        if (!std::isfinite(v))
          throw Error(ADM_ERR_INVALID, "observation points must be finite");
        omin[d] = std::fmin(omin[d], v);
        omax[d] = std::fmax(omax[d], v);
      }
    double diag2 = 0.0;
    for (int d = 0; d < 3; ++d)
    {
      lo[d] = std::fmin(omin[d], origin[d]);
      hi[d] = std::fmax(omax[d], origin[d] + (double)(nodes[d] - 1) * spacing[d]);
      diag2 += (hi[d] - lo[d]) * (hi[d] - lo[d]);
    }
    bool const covers_all = cutoff * cutoff >= diag2;
    loc_m = m;
    if (covers_all && function != ADM_LOC_GASPARI_COHN)
    {
      loc = false; // every pair in the pattern, every weight 1
      return;
    }
    // buckets of at least the cutoff (at most 64 per axis over the points)
    int64_t nbt = 1;
    for (int d = 0; d < 3; ++d)
    {
      double const ext = omax[d] - omin[d];
      g.bmin[d] = omin[d];
      g.bmax[d] = omax[d];
      if (covers_all || ext <= 0.0)
      {
        g.nb[d] = 1;
        g.bsize[d] = 1.0;
      }
      else
      {
        g.bsize[d] = std::fmax(cutoff, ext / 64.0);
        g.nb[d] = (int)std::fmin(65.0, std::floor(ext / g.bsize[d]) + 1.0);
      }
      nbt *= g.nb[d];
    }
    std::vector<int> bucket(m), start(nbt + 1, 0), order(m);
    for (int j = 0; j < m; ++j)
    {
      int q[3];
      for (int d = 0; d < 3; ++d)
      {
        double const f = g.nb[d] == 1 ? 0.0 : std::floor((xyz[3 * j + d] - g.bmin[d]) / g.bsize[d]);
        q[d] = (int)std::fmin(std::fmax(f, 0.0), (double)(g.nb[d] - 1));
      }
      bucket[j] = q[0] + g.nb[0] * (q[1] + g.nb[1] * q[2]);
      ++start[bucket[j] + 1];
    }
    for (int64_t b = 0; b < nbt; ++b)
      start[b + 1] += start[b];
    std::vector<int> fill(start.begin(), start.end() - 1);
    std::vector<double> sorted(3 * (size_t)m);
    for (int j = 0; j < m; ++j)
    {
      int const s = fill[bucket[j]]++;
      order[s] = j;
      for (int d = 0; d < 3; ++d)
        sorted[3 * (size_t)s + d] = xyz[3 * j + d];
    }
    ADM_CK(cudaSetDevice(device));
    oxyz.alloc(3 * (size_t)m);
    sxyz.alloc(3 * (size_t)m);
    perm.alloc(m);
    bstart.alloc(nbt + 1);
    ADM_CK(cudaMemcpyAsync(oxyz.p, xyz, 3 * sizeof(double) * m, cudaMemcpyHostToDevice, stream));
    ADM_CK(cudaMemcpyAsync(sxyz.p, sorted.data(), 3 * sizeof(double) * m, cudaMemcpyHostToDevice, stream));
    ADM_CK(cudaMemcpyAsync(perm.p, order.data(), sizeof(int) * m, cudaMemcpyHostToDevice, stream));
    ADM_CK(cudaMemcpyAsync(bstart.p, start.data(), sizeof(int) * (nbt + 1), cudaMemcpyHostToDevice, stream));
    ADM_CK(cudaStreamSynchronize(stream));
    lg = g;
    loc = true;
  }

  void check_loc(int m, int64_t n_state) const
  {
    if (loc_m && m != loc_m)
      throw Error(ADM_ERR_INVALID, "the number of observations differs from the localization's");
    if (loc && n_state != lg.pitch * lg.nn[1] * lg.nn[2])
      throw Error(ADM_ERR_INVALID, "n_state differs from the localization grid (pitch * nodes[1] * nodes[2])");
  }

  // U[l][i] of the state rows from the localized gain (HA, Z of N members;
  // the n_k members seen start at k0), then nothing else
  void launch_loc_state(double const *states, int64_t stride, int n_k, int k0, double const *sum, int N, int m,
                        double *Uout, int64_t rows)
  {
    HAt.alloc((size_t)N * m);
    Zt.alloc((size_t)N * m);
    int64_t const nm = (int64_t)N * m;
    transpose_kernel<<<(unsigned)((nm + 255) / 256), 256, 0, stream>>>(HA.p, N, m, HAt.p);
    transpose_kernel<<<(unsigned)((nm + 255) / 256), 256, 0, stream>>>(Z.p, N, m, Zt.p);
    ADM_CK(cudaGetLastError());
    int64_t const nbx = (lg.pitch + 31) / 32, nby = (lg.nn[1] + 3) / 4, nbz = (lg.nn[2] + 1) / 2;
    dim3 const grid((unsigned)(nbx * nby * nbz), (unsigned)((N + 31) / 32));
    double const scale = 1.0 / (N - 1.0);
    if (n_k <= 32)
      loc_state_kernel<32><<<grid, 256, 0, stream>>>(lg, states, stride, n_k, k0, sum, N, HAt.p, Zt.p, N, N, scale,
                                                     bstart.p, perm.p, sxyz.p, Uout, rows);
    else
      loc_state_kernel<64><<<grid, 256, 0, stream>>>(lg, states, stride, n_k, k0, sum, N, HAt.p, Zt.p, N, N, scale,
                                                     bstart.p, perm.p, sxyz.p, Uout, rows);
    ADM_CK(cudaGetLastError());
  }

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
    check_loc(m, n_state);
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
    // stops before touching the states if an index or a pivot was bad
    if (!woodbury_w(N, m, var, cov, W.p))
    {
      factor_checked(N, m, scale, var, cov);
      solve_and_w(N, m, scale, W.p);
    }
    int64_t const rows = n_state + n_params;
    if (!loc)
    {
      update_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(states, stride, N, n_state, params,
                                                                        n_params, mask, W.p);
      ADM_CK(cudaGetLastError());
    }
    else
    {
      // U = every member's update (parameter rows through W, state rows
      // localized), then x += U
      U.alloc((size_t)N * rows);
      sumb.alloc(rows);
      local_sum_kernel<<<(unsigned)((rows + 255) / 256), 256, 0, stream>>>(states, stride, N, n_state, params,
                                                                          n_params, sumb.p);
      ADM_CK(cudaGetLastError());
      if (n_params > 0)
      {
        size_t const smem = sizeof(double) * (size_t)N * N;
        ADM_CK(cudaFuncSetAttribute(partial_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        partial_update_kernel<<<(unsigned)((n_params + 255) / 256), 256, smem, stream>>>(
            states, stride, N, N, n_state, params, n_params, sumb.p, W.p, U.p, n_state);
        ADM_CK(cudaGetLastError());
      }
      launch_loc_state(states, stride, N, 0, sumb.p, N, m, U.p, rows);
      int64_t const total = (int64_t)N * rows;
      apply_kernel<<<(unsigned)((total + 255) / 256), 256, 0, stream>>>(states, stride, N, n_state, params,
                                                                       n_params, U.p, mask);
      ADM_CK(cudaGetLastError());
    }
    ADM_CK(cudaStreamSynchronize(stream));
  }

  // ---- building blocks of the sharded analysis (members split over GPUs)
  int read_err()
  {
    int h_err = 0;
    ADM_CK(cudaMemcpyAsync(&h_err, err.p, sizeof(int), cudaMemcpyDeviceToHost, stream));
    ADM_CK(cudaStreamSynchronize(stream));
    return h_err;
  }

  void check_err() { raise_err(read_err()); }

  // Cholesky of C; a localized C that may be indefinite (step function or
  // "none") and is found not positive definite is factored again by LU
  void factor_checked(int N, int m, double scale, double const *var, double const *cov)
  {
    factored_lu = false;
    factor(N, m, scale, var, cov);
    int e = read_err();
    if (e == EERR_NOT_SPD && use_lu())
    {
      ADM_CK(cudaMemsetAsync(err.p, 0, sizeof(int), stream));
      factor_lu(N, m, scale, var, cov);
      factored_lu = true;
      e = read_err();
    }
    raise_err(e);
  }

  static void raise_err(int h_err)
  {
    if (h_err == EERR_BAD_INDEX)
      throw Error(ADM_ERR_INVALID, "an observation index is outside [0, n_state)");
    if (h_err == EERR_NOT_SPD)
      throw Error(ADM_ERR_DEVICE, "H P H^T + R is not positive definite (Cholesky pivot <= 0)");
    if (h_err == EERR_SINGULAR)
      throw Error(ADM_ERR_DEVICE, "the localized H P H^T + R is singular (zero LU pivot)");
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
    if (loc_m && m != loc_m)
      throw Error(ADM_ERR_INVALID, "the number of observations differs from the localization's");
    gain_n = gain_m = 0;
    center_kernel<<<(m + 127) / 128, 128, 0, stream>>>(hx, N, m, obs, pert, HA.p, D.p);
    ADM_CK(cudaGetLastError());
    double const scale = 1.0 / (N - 1.0);
    if (!woodbury_w(N, m, var, cov, Wout))
    {
      factor_checked(N, m, scale, var, cov);
      solve_and_w(N, m, scale, Wout);
    }
    ADM_CK(cudaStreamSynchronize(stream));
    gain_n = N;
    gain_m = m;
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
        states, stride, n_local, N, n_state, params, n_params, sum, w_rows, U, 0);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaStreamSynchronize(stream));
  }

  void partial_update_localized(int n_local, int first, int N, double const *states, int64_t stride,
                                int64_t n_state, double const *params, int n_params, double const *sum,
                                double const *w_rows, double *Uout)
  {
    if (!loc)
    {
      partial_update(n_local, N, states, stride, n_state, params, n_params, sum, w_rows, Uout);
      return;
    }
    if (n_local < 1 || n_local > kMaxN || first < 0 || first + n_local > N || N > kMaxGain || !states || !sum ||
        !w_rows || !Uout || stride < n_state || n_params < 0 || (n_params > 0 && !params))
      throw Error(ADM_ERR_INVALID, "invalid partial-update arguments (at most 64 local members)");
    if (gain_n != N || gain_m != loc_m)
      throw Error(ADM_ERR_INVALID, "the localized partial update needs adm_enkf_gain of the same ensemble first");
    check_loc(gain_m, n_state);
    ADM_CK(cudaSetDevice(device));
    int64_t const rows = n_state + n_params;
    if (n_params > 0)
    {
      size_t const smem = sizeof(double) * (size_t)n_local * N;
      ADM_CK(cudaFuncSetAttribute(partial_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      partial_update_kernel<<<(unsigned)((n_params + 255) / 256), 256, smem, stream>>>(
          states, stride, n_local, N, n_state, params, n_params, sum, w_rows, Uout, n_state);
      ADM_CK(cudaGetLastError());
    }
    launch_loc_state(states, stride, n_local, first, sum, N, gain_m, Uout, rows);
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
  void factor_lu(int N, int m, double scale, double const *var, double const *cov)
  {
    int const t32 = (m + 31) / 32;
    cov_kernel<<<dim3(t32, t32), 256, 0, stream>>>(HA.p, N, m, scale, var, cov, C.p, loc ? oxyz.p : nullptr, lg, 1);
    ADM_CK(cudaGetLastError());
    {
      piv.alloc(m);
      size_t const psm = sizeof(double) * ((size_t)m + kNB);
      ADM_CK(cudaFuncSetAttribute(lu_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)psm));
      for (int k0 = 0; k0 < m; k0 += kNB)
      {
        lu_panel_kernel<<<1, 1024, sizeof(double) * ((size_t)(m - k0) + kNB), stream>>>(C.p, m, k0, piv.p, err.p);
        lu_swap_kernel<<<(m + 255) / 256, 256, 0, stream>>>(C.p, m, k0, piv.p);
        int const right = m - k0 - kNB;
        if (right > 0)
        {
          lu_trsm_kernel<<<(right + 127) / 128, 128, 0, stream>>>(C.p, m, k0);
          int const t = (right + 63) / 64;
          lu_update_kernel<<<dim3(t, t), 256, 0, stream>>>(C.p, m, k0);
        }
        ADM_CK(cudaGetLastError());
      }
    }
  }

  // Cholesky of C = HA^T HA scale (localized) + R by blocks of kNB, carrying
  // the forward solve L Y = D^T of the right-hand sides along (Rt, m x N):
  // the panel kernel takes each block's solve, the trailing update the
  // rows below.
  void factor(int N, int m, double scale, double const *var, double const *cov)
  {
    int const t32 = (m + 31) / 32;
    cov_kernel<<<dim3(t32, t32), 256, 0, stream>>>(HA.p, N, m, scale, var, cov, C.p, loc ? oxyz.p : nullptr, lg, 0);
    ADM_CK(cudaGetLastError());
    Rt.alloc((size_t)m * N);
    int64_t const nm = (int64_t)N * m;
    transpose_kernel<<<(unsigned)((nm + 255) / 256), 256, 0, stream>>>(D.p, N, m, Rt.p);
    ADM_CK(cudaGetLastError());
    Linv.alloc((size_t)((m + kNB - 1) / kNB) * kNB * kNB);
    ADM_CK(cudaFuncSetAttribute(potrf_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPotrfSmem));
    ADM_CK(cudaFuncSetAttribute(trsm_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmem));
    int const nchunk = (N + 63) / 64;
    for (int k0 = 0; k0 < m; k0 += kNB)
    {
      double *const li = Linv.p + (size_t)(k0 / kNB) * kNB * kNB;
      potrf_diag_kernel<<<1, 256, kPotrfSmem, stream>>>(C.p, m, k0, err.p, li);
      int const below = std::max(0, m - k0 - kNB);
      int const t = (below + 63) / 64;
      trsm_panel_kernel<<<t + nchunk, 256, kPanelSmem, stream>>>(C.p, m, k0, li, Rt.p, N);
      if (below > 0)
        syrk_update_kernel<<<dim3(t + nchunk, t), 256, 0, stream>>>(C.p, m, k0, Rt.p, N);
      ADM_CK(cudaGetLastError());
    }
  }

  // Z = C^-1 D, W = HA^T Z scale
  void solve_and_w(int N, int m, double scale, double *Wout)
  {
    if (factored_lu)
    {
      size_t const smem = (size_t)m * sizeof(double);
      ADM_CK(cudaFuncSetAttribute(lu_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      lu_solve_kernel<<<N, 256, smem, stream>>>(C.p, piv.p, m, D.p, Z.p);
    }
    else
    {
      // blocked backward solve of all N columns (m x N layout, 64 columns
      // per CTA) from the forward solution that the factorization left in Rt
      Yt.alloc((size_t)m * N);
      int64_t const nm = (int64_t)N * m;
      ADM_CK(cudaFuncSetAttribute(trsm_back_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
      int const nblk = (m + kNB - 1) / kNB;
      unsigned const nchunk = (unsigned)((N + 63) / 64);
      for (int b = nblk - 1; b >= 0; --b)
      {
        int const k0 = b * kNB;
        trsm_back_kernel<<<dim3(std::max(1, (k0 + kNB - 1) / kNB), nchunk), 256, kTrsmSmem, stream>>>(
            C.p, Linv.p + (size_t)b * kNB * kNB, m, N, k0, Rt.p, Yt.p);
      }
      ADM_CK(cudaGetLastError());
      // Yt holds Z (m x N)
      transpose_kernel<<<(unsigned)((nm + 255) / 256), 256, 0, stream>>>(Yt.p, m, N, Z.p);
    }
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

int adm_enkf_set_localization(adm_enkf *e, int32_t function, double cutoff, int32_t n_obs, double const *obs_xyz,
                              double const *origin, double const *spacing, int64_t const *nodes, int64_t pitch)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    reinterpret_cast<adm::Enkf *>(e)->set_localization(function, cutoff, n_obs, obs_xyz, origin, spacing, nodes,
                                                       pitch);
  });
}

int adm_enkf_partial_update_localized(adm_enkf *e, int32_t n_local, int32_t first_member, int32_t n_members,
                                      double const *states, int64_t stride, int64_t n_state, double const *params,
                                      int32_t n_params, double const *sum, double const *w_rows, double *u)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    reinterpret_cast<adm::Enkf *>(e)->partial_update_localized(n_local, first_member, n_members, states, stride,
                                                               n_state, params, n_params, sum, w_rows, u);
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
