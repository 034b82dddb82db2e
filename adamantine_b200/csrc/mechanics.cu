/* Thermoelastic displacement on the thermal mesh: the isotropic elasticity
 * operator of MechanicalOperator::assemble_matrix
 * (source/MechanicalOperator.cc:183-280), its right-hand side
 * (assemble_rhs, :283-486: thermal expansion and gravity), the cell
 * selection of MechanicalPhysics::setup_dofs (source/MechanicalPhysics.cc
 * :280-440: thermally active cells with a solid ratio above 0.99) and the
 * CG solve of MechanicalPhysics::solve (:488-520), matrix-free on the GPU;
 * then the J2 stress update of compute_stress (:542-634) at every Gauss
 * point, one thread per point.
 *
 * Layout: the thermal handle's node layout (pitch, z-slabs); a displacement
 * vector is three node vectors (x, y, z components). Work, FE_Q(2): one
 * warp per cell that carries displacement; the reference-element tables
 * (values and gradients of the (p+1)^3 nodal functions at the (p+1)^3
 * Gauss points) sit in a per-handle device buffer; each lane gathers one
 * node's three components, then evaluates one quadrature point's stress,
 * then integrates one node's three test functions and adds them into the
 * result (FP64 atomics: a node is shared by up to 8 cells). FE_Q(1): one
 * thread per node gathers its row from the element matrices of its cells
 * (elastic_gather_q1_kernel, no atomics). Clamped displacements are
 * eliminated: their columns are dropped and their rows are the identity.
 */
#include "capi_common.hpp"
#include "thermal.hpp"
#include "../../include/adamantine_b200_mechanics.h"

#include <algorithm>
#include <cmath>
#include <memory>
#include <vector>

namespace adm
{
namespace
{
constexpr int kMaxN = 27; // nodes (and quadrature points) of a Q2 cell
constexpr double kGravity = 9.80665; // GravityForce::g (source/BodyForce.hh:53)

// Reference-element tables of one handle, in that handle's device buffer
// (handles of different FE degrees coexist on a device): values
// [q][n] phi_n(x_q), gradients [q][n][d] d phi_n / d xi_d (x_q) and the
// reference weights of the Gauss points, at these offsets.
constexpr int kTabVal = 0;
constexpr int kTabGrad = kMaxN * kMaxN;
constexpr int kTabWq = kTabGrad + kMaxN * kMaxN * 3;
constexpr int kTabSize = kTabWq + kMaxN;

struct MechArgs
{
  int p, N; // degree, nodes (= quadrature points) per cell
  int nc[3], nn[3], pitch;
  int64_t m; // node vector length (component stride)
  double inv_h[3], jxw; // 1 / h and the cell volume (x the reference weight)
  int32_t const *cells; // cells that carry displacement
  int n_cells;
  uint8_t const *node_mask; // 0 none, 1 free, 2 clamped
  uint8_t const *matid;
  double lambda[4], mu[4], alpha[4], rho[4], tref[4];
  double tinit;
  int thermoelastic, gravity;
  uint8_t const *melted;
  double const *tab; // the handle's reference-element tables (kTab* offsets)
  double plastic_modulus[4], iso_hardening[4], elastic_limit[4];
  double const *cell_coef; // multigrid levels: (lambda, mu) per cell instead of per material, or null
};

// Lame parameters of cell c
__device__ __forceinline__ void cell_lame(MechArgs const &a, int c, double &lam, double &mu)
{
  if (a.cell_coef)
  {
    lam = a.cell_coef[2 * (int64_t)c];
    mu = a.cell_coef[2 * (int64_t)c + 1];
  }
  else
  {
    int const mat = a.matid[c];
    lam = a.lambda[mat];
    mu = a.mu[mat];
  }
}

__device__ __forceinline__ int64_t node_of(MechArgs const &a, int cx, int cy, int cz, int n)
{
  int const np = a.p + 1;
  int const i = n % np, j = (n / np) % np, k = n / (np * np);
  return (int64_t)(a.p * cx + i) + (int64_t)a.pitch * ((a.p * cy + j) + (int64_t)a.nn[1] * (a.p * cz + k));
}

// The stress state at the Gauss points: plastic internal variable [C N],
// stress and back stress [6][C N] (xx, yy, zz, xy, xz, yz), point q of cell
// c at c N + q.
struct J2State
{
  double *kappa, *stress, *back;
  int64_t cq; // C N
};

// A cell that starts carrying displacement: the elastic limit, zero stress
// and back stress at its points (MechanicalPhysics::setup_dofs,
// source/MechanicalPhysics.cc:366-378; the constructor, :76-98).
__global__ void j2_init_kernel(MechArgs a, J2State s, int32_t const *cells, int n)
{
  int64_t const t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)n * a.N)
    return;
  int const c = cells[t / a.N], q = (int)(t % a.N);
  int64_t const i = (int64_t)c * a.N + q;
  s.kappa[i] = a.elastic_limit[a.matid[c]];
  for (int k = 0; k < 6; ++k)
  {
    s.stress[k * s.cq + i] = 0.0;
    s.back[k * s.cq + i] = 0.0;
  }
}

// MechanicalPhysics::compute_stress (source/MechanicalPhysics.cc:542-634),
// one thread per Gauss point of a cell that carries displacement: the
// symmetric gradient of the displacement increment u - u_old (u_old NULL:
// none yet), the trial stress sigma + lambda tr(eps) I + 2 mu eps, and where
// |dev(sigma) - beta| reaches the plastic internal variable kappa the radial
// return with increment (|eta| - kappa) / (2 mu + H) along n = eta / |eta|:
// sigma -= 2 mu dgamma n, kappa += h H dgamma, beta += (1 - h) H^2 n (the
// reference's back-stress update, :626-630, as written there: H^2 n, not
// H dgamma n). |.| is the Frobenius norm (off-diagonal entries twice).
__global__ void __launch_bounds__(128) j2_stress_kernel(MechArgs a, J2State s, double const *u,
                                                        double const *u_old)
{
  int64_t const t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)a.n_cells * a.N)
    return;
  int const c = a.cells[t / a.N], q = (int)(t % a.N);
  int const cx = c % a.nc[0], cy = (c / a.nc[0]) % a.nc[1], cz = c / (a.nc[0] * a.nc[1]);
  int const mat = a.matid[c];
  double const lam = a.lambda[mat], mu = a.mu[mat];
  double G3[3][3] = {{0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}, {0.0, 0.0, 0.0}};
  for (int n = 0; n < a.N; ++n)
  {
    int64_t const g = node_of(a, cx, cy, cz, n);
    double const *gr = a.tab + kTabGrad + (q * kMaxN + n) * 3;
#pragma unroll
    for (int comp = 0; comp < 3; ++comp)
    {
      double const d = u[comp * a.m + g] - (u_old ? u_old[comp * a.m + g] : 0.0);
#pragma unroll
      for (int k = 0; k < 3; ++k)
        G3[comp][k] = fma(d, gr[k], G3[comp][k]);
    }
  }
#pragma unroll
  for (int comp = 0; comp < 3; ++comp)
#pragma unroll
    for (int k = 0; k < 3; ++k)
      G3[comp][k] *= a.inv_h[k];
  // strain (symmetric gradient), xx yy zz xy xz yz
  double const e[6] = {G3[0][0], G3[1][1], G3[2][2], 0.5 * (G3[0][1] + G3[1][0]), 0.5 * (G3[0][2] + G3[2][0]),
                       0.5 * (G3[1][2] + G3[2][1])};
  double const tr = e[0] + e[1] + e[2];
  int64_t const i = (int64_t)c * a.N + q;
  double sig[6], eta[6];
#pragma unroll
  for (int k = 0; k < 6; ++k)
    sig[k] = s.stress[k * s.cq + i] + ((k < 3 ? lam * tr : 0.0) + 2.0 * mu * e[k]);
  double const mean = (sig[0] + sig[1] + sig[2]) / 3.0;
  double nrm2 = 0.0;
#pragma unroll
  for (int k = 0; k < 6; ++k)
  {
    eta[k] = (k < 3 ? sig[k] - mean : sig[k]) - s.back[k * s.cq + i];
    nrm2 += (k < 3 ? 1.0 : 2.0) * eta[k] * eta[k];
  }
  double const nrm = sqrt(nrm2);
  double const kap = s.kappa[i];
  if (nrm < kap)
  {
#pragma unroll
    for (int k = 0; k < 6; ++k)
      s.stress[k * s.cq + i] = sig[k];
    return;
  }
  double const H = a.plastic_modulus[mat], h = a.iso_hardening[mat];
  double const dg = (nrm - kap) / (2.0 * mu + H);
#pragma unroll
  for (int k = 0; k < 6; ++k)
  {
    double const nk = eta[k] / nrm;
    s.stress[k * s.cq + i] = sig[k] - 2.0 * mu * dg * nk;
    s.back[k * s.cq + i] += (1.0 - h) * H * H * nk;
  }
  s.kappa[i] = kap + h * H * dg;
}

// The previous displacement after the cells that carry displacement changed
// (MechanicalPhysics::setup_dofs, source/MechanicalPhysics.cc:296-337 and
// :418-437): every cell that now carries displacement writes, in cell order,
// its saved values -- the old displacement if it carried displacement
// before, zeros if not -- so a node keeps its old value when the last such
// cell touching it carried displacement before, else gets 0 (0 as well at
// nodes of no such cell).
__global__ void old_displacement_transfer_kernel(MechArgs a, uint8_t const *carry_prev, uint8_t const *carry_now,
                                                 double *u_old)
{
  int64_t const g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= a.m)
    return;
  int const gx = (int)(g % a.pitch);
  int64_t const r = g / a.pitch;
  int const gy = (int)(r % a.nn[1]), gz = (int)(r / a.nn[1]);
  bool keep = false;
  if (gx < a.nn[0])
  {
    // the cells around the node, in increasing cell index: the last one that
    // carries displacement now decides
    int64_t last = -1;
    for (int dz = 1; dz >= 0; --dz)
      for (int dy = 1; dy >= 0; --dy)
        for (int dx = 1; dx >= 0; --dx)
        {
          // cell (cx, cy, cz) touches node (gx, gy, gz) when p cx <= gx <= p (cx + 1)
          int const cx = gx / a.p - dx, cy = gy / a.p - dy, cz = gz / a.p - dz;
          if (cx < 0 || cy < 0 || cz < 0 || cx >= a.nc[0] || cy >= a.nc[1] || cz >= a.nc[2])
            continue;
          if (gx > a.p * (cx + 1) || gy > a.p * (cy + 1) || gz > a.p * (cz + 1))
            continue;
          int64_t const c = cx + (int64_t)a.nc[0] * (cy + (int64_t)a.nc[1] * cz);
          if (carry_now[c] && c > last)
            last = c;
        }
    keep = last >= 0 && carry_prev[last];
  }
  for (int comp = 0; comp < 3; ++comp)
    if (!keep)
      u_old[comp * a.m + g] = 0.0;
}

// dst += A src on the free rows; 4 warps per block, 32 / N cells per warp
// (4 for FE_Q(1), 1 for FE_Q(2)), N lanes per cell.
__global__ void __launch_bounds__(128) elastic_apply_kernel(MechArgs a, double const *src, double *dst)
{
  __shared__ double u[4][3][32];
  __shared__ double S[4][32][9];
  // the gradient table in shared memory: the lanes of a warp read
  // different quadrature points' rows, which constant memory serializes
  __shared__ double grad_s[kMaxN * kMaxN * 3];
  for (int e = threadIdx.x; e < kMaxN * kMaxN * 3; e += blockDim.x)
    grad_s[e] = a.tab[kTabGrad + e];
  __syncthreads();
  int const w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int const G = 32 / a.N; // cells per warp
  int const g = lane / a.N, l = lane - g * a.N;
  bool const on = g < G;
  int const gw = blockIdx.x * 4 + w, nw = gridDim.x * 4;
  // every lane runs the same number of rounds (the warp syncs inside)
  int const rounds = (a.n_cells + nw * G - 1) / (nw * G);
  for (int rd = 0; rd < rounds; ++rd)
  {
    int const ci = (rd * nw + gw) * G + g;
    bool const act = on && ci < a.n_cells;
    int64_t gidx = 0;
    bool freen = false;
    double lam = 0.0, mu = 0.0;
    if (act)
    {
      int const c = a.cells[ci];
      int const cx = c % a.nc[0], cy = (c / a.nc[0]) % a.nc[1], cz = c / (a.nc[0] * a.nc[1]);
      cell_lame(a, c, lam, mu);
      gidx = node_of(a, cx, cy, cz, l);
      freen = a.node_mask[gidx] == 1;
      for (int comp = 0; comp < 3; ++comp)
        u[w][comp][g * a.N + l] = freen ? src[comp * a.m + gidx] : 0.0;
    }
    __syncwarp();
    if (act)
    {
      int const q = l;
      double const *uc = &u[w][0][g * a.N];
      double G3[3][3];
#pragma unroll
      for (int comp = 0; comp < 3; ++comp)
#pragma unroll
        for (int d = 0; d < 3; ++d)
        {
          double s = 0.0;
          for (int n = 0; n < a.N; ++n)
            s = fma(uc[comp * 32 + n], grad_s[(q * kMaxN + n) * 3 + d], s);
          G3[comp][d] = s * a.inv_h[d];
        }
      double const div = G3[0][0] + G3[1][1] + G3[2][2];
      double const jw = a.jxw * a.tab[kTabWq + q];
#pragma unroll
      for (int comp = 0; comp < 3; ++comp)
#pragma unroll
        for (int d = 0; d < 3; ++d)
          S[w][g * a.N + q][comp * 3 + d] = jw * ((comp == d ? lam * div : 0.0) + mu * (G3[comp][d] + G3[d][comp]));
    }
    __syncwarp();
    if (act && freen)
    {
      int const n = l;
      for (int comp = 0; comp < 3; ++comp)
      {
        double r = 0.0;
        for (int q = 0; q < a.N; ++q)
          for (int d = 0; d < 3; ++d)
            r = fma(S[w][g * a.N + q][comp * 3 + d], grad_s[(q * kMaxN + n) * 3 + d] * a.inv_h[d], r);
        atomicAdd(dst + comp * a.m + gidx, r);
      }
    }
    __syncwarp();
  }
}

// FE_Q(1) element matrices of one level's cell size, passed by value (the
// kernel-parameter bank): [2][8][8][3][3], K_lambda[a][b][ca][cb] =
// int d_ca phi_a d_cb phi_b, then K_mu[a][b][ca][cb] = int (delta_ca,cb
// grad phi_a . grad phi_b + d_cb phi_a d_ca phi_b).
struct Q1Matrices
{
  double k[2 * 576];
};

// dst += A src on the free rows of an FE_Q(1) operator, one thread per
// node and no atomics: the node's row gathers lambda K_lambda + mu K_mu of
// its (up to eight) cells, (lambda, mu) per cell from a.cell_coef (0 for
// the cells that carry no displacement); clamped and absent columns read
// as 0. The loops are unrolled so that every matrix entry is a constant
// operand of its FMA (no load), and the 27 neighbour values are read once:
// the lower node layer and the middle one serve the four lower cells, then
// the upper layer replaces the lower one for the four upper cells.
__global__ void __launch_bounds__(128) elastic_gather_q1_kernel(MechArgs a, const __grid_constant__ Q1Matrices kq,
                                                                double const *src, double *dst)
{
  int64_t const g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= a.m || a.node_mask[g] != 1)
    return;
  int const i = (int)(g % a.pitch);
  int64_t const rest = g / a.pitch;
  int const j = (int)(rest % a.nn[1]), k = (int)(rest / a.nn[1]);
  int64_t const sy = a.pitch, sz = (int64_t)a.pitch * a.nn[1];
  // u[layer][dy + 1][dx + 1][component] of the two node layers in use
  double u[2][3][3][3];
  auto load_layer = [&](int slot, int dz) {
#pragma unroll
    for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
      for (int dx = -1; dx <= 1; ++dx)
      {
        bool const ok = i + dx >= 0 && i + dx < a.nn[0] && j + dy >= 0 && j + dy < a.nn[1] && k + dz >= 0 &&
                        k + dz < a.nn[2];
        int64_t const gn = g + dx + sy * dy + sz * dz;
        bool const fr = ok && a.node_mask[gn] == 1;
#pragma unroll
        for (int c = 0; c < 3; ++c)
          u[slot][dy + 1][dx + 1][c] = fr ? src[c * a.m + gn] : 0.0;
      }
  };
  double acc[3] = {0.0, 0.0, 0.0};
  load_layer(0, -1);
  load_layer(1, 0);
#pragma unroll
  for (int oz = 0; oz < 2; ++oz)
  {
    if (oz == 1)
      load_layer(0, 1); // slot 0 now holds the upper layer
#pragma unroll
    for (int oy = 0; oy < 2; ++oy)
#pragma unroll
      for (int ox = 0; ox < 2; ++ox)
      {
        int const cx = i - 1 + ox, cy = j - 1 + oy, cz = k - 1 + oz;
        if (cx < 0 || cy < 0 || cz < 0 || cx >= a.nc[0] || cy >= a.nc[1] || cz >= a.nc[2])
          continue;
        int64_t const c = cx + (int64_t)a.nc[0] * (cy + (int64_t)a.nc[1] * cz);
        double const lam = a.cell_coef[2 * c], mu = a.cell_coef[2 * c + 1];
        if (lam == 0.0 && mu == 0.0)
          continue;
        int const la = (1 - ox) + 2 * (1 - oy) + 4 * (1 - oz); // the node's corner in the cell
        double al[3] = {0.0, 0.0, 0.0}, am[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int b = 0; b < 8; ++b)
        {
          int const bx = b & 1, by = (b >> 1) & 1, bz = b >> 2;
          // the cell node's layer: lower cells use slots 0 (dz -1) and 1
          // (dz 0); upper cells slots 1 (dz 0) and 0 (dz +1)
          int const slot = oz == 0 ? bz : 1 - bz;
          double const *uv = u[slot][oy + by][ox + bx];
          double const *Kl = &kq.k[(la * 8 + b) * 9];
          double const *Km = Kl + 576;
#pragma unroll
          for (int ca = 0; ca < 3; ++ca)
          {
            al[ca] = fma(Kl[3 * ca], uv[0], fma(Kl[3 * ca + 1], uv[1], fma(Kl[3 * ca + 2], uv[2], al[ca])));
            am[ca] = fma(Km[3 * ca], uv[0], fma(Km[3 * ca + 1], uv[1], fma(Km[3 * ca + 2], uv[2], am[ca])));
          }
        }
#pragma unroll
        for (int ca = 0; ca < 3; ++ca)
          acc[ca] = fma(lam, al[ca], fma(mu, am[ca], acc[ca]));
      }
  }
#pragma unroll
  for (int ca = 0; ca < 3; ++ca)
    dst[ca * a.m + g] += acc[ca];
}

// rhs += sum_q JxW ((3 lambda + 2 mu) alpha (T - T_ref) div v + f . v)
__global__ void __launch_bounds__(128) elastic_rhs_kernel(MechArgs a, double const *T, double *rhs)
{
  __shared__ double Tn[4][kMaxN];
  __shared__ double B[4][kMaxN], F[4][kMaxN];
  // the tables in shared memory (lane-divergent rows; see the operator)
  __shared__ double val_s[kMaxN * kMaxN], grad_s[kMaxN * kMaxN * 3];
  for (int e = threadIdx.x; e < kMaxN * kMaxN * 3; e += blockDim.x)
  {
    grad_s[e] = a.tab[kTabGrad + e];
    if (e < kMaxN * kMaxN)
      val_s[e] = a.tab[kTabVal + e];
  }
  __syncthreads();
  int const w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int const gw = blockIdx.x * 4 + w, nw = gridDim.x * 4;
  for (int ci = gw; ci < a.n_cells; ci += nw)
  {
    int const c = a.cells[ci];
    int const cx = c % a.nc[0], cy = (c / a.nc[0]) % a.nc[1], cz = c / (a.nc[0] * a.nc[1]);
    int const mat = a.matid[c];
    double const lam = a.lambda[mat], mu = a.mu[mat];
    double const tref = (a.melted && a.melted[c]) ? a.tref[mat] : a.tinit;
    int64_t g = 0;
    if (lane < a.N)
    {
      g = node_of(a, cx, cy, cz, lane);
      Tn[w][lane] = T ? T[g] : 0.0;
    }
    __syncwarp();
    if (lane < a.N)
    {
      int const q = lane;
      double const jw = a.jxw * a.tab[kTabWq + q];
      double b = 0.0;
      if (a.thermoelastic)
      {
        double dT = -tref;
        for (int n = 0; n < a.N; ++n)
          dT = fma(val_s[q * kMaxN + n], Tn[w][n], dT);
        b = (3.0 * lam + 2.0 * mu) * a.alpha[mat] * dT;
      }
      B[w][q] = jw * b;
      F[w][q] = a.gravity ? jw * (-a.rho[mat] * kGravity) : 0.0;
    }
    __syncwarp();
    if (lane < a.N && a.node_mask[g] == 1)
    {
      int const n = lane;
      for (int comp = 0; comp < 3; ++comp)
      {
        double r = 0.0;
        for (int q = 0; q < a.N; ++q)
        {
          r = fma(B[w][q], grad_s[(q * kMaxN + n) * 3 + comp] * a.inv_h[comp], r);
          if (comp == 2)
            r = fma(F[w][q], val_s[q * kMaxN + n], r);
        }
        atomicAdd(rhs + comp * a.m + g, r);
      }
    }
    __syncwarp();
  }
}

// diag += the operator's diagonal on the free rows
__global__ void __launch_bounds__(128) elastic_diag_kernel(MechArgs a, double *diag)
{
  __shared__ double grad_s[kMaxN * kMaxN * 3];
  for (int e = threadIdx.x; e < kMaxN * kMaxN * 3; e += blockDim.x)
    grad_s[e] = a.tab[kTabGrad + e];
  __syncthreads();
  int const w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int const gw = blockIdx.x * 4 + w, nw = gridDim.x * 4;
  for (int ci = gw; ci < a.n_cells; ci += nw)
  {
    int const c = a.cells[ci];
    int const cx = c % a.nc[0], cy = (c / a.nc[0]) % a.nc[1], cz = c / (a.nc[0] * a.nc[1]);
    double lam, mu;
    cell_lame(a, c, lam, mu);
    if (lane >= a.N)
      continue;
    int64_t const g = node_of(a, cx, cy, cz, lane);
    if (a.node_mask[g] != 1)
      continue;
    int const n = lane;
    for (int comp = 0; comp < 3; ++comp)
    {
      double r = 0.0;
      for (int q = 0; q < a.N; ++q)
      {
        double gg = 0.0, gc = 0.0;
        for (int d = 0; d < 3; ++d)
        {
          double const gd = grad_s[(q * kMaxN + n) * 3 + d] * a.inv_h[d];
          gg += gd * gd;
          if (d == comp)
            gc = gd;
        }
        r += a.jxw * a.tab[kTabWq + q] * ((lam + mu) * gc * gc + mu * gg);
      }
      atomicAdd(diag + comp * a.m + g, r);
    }
  }
}

// constrained rows: dst = src; rows without displacement: 0
__global__ void identity_rows_kernel(int64_t m, uint8_t const *mask, double const *src, double *dst)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 3 * m)
    return;
  uint8_t const k = mask[i % m];
  if (k == 2)
    dst[i] = src[i];
  else if (k == 0)
    dst[i] = 0.0;
}

// ---- CG vector kernels (3 m entries)
__global__ void dot_kernel(int64_t n, double const *x, double const *y, double *out)
{
  __shared__ double red[256];
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s = fma(x[i], y[i], s);
  red[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1)
  {
    if (threadIdx.x < o)
      red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    atomicAdd(out, red[0]);
}

// z = r / diag (diag 0: z = r)
__global__ void jacobi_kernel(int64_t n, double const *r, double const *diag, double *z)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n)
    z[i] = diag[i] != 0.0 ? r[i] / diag[i] : r[i];
}

// x += alpha p, r -= alpha q  (alpha = s[0] / s[1])
__global__ void cg_update_kernel(int64_t n, double const *s, double const *p, double const *q, double *x, double *r)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double const alpha = s[0] / s[1];
  x[i] = fma(alpha, p[i], x[i]);
  r[i] = fma(-alpha, q[i], r[i]);
}

// p = z + beta p (beta = s_new / s_old)
__global__ void cg_direction_kernel(int64_t n, double const *s_new, double const *s_old, double const *z, double *p)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  p[i] = fma(s_new[0] / s_old[0], p[i], z[i]);
}

// ---- geometric multigrid preconditioner of the CG
//
// The reference preconditions its CG with algebraic multigrid
// (MechanicalPhysics::solve, source/MechanicalPhysics.cc:488-520). Here: a
// V-cycle over a hierarchy of structured levels, the finest the operator
// itself (FE_Q(1) or FE_Q(2)), every coarser one FE_Q(1) rediscretized
// on a box with half the cells per direction (per direction while that
// count is even; an FE_Q(2) level first goes to FE_Q(1) on the same
// cells), (lambda, mu) of a coarse cell the volume average over its
// children (0 for children that carry no displacement); transfers are the
// trilinear interpolation between the node lattices and its transpose;
// the smoother is Chebyshev on diag^-1 A, the coarsest level is solved
// exactly (dense inverse) when it is small. The same Chebyshev polynomial
// before and after the coarse correction keeps the preconditioner
// symmetric, as CG needs.

// Node lattice of one level: x fastest with row pitch, m nodes per component.
struct Lattice
{
  int nn[3];
  int pitch;
  int64_t m;
};

// 1-D interpolation stencil from the coarse lattice (ratio r: 1 same
// index, 2 every other fine node coincides with a coarse one)
__device__ __forceinline__ int mg_stencil(int i, int r, int *ci, double *cw)
{
  if (r == 1 || (i & 1) == 0)
  {
    ci[0] = i / r;
    cw[0] = 1.0;
    return 1;
  }
  ci[0] = i >> 1;
  ci[1] = (i >> 1) + 1;
  cw[0] = cw[1] = 0.5;
  return 2;
}

// x_f += P x_c on the fine free rows (fine dinv != 0); the fine residual
// buffer q_f is cleared on the way for the next operator application
__global__ void mg_prolong_add_kernel(Lattice f, Lattice c, int r0, int r1, int r2, double const *dinv_f,
                                      double const *xc, double *xf, double *qf)
{
  int64_t const t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= f.m)
    return;
  for (int comp = 0; comp < 3; ++comp)
    qf[comp * f.m + t] = 0.0;
  if (dinv_f[t] == 0.0 && dinv_f[f.m + t] == 0.0 && dinv_f[2 * f.m + t] == 0.0)
    return;
  int const i = (int)(t % f.pitch);
  int64_t const rest = t / f.pitch;
  int const j = (int)(rest % f.nn[1]), k = (int)(rest / f.nn[1]);
  int ix[2], iy[2], iz[2];
  double wx[2], wy[2], wz[2];
  int const nx = mg_stencil(i, r0, ix, wx), ny = mg_stencil(j, r1, iy, wy), nz = mg_stencil(k, r2, iz, wz);
  for (int comp = 0; comp < 3; ++comp)
  {
    if (dinv_f[comp * f.m + t] == 0.0)
      continue;
    double const *x = xc + comp * c.m;
    double s = 0.0;
    for (int cz = 0; cz < nz; ++cz)
      for (int cy = 0; cy < ny; ++cy)
        for (int cx = 0; cx < nx; ++cx)
          s = fma(wx[cx] * wy[cy] * wz[cz], x[ix[cx] + (int64_t)c.pitch * (iy[cy] + (int64_t)c.nn[1] * iz[cz])], s);
    xf[comp * f.m + t] += s;
  }
}

// b_c = P^T r_f on the coarse free rows (coarse dinv != 0), 0 elsewhere;
// only fine free rows carry residual (the others are 0)
__global__ void mg_restrict_kernel(Lattice f, Lattice c, int r0, int r1, int r2, double const *dinv_c,
                                   double const *rf, double *bc)
{
  int64_t const t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= c.m)
    return;
  int const I = (int)(t % c.pitch);
  int64_t const rest = t / c.pitch;
  int const J = (int)(rest % c.nn[1]), K = (int)(rest / c.nn[1]);
  int const r[3] = {r0, r1, r2}, C[3] = {I, J, K};
  int lo[3], hi[3];
  for (int d = 0; d < 3; ++d)
  {
    int const cen = r[d] * C[d];
    lo[d] = r[d] == 1 ? cen : max(cen - 1, 0);
    hi[d] = r[d] == 1 ? cen : min(cen + 1, f.nn[d] - 1);
  }
  for (int comp = 0; comp < 3; ++comp)
  {
    double s = 0.0;
    if (dinv_c[comp * c.m + t] != 0.0)
    {
      double const *x = rf + comp * f.m;
      for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
          for (int i = lo[0]; i <= hi[0]; ++i)
          {
            double const w = (i == r0 * I ? 1.0 : 0.5) * (j == r1 * J ? 1.0 : 0.5) * (k == r2 * K ? 1.0 : 0.5);
            s = fma(w, x[i + (int64_t)f.pitch * (j + (int64_t)f.nn[1] * k)], s);
          }
    }
    bc[comp * c.m + t] = s;
  }
}

// One Chebyshev step: d = cd d + cr dinv (b - q), x += d (first: x = d, no
// q); q is cleared for the next operator application. Rows with dinv 0
// (no displacement, clamped) stay 0.
__global__ void mg_cheb_kernel(int64_t n, double const *b, double *q, double const *dinv, double *d, double *x,
                               double cd, double cr, int first)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double r = b[i];
  if (!first)
  {
    r -= q[i];
    q[i] = 0.0;
  }
  double const dn = (first ? 0.0 : cd * d[i]) + cr * dinv[i] * r;
  d[i] = dn;
  x[i] = first ? dn : x[i] + dn;
}

// r = b - q into rv; q cleared
__global__ void mg_residual_kernel(int64_t n, double const *b, double *q, double *rv)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  rv[i] = b[i] - q[i];
  q[i] = 0.0;
}

// x[idx[row]] = sum_j inv[row][j] b[idx[j]]: the coarsest level's exact
// solve (one warp per row)
__global__ void mg_dense_solve_kernel(int n, int64_t const *idx, double const *inv, double const *b, double *x)
{
  int const row = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
  int const lane = threadIdx.x & 31;
  if (row >= n)
    return;
  double s = 0.0;
  for (int j = lane; j < n; j += 32)
    s = fma(inv[(int64_t)row * n + j], b[idx[j]], s);
  for (int o = 16; o > 0; o >>= 1)
    s += __shfl_xor_sync(0xffffffffu, s, o);
  if (lane == 0)
    x[idx[row]] = s;
}

// dinv = 1 / diag on the free rows (diag != 0), 0 elsewhere
__global__ void mg_invert_diag_kernel(int64_t n, double const *diag, double *dinv)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n)
    dinv[i] = diag[i] != 0.0 ? 1.0 / diag[i] : 0.0;
}

// a seeded vector in [-1, 1] on the free rows (power iteration start)
__global__ void mg_seed_kernel(int64_t n, double const *dinv, double *v)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  uint64_t h = (uint64_t)i * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
  h ^= h >> 31;
  h *= 0xBF58476D1CE4E5B9ull;
  h ^= h >> 29;
  v[i] = dinv[i] != 0.0 ? (double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0 : 0.0;
}

// v = dinv q / s (s on the device: a norm), q cleared
__global__ void mg_power_kernel(int64_t n, double const *dinv, double *q, double const *s, double *v)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  v[i] = dinv[i] * q[i] / sqrt(*s);
  q[i] = 0.0;
}

unsigned blocks_for(int64_t n) { return (unsigned)std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 16)); }

// 1-D Gauss points / weights on [0, 1] and the Lagrange basis on the
// equidistant (Gauss-Lobatto for p <= 2) nodes
void gauss_1d(int n, double *x, double *w)
{
  if (n == 2)
  {
    double const s = 0.5 / std::sqrt(3.0);
    x[0] = 0.5 - s;
    x[1] = 0.5 + s;
    w[0] = w[1] = 0.5;
  }
  else
  {
    double const s = 0.5 * std::sqrt(0.6);
    x[0] = 0.5 - s;
    x[1] = 0.5;
    x[2] = 0.5 + s;
    w[0] = w[2] = 5.0 / 18.0;
    w[1] = 8.0 / 18.0;
  }
}

double lag(int p, int a, double u)
{
  double v = 1.0;
  for (int b = 0; b <= p; ++b)
    if (b != a)
      v *= (u * p - b) / (double)(a - b);
  return v;
}

double lag_d(int p, int a, double u)
{
  double s = 0.0;
  for (int k = 0; k <= p; ++k)
  {
    if (k == a)
      continue;
    double v = p / (double)(a - k);
    for (int b = 0; b <= p; ++b)
      if (b != a && b != k)
        v *= (u * p - b) / (double)(a - b);
    s += v;
  }
  return s;
}
} // namespace

class Mechanics
{
public:
  Mechanics(Thermal &th, adm_mech_config const &cfg) : th_(th), cfg_(cfg)
  {
    Mesh const &M = th_.mesh_;
    if (M.deg != 1 && M.deg != 2)
      throw Error(ADM_ERR_UNSUPPORTED, "mechanics takes FE degree 1 or 2");
    if (cfg_.clamped_faces < 0 || cfg_.clamped_faces > 63)
      throw Error(ADM_ERR_INVALID, "clamped_faces is a 6-bit mask");
    for (int k = 0; k < th_.cfg_.n_materials; ++k)
    {
      if (!(cfg_.lame_second[k] > 0.0) || !(cfg_.lame_first[k] > -2.0 / 3.0 * cfg_.lame_second[k]))
        throw Error(ADM_ERR_INVALID, "Lame parameters must give a positive definite elasticity tensor");
      if (std::isnan(cfg_.elastic_limit[k]) ||
          (std::isfinite(cfg_.elastic_limit[k]) && !(2.0 * cfg_.lame_second[k] + cfg_.plastic_modulus[k] > 0.0)))
        throw Error(ADM_ERR_INVALID, "J2 plasticity needs an elastic limit and 2 mu + plastic_modulus > 0");
    }
    p_ = M.deg;
    N_ = (p_ + 1) * (p_ + 1) * (p_ + 1);
    ADM_CK(cudaSetDevice(th_.device_));
    // reference-element tables of the degree, and of FE_Q(1) for the
    // multigrid levels
    std::vector<double> const tab = element_tables(p_);
    tab_.alloc(kTabSize);
    ADM_CK(cudaMemcpyAsync(tab_.p, tab.data(), kTabSize * sizeof(double), cudaMemcpyHostToDevice, th_.stream_));
    tab1_h_ = element_tables(1);
    tab1_.alloc(kTabSize);
    ADM_CK(cudaMemcpyAsync(tab1_.p, tab1_h_.data(), kTabSize * sizeof(double), cudaMemcpyHostToDevice,
                           th_.stream_));
    ADM_CK(cudaStreamSynchronize(th_.stream_));
  }

  ~Mechanics()
  {
    release_vcycle_graph();
    if (cap_stream_)
      cudaStreamDestroy(cap_stream_);
  }
  Mechanics(Mechanics const &) = delete;
  Mechanics &operator=(Mechanics const &) = delete;

  // FE_Q(1) element matrices of a cell of size h: [2][8][8][3][3], the
  // lambda part then the mu part (elastic_gather_q1_kernel)
  Q1Matrices q1_element_matrices(double const h[3]) const
  {
    Q1Matrices M{};
    double *K = M.k;
    double const inv_h[3] = {1.0 / h[0], 1.0 / h[1], 1.0 / h[2]};
    double const jxw = h[0] * h[1] * h[2];
    for (int q = 0; q < 8; ++q)
    {
      double const jw = jxw * tab1_h_[kTabWq + q];
      double gr[8][3];
      for (int a = 0; a < 8; ++a)
        for (int d = 0; d < 3; ++d)
          gr[a][d] = tab1_h_[kTabGrad + (q * kMaxN + a) * 3 + d] * inv_h[d];
      for (int a = 0; a < 8; ++a)
        for (int b = 0; b < 8; ++b)
        {
          double const dot = gr[a][0] * gr[b][0] + gr[a][1] * gr[b][1] + gr[a][2] * gr[b][2];
          for (int ca = 0; ca < 3; ++ca)
            for (int cb = 0; cb < 3; ++cb)
            {
              size_t const e = (size_t)(a * 8 + b) * 9 + ca * 3 + cb;
              K[e] += jw * gr[a][ca] * gr[b][cb];
              K[576 + e] += jw * (gr[a][cb] * gr[b][ca] + (ca == cb ? dot : 0.0));
            }
        }
    }
    return M;
  }

  // values [q][n], reference gradients [q][n][d] and weights of the
  // (p+1)^3 Gauss points of FE_Q(p) on [0, 1]^3, at the kTab* offsets
  static std::vector<double> element_tables(int p)
  {
    int const np = p + 1, N = np * np * np;
    double x[3], w[3];
    gauss_1d(np, x, w);
    std::vector<double> tab(kTabSize, 0.0);
    for (int q = 0; q < N; ++q)
    {
      int const qi = q % np, qj = (q / np) % np, qk = q / (np * np);
      tab[kTabWq + q] = w[qi] * w[qj] * w[qk];
      for (int n = 0; n < N; ++n)
      {
        int const ni = n % np, nj = (n / np) % np, nk = n / (np * np);
        double const vx = lag(p, ni, x[qi]), vy = lag(p, nj, x[qj]), vz = lag(p, nk, x[qk]);
        tab[kTabVal + q * kMaxN + n] = vx * vy * vz;
        tab[kTabGrad + (q * kMaxN + n) * 3 + 0] = lag_d(p, ni, x[qi]) * vy * vz;
        tab[kTabGrad + (q * kMaxN + n) * 3 + 1] = vx * lag_d(p, nj, x[qj]) * vz;
        tab[kTabGrad + (q * kMaxN + n) * 3 + 2] = vx * vy * lag_d(p, nk, x[qk]);
      }
    }
    return tab;
  }

  void setup(double const *temperature)
  {
    Thermal &t = th_;
    Mesh const &M = t.mesh_;
    if (!t.setup_done_)
      throw Error(ADM_ERR_INVALID, "the thermal handle is not set up");
    ADM_CK(cudaSetDevice(t.device_));
    size_t const C = M.n_cells;
    int const ns = t.ns_;
    // cell states (MaterialProperty state after set_state_to_material_properties)
    t.set_state_to_material_properties();
    std::vector<double> st((size_t)ns * C);
    t.get_cell_state(st.data());
    std::vector<int32_t> cells;
    for (size_t c = 0; c < C; ++c)
      if (t.active_[c] && st[c] > 0.99) // state 0: solid
        cells.push_back((int32_t)c);
    n_cells_ = (int64_t)cells.size();
    std::vector<uint8_t> carry(C, 0);
    for (int32_t c : cells)
      carry[c] = 1;
    // nodes of those cells; clamped: on a clamped box face
    m_ = (int64_t)M.n_nodes;
    std::vector<uint8_t> mask(m_, 0);
    int const np = p_ + 1;
    for (int32_t c : cells)
    {
      int const cx = c % M.nc[0], cy = (c / M.nc[0]) % M.nc[1], cz = c / (M.nc[0] * M.nc[1]);
      for (int n = 0; n < N_; ++n)
      {
        int const i = p_ * cx + n % np, j = p_ * cy + (n / np) % np, k = p_ * cz + n / (np * np);
        int const ijk[3] = {i, j, k};
        bool clamped = false;
        for (int f = 0; f < 6; ++f)
          if ((cfg_.clamped_faces >> f) & 1)
          {
            int const d = f / 2;
            if (ijk[d] == ((f & 1) ? M.nn[d] - 1 : 0))
              clamped = true;
          }
        uint8_t &mk = mask[i + (int64_t)M.pitch * (j + (int64_t)M.nn[1] * k)];
        mk = clamped ? 2 : std::max<uint8_t>(mk, 1);
      }
    }
    n_dofs_ = 0;
    for (uint8_t v : mask)
      n_dofs_ += v ? 3 : 0;
    mask_h_ = mask;
    cells_.alloc(std::max<size_t>(1, cells.size()));
    mask_.alloc(m_);
    matid_.alloc(C);
    melted_.alloc(C);
    cudaStream_t const s = t.stream_;
    if (!cells.empty())
      ADM_CK(cudaMemcpyAsync(cells_.p, cells.data(), cells.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    ADM_CK(cudaMemcpyAsync(mask_.p, mask.data(), m_, cudaMemcpyHostToDevice, s));
    ADM_CK(cudaMemcpyAsync(matid_.p, t.matid_.data(), C, cudaMemcpyHostToDevice, s));
    ADM_CK(cudaMemcpyAsync(melted_.p, t.has_melted_.data(), C, cudaMemcpyHostToDevice, s));
    setup_stress_state(carry, cells);
    // FE_Q(1): (lambda, mu) per cell (0 where no displacement) and the
    // element matrices of the gather operator
    if (p_ == 1)
    {
      std::vector<double> coef(2 * C, 0.0);
      for (int32_t c : cells)
      {
        coef[2 * c] = cfg_.lame_first[t.matid_[c]];
        coef[2 * c + 1] = cfg_.lame_second[t.matid_[c]];
      }
      coef0_d_.alloc(2 * C);
      ADM_CK(cudaMemcpyAsync(coef0_d_.p, coef.data(), 2 * C * sizeof(double), cudaMemcpyHostToDevice, s));
      double const h[3] = {M.h[0], M.h[1], M.h[2]};
      kq0_ = q1_element_matrices(h);
      ADM_CK(cudaStreamSynchronize(s));
    }
    // right-hand side and Jacobi diagonal
    rhs_.alloc(3 * m_);
    diag_.alloc(3 * m_);
    ADM_CK(cudaMemsetAsync(rhs_.p, 0, 3 * m_ * sizeof(double), s));
    ADM_CK(cudaMemsetAsync(diag_.p, 0, 3 * m_ * sizeof(double), s));
    MechArgs const a = args();
    unsigned const nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_cells_ + 3) / 4, 148 * 16));
    if (n_cells_ > 0)
    {
      if (cfg_.thermoelastic && !temperature)
        throw Error(ADM_ERR_INVALID, "a thermoelastic setup needs the temperature");
      elastic_rhs_kernel<<<nb, 128, 0, s>>>(a, cfg_.thermoelastic ? temperature : nullptr, rhs_.p);
      elastic_diag_kernel<<<nb, 128, 0, s>>>(a, diag_.p);
      ADM_CK(cudaGetLastError());
    }
    ADM_CK(cudaStreamSynchronize(s));
    carry_now_ = carry;
    release_vcycle_graph();
    mg_.clear();
    ready_ = true;
  }

  void vmult(double *dst, double const *src)
  {
    require();
    cudaStream_t const s = th_.stream_;
    ADM_CK(cudaSetDevice(th_.device_));
    ADM_CK(cudaMemsetAsync(dst, 0, 3 * m_ * sizeof(double), s));
    apply_free(dst, src);
    identity_rows_kernel<<<(unsigned)((3 * m_ + 255) / 256), 256, 0, s>>>(m_, mask_.p, src, dst);
    ADM_CK(cudaGetLastError());
  }

  void copy_rhs(double *dst)
  {
    require();
    ADM_CK(cudaMemcpyAsync(dst, rhs_.p, 3 * m_ * sizeof(double), cudaMemcpyDeviceToDevice, th_.stream_));
    ADM_CK(cudaStreamSynchronize(th_.stream_));
  }

  // Preconditioned CG (multigrid V-cycle or Jacobi) from x = 0 (the
  // constrained and absent entries stay 0): stops at |r| <= rel_tol |rhs| (SolverControl of
  // MechanicalPhysics::solve) or after max_iter iterations (an error).
  void solve(double *x, int32_t *iterations, double *residual)
  {
    require();
    cudaStream_t const s = th_.stream_;
    ADM_CK(cudaSetDevice(th_.device_));
    int64_t const n = 3 * m_;
    r_.alloc(n);
    z_.alloc(n);
    pv_.alloc(n);
    qv_.alloc(n);
    sc_.alloc(8);
    ADM_CK(cudaMemsetAsync(x, 0, n * sizeof(double), s));
    ADM_CK(cudaMemsetAsync(z_.p, 0, n * sizeof(double), s));
    ADM_CK(cudaMemcpyAsync(r_.p, rhs_.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (precond_ == ADM_MECH_PRECONDITIONER_MULTIGRID && mg_.empty() && n_cells_ > 0)
      setup_multigrid();
    double const rhs_norm = std::sqrt(dot(rhs_.p, rhs_.p, 0));
    double const tol = (cfg_.rel_tol > 0.0 ? cfg_.rel_tol : 1e-12) * rhs_norm;
    int const max_iter = cfg_.max_iter > 0 ? cfg_.max_iter : (int)std::max<int64_t>(1, n_dofs_);
    double res = rhs_norm;
    int it = 0;
    if (res > tol)
    {
      precondition(r_.p, z_.p);
      ADM_CK(cudaMemcpyAsync(pv_.p, z_.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
      dot_device(r_.p, z_.p, 0); // sc[0] = r.z
      for (it = 1; it <= max_iter; ++it)
      {
        vmult(qv_.p, pv_.p);
        dot_device(pv_.p, qv_.p, 1); // sc[1] = p.q (alpha = sc[0] / sc[1] on the device)
        cg_update_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, sc_.p, pv_.p, qv_.p, x, r_.p);
        ADM_CK(cudaGetLastError());
        res = std::sqrt(dot(r_.p, r_.p, 2));
        if (res <= tol)
          break;
        precondition(r_.p, z_.p);
        dot_device(r_.p, z_.p, 3); // sc[3] = new r.z
        cg_direction_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, sc_.p + 3, sc_.p, z_.p, pv_.p);
        ADM_CK(cudaGetLastError());
        ADM_CK(cudaMemcpyAsync(sc_.p, sc_.p + 3, sizeof(double), cudaMemcpyDeviceToDevice, s));
      }
      if (it > max_iter)
        throw Error(ADM_ERR_DEVICE, "the mechanical CG did not converge within max_iter iterations");
    }
    if (iterations)
      *iterations = it;
    if (residual)
      *residual = res;
    update_stress(x);
  }

  // stress state of the Gauss points into caller device arrays
  void stress_state(double *stress, double *back, double *plastic)
  {
    require();
    cudaStream_t const s = th_.stream_;
    ADM_CK(cudaSetDevice(th_.device_));
    int64_t const cq = (int64_t)th_.mesh_.n_cells * N_;
    if (stress)
      ADM_CK(cudaMemcpyAsync(stress, stress_.p, 6 * cq * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (back)
      ADM_CK(cudaMemcpyAsync(back, back_.p, 6 * cq * sizeof(double), cudaMemcpyDeviceToDevice, s));
    if (plastic)
      ADM_CK(cudaMemcpyAsync(plastic, kappa_.p, cq * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ADM_CK(cudaStreamSynchronize(s));
  }

  void set_preconditioner(int kind)
  {
    if (kind != ADM_MECH_PRECONDITIONER_JACOBI && kind != ADM_MECH_PRECONDITIONER_MULTIGRID)
      throw Error(ADM_ERR_INVALID, "unknown preconditioner");
    precond_ = kind;
  }

  void multigrid_levels(int32_t *n_levels, int64_t *coarsest) const
  {
    if (n_levels)
      *n_levels = (int32_t)mg_.size();
    if (coarsest)
      *coarsest = mg_.empty() ? 0 : 3 * mg_.back()->n_free;
  }

  int64_t n_dofs() const { return n_dofs_; }
  int64_t n_cells() const { return n_cells_; }
  std::vector<uint8_t> const &mask() const { return mask_h_; }

private:
  void require() const
  {
    if (!ready_)
      throw Error(ADM_ERR_INVALID, "adm_mechanics_setup has not been called");
  }

  J2State j2() const { return J2State{kappa_.p, stress_.p, back_.p, (int64_t)th_.mesh_.n_cells * N_}; }

  // The Gauss-point state and the previous displacement when the cells that
  // carry displacement are (re)chosen: cells that start carrying it start
  // from the elastic limit and zero stresses, and the previous displacement
  // follows MechanicalPhysics::setup_dofs (old_displacement_transfer_kernel).
  void setup_stress_state(std::vector<uint8_t> const &carry, std::vector<int32_t> const &cells)
  {
    cudaStream_t const s = th_.stream_;
    size_t const C = th_.mesh_.n_cells;
    bool const first = carry_prev_.empty();
    std::vector<int32_t> fresh;
    bool changed = first;
    for (int32_t c : cells)
      if (first || !carry_prev_[c])
        fresh.push_back(c);
    if (!first)
      for (size_t c = 0; c < C; ++c)
        changed = changed || (carry[c] != carry_prev_[c]);
    if (first)
    {
      int64_t const cq = (int64_t)C * N_;
      kappa_.alloc(std::max<int64_t>(1, cq));
      stress_.alloc(std::max<int64_t>(1, 6 * cq));
      back_.alloc(std::max<int64_t>(1, 6 * cq));
      ADM_CK(cudaMemsetAsync(stress_.p, 0, 6 * cq * sizeof(double), s));
      ADM_CK(cudaMemsetAsync(back_.p, 0, 6 * cq * sizeof(double), s));
      // every cell starts at its material's elastic limit
      std::vector<int32_t> all(C);
      for (size_t c = 0; c < C; ++c)
        all[c] = (int32_t)c;
      init_points(all);
      u_old_.alloc(3 * m_);
      carry_d_.alloc(2 * C);
    }
    else if (!fresh.empty())
      init_points(fresh);
    if (!first && changed && has_old_)
    {
      ADM_CK(cudaMemcpyAsync(carry_d_.p, carry_prev_.data(), C, cudaMemcpyHostToDevice, s));
      ADM_CK(cudaMemcpyAsync(carry_d_.p + C, carry.data(), C, cudaMemcpyHostToDevice, s));
      old_displacement_transfer_kernel<<<(unsigned)((m_ + 255) / 256), 256, 0, s>>>(args(), carry_d_.p,
                                                                                     carry_d_.p + C, u_old_.p);
      ADM_CK(cudaGetLastError());
    }
    ADM_CK(cudaStreamSynchronize(s));
    carry_prev_ = carry;
  }

  void init_points(std::vector<int32_t> const &list)
  {
    if (list.empty())
      return;
    cudaStream_t const s = th_.stream_;
    DevBuf<int32_t> d;
    d.alloc(list.size());
    ADM_CK(cudaMemcpyAsync(d.p, list.data(), list.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    MechArgs a = args();
    a.matid = matid_.p;
    int64_t const n = (int64_t)list.size() * N_;
    j2_init_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(a, j2(), d.p, (int)list.size());
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaStreamSynchronize(s)); // d is released on return
  }

  // after a solve: stress from the displacement increment, then the
  // displacement becomes the previous one
  void update_stress(double const *u)
  {
    if (n_cells_ == 0)
      return;
    cudaStream_t const s = th_.stream_;
    int64_t const n = n_cells_ * N_;
    j2_stress_kernel<<<(unsigned)((n + 127) / 128), 128, 0, s>>>(args(), j2(), u, has_old_ ? u_old_.p : nullptr);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaMemcpyAsync(u_old_.p, u, 3 * m_ * sizeof(double), cudaMemcpyDeviceToDevice, s));
    ADM_CK(cudaStreamSynchronize(s));
    has_old_ = true;
  }

  MechArgs args() const
  {
    Thermal const &t = th_;
    Mesh const &M = t.mesh_;
    MechArgs a{};
    a.p = p_;
    a.N = N_;
    for (int d = 0; d < 3; ++d)
    {
      a.nc[d] = M.nc[d];
      a.nn[d] = M.nn[d];
      a.inv_h[d] = 1.0 / M.h[d];
    }
    a.pitch = M.pitch;
    a.m = m_;
    a.jxw = M.h[0] * M.h[1] * M.h[2];
    a.cells = cells_.p;
    a.n_cells = (int)n_cells_;
    a.node_mask = mask_.p;
    a.matid = matid_.p;
    for (int k = 0; k < 4; ++k)
    {
      a.lambda[k] = cfg_.lame_first[k];
      a.mu[k] = cfg_.lame_second[k];
      a.alpha[k] = cfg_.thermal_expansion[k];
      a.rho[k] = cfg_.density[k];
      a.tref[k] = cfg_.reference_temperature[k];
      a.plastic_modulus[k] = cfg_.plastic_modulus[k];
      a.iso_hardening[k] = cfg_.isotropic_hardening[k];
      a.elastic_limit[k] = cfg_.elastic_limit[k];
    }
    a.tinit = cfg_.initial_temperature;
    a.thermoelastic = cfg_.thermoelastic;
    a.gravity = cfg_.gravity;
    a.melted = melted_.p;
    a.tab = tab_.p;
    a.cell_coef = p_ == 1 ? coef0_d_.p : nullptr;
    return a;
  }

  void apply_free(double *dst, double const *src)
  {
    if (n_cells_ == 0)
      return;
    if (p_ == 1)
    {
      elastic_gather_q1_kernel<<<(unsigned)((m_ + 127) / 128), 128, 0, th_.stream_>>>(args(), kq0_, src, dst);
      ADM_CK(cudaGetLastError());
      return;
    }
    int64_t const per_warp = 32 / N_;
    unsigned const nb =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((n_cells_ + 4 * per_warp - 1) / (4 * per_warp), 148 * 16));
    elastic_apply_kernel<<<nb, 128, 0, th_.stream_>>>(args(), src, dst);
    ADM_CK(cudaGetLastError());
  }

  void precondition(double const *r, double *z)
  {
    if (precond_ == ADM_MECH_PRECONDITIONER_MULTIGRID)
    {
      // the V-cycle (some 20 launches per level) replays as one CUDA graph,
      // captured on a stream of our own (the handle's may be the legacy
      // default stream, which cannot be captured)
      if (!vc_exec_ || vc_r_ != r || vc_z_ != z)
      {
        release_vcycle_graph();
        if (!cap_stream_)
          ADM_CK(cudaStreamCreateWithFlags(&cap_stream_, cudaStreamNonBlocking));
        MgLevel &L = *mg_[0];
        L.bp = const_cast<double *>(r);
        L.xp = z;
        cudaGraph_t graph;
        ls_ = cap_stream_;
        ADM_CK(cudaStreamBeginCapture(cap_stream_, cudaStreamCaptureModeThreadLocal));
        try
        {
          mg_vcycle(0);
        }
        catch (...)
        {
          cudaStreamEndCapture(cap_stream_, &graph);
          ls_ = nullptr;
          throw;
        }
        cudaError_t const e = cudaStreamEndCapture(cap_stream_, &graph);
        ls_ = nullptr;
        ADM_CK(e);
        ADM_CK(cudaGraphInstantiate(&vc_exec_, graph, 0));
        cudaGraphDestroy(graph);
        vc_r_ = r;
        vc_z_ = z;
      }
      ADM_CK(cudaGraphLaunch(vc_exec_, th_.stream_));
      return;
    }
    int64_t const n = 3 * m_;
    jacobi_kernel<<<(unsigned)((n + 255) / 256), 256, 0, th_.stream_>>>(n, r, diag_.p, z);
    ADM_CK(cudaGetLastError());
  }

  // ---- geometric multigrid (the kernels' comment above tells the design)
  static constexpr int kSmoothDegree = 3;   // Chebyshev steps before and after the coarse correction
  static constexpr double kSmoothRange = 15.0; // smoothed part of the spectrum: [lmax / range, lmax]
  static constexpr int kCoarseDegree = 12;  // Chebyshev steps on a coarsest level too large to invert
  static constexpr int kDirectMax = 640;    // free DoFs of a coarsest level solved by a dense inverse
  static constexpr int kPowerSteps = 16;    // power iterations for lmax(diag^-1 A)

  struct MgLevel
  {
    int p = 1, N = 8;
    int nc[3] = {0, 0, 0};
    int r[3] = {1, 1, 1}; // node-lattice ratio to the next coarser level
    double h[3] = {0, 0, 0};
    Lattice lat{};
    std::vector<uint8_t> carry; // per cell: carries displacement
    std::vector<double> coef;   // per cell: (lambda, mu), 0 where it carries none
    std::vector<uint8_t> mask;  // per node: 0 none, 1 free, 2 clamped
    int64_t n_cells = 0, n_free = 0;
    DevBuf<int32_t> cells;
    DevBuf<uint8_t> maskd;
    DevBuf<double> coefd, dinv, b, x, q, d;
    double *bp = nullptr, *xp = nullptr; // right-hand side and solution (level 0: the CG's)
    std::vector<double> cd, cr;          // Chebyshev step coefficients
    double lmax = 0.0;
    Q1Matrices kq{};                 // FE_Q(1) element matrices of the level's cells (gather apply)
    Q1Matrices const *kqp = nullptr; // kq, or the finest level's
    int n_direct = 0; // > 0: coarsest level solved by the dense inverse
    DevBuf<int64_t> didx;
    DevBuf<double> dinvm;
    MechArgs a{};
  };

  int64_t count_free(std::vector<uint8_t> const &mask) const
  {
    int64_t n = 0;
    for (uint8_t v : mask)
      n += v == 1;
    return n;
  }

  // node mask of a box level from the cells that carry displacement
  std::vector<uint8_t> level_mask(MgLevel const &L) const
  {
    std::vector<uint8_t> mask(L.lat.m, 0);
    int const np = L.p + 1;
    for (int64_t c = 0; c < (int64_t)L.carry.size(); ++c)
    {
      if (!L.carry[c])
        continue;
      int const cx = (int)(c % L.nc[0]), cy = (int)((c / L.nc[0]) % L.nc[1]), cz = (int)(c / ((int64_t)L.nc[0] * L.nc[1]));
      for (int n = 0; n < L.N; ++n)
      {
        int const ijk[3] = {L.p * cx + n % np, L.p * cy + (n / np) % np, L.p * cz + n / (np * np)};
        bool clamped = false;
        for (int f = 0; f < 6; ++f)
          if ((cfg_.clamped_faces >> f) & 1)
            clamped = clamped || ijk[f / 2] == ((f & 1) ? L.lat.nn[f / 2] - 1 : 0);
        uint8_t &mk = mask[ijk[0] + (int64_t)L.lat.pitch * (ijk[1] + (int64_t)L.lat.nn[1] * ijk[2])];
        mk = clamped ? 2 : std::max<uint8_t>(mk, 1);
      }
    }
    return mask;
  }

  // the stream the V-cycle's launches go to (the capture stream while one
  // is captured)
  cudaStream_t ls() const { return ls_ ? ls_ : th_.stream_; }

  void release_vcycle_graph()
  {
    if (vc_exec_)
      cudaGraphExecDestroy(vc_exec_);
    vc_exec_ = nullptr;
    vc_r_ = nullptr;
    vc_z_ = nullptr;
  }

  void mg_apply(MgLevel &L, double const *src)
  {
    if (L.n_cells == 0)
      return;
    if (L.p == 1)
    {
      elastic_gather_q1_kernel<<<(unsigned)((L.lat.m + 127) / 128), 128, 0, ls()>>>(L.a, *L.kqp, src, L.q.p);
      ADM_CK(cudaGetLastError());
      return;
    }
    int64_t const per_warp = 32 / L.N;
    unsigned const nb =
        (unsigned)std::max<int64_t>(1, std::min<int64_t>((L.n_cells + 4 * per_warp - 1) / (4 * per_warp), 148 * 16));
    elastic_apply_kernel<<<nb, 128, 0, ls()>>>(L.a, src, L.q.p);
    ADM_CK(cudaGetLastError());
  }

  void mg_smooth(MgLevel &L, bool zero_start)
  {
    cudaStream_t const s = ls();
    int64_t const n = 3 * L.lat.m;
    for (size_t j = 0; j < L.cd.size(); ++j)
    {
      bool const first = zero_start && j == 0;
      if (!first)
        mg_apply(L, L.xp);
      mg_cheb_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, L.bp, L.q.p, L.dinv.p, L.d.p, L.xp, L.cd[j],
                                                                  L.cr[j], first ? 1 : 0);
      ADM_CK(cudaGetLastError());
    }
  }

  void mg_vcycle(size_t l)
  {
    cudaStream_t const s = ls();
    MgLevel &L = *mg_[l];
    if (l + 1 == mg_.size())
    {
      if (L.n_direct > 0)
      {
        mg_dense_solve_kernel<<<(unsigned)((L.n_direct + 7) / 8), 256, 0, s>>>(L.n_direct, L.didx.p, L.dinvm.p,
                                                                                L.bp, L.xp);
        ADM_CK(cudaGetLastError());
      }
      else
        mg_smooth(L, true);
      return;
    }
    MgLevel &C = *mg_[l + 1];
    int64_t const n = 3 * L.lat.m;
    mg_smooth(L, true);
    mg_apply(L, L.xp);
    mg_residual_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, L.bp, L.q.p, L.d.p);
    mg_restrict_kernel<<<(unsigned)((C.lat.m + 255) / 256), 256, 0, s>>>(L.lat, C.lat, L.r[0], L.r[1], L.r[2],
                                                                         C.dinv.p, L.d.p, C.bp);
    ADM_CK(cudaGetLastError());
    mg_vcycle(l + 1);
    mg_prolong_add_kernel<<<(unsigned)((L.lat.m + 255) / 256), 256, 0, s>>>(L.lat, C.lat, L.r[0], L.r[1], L.r[2],
                                                                            L.dinv.p, C.xp, L.xp, L.q.p);
    ADM_CK(cudaGetLastError());
    mg_smooth(L, false);
  }

  // the level's device buffers, its operator arguments and diag^-1
  void mg_device(MgLevel &L, bool finest)
  {
    cudaStream_t const s = th_.stream_;
    int64_t const n = 3 * L.lat.m;
    L.dinv.alloc(n);
    L.q.alloc(n);
    L.d.alloc(n);
    ADM_CK(cudaMemsetAsync(L.q.p, 0, n * sizeof(double), s));
    ADM_CK(cudaMemsetAsync(L.d.p, 0, n * sizeof(double), s));
    if (finest)
    {
      L.a = args();
      L.kqp = &kq0_;
      mg_invert_diag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, diag_.p, L.dinv.p);
      ADM_CK(cudaGetLastError());
      return;
    }
    L.kq = q1_element_matrices(L.h);
    L.kqp = &L.kq;
    std::vector<int32_t> cells;
    for (int64_t c = 0; c < (int64_t)L.carry.size(); ++c)
      if (L.carry[c])
        cells.push_back((int32_t)c);
    L.n_cells = (int64_t)cells.size();
    L.cells.alloc(std::max<size_t>(1, cells.size()));
    L.maskd.alloc(L.lat.m);
    L.coefd.alloc(std::max<size_t>(2, L.coef.size()));
    L.b.alloc(n);
    L.x.alloc(n);
    ADM_CK(cudaMemsetAsync(L.x.p, 0, n * sizeof(double), s));
    if (!cells.empty())
      ADM_CK(cudaMemcpyAsync(L.cells.p, cells.data(), cells.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    ADM_CK(cudaMemcpyAsync(L.maskd.p, L.mask.data(), L.lat.m, cudaMemcpyHostToDevice, s));
    ADM_CK(cudaMemcpyAsync(L.coefd.p, L.coef.data(), L.coef.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    L.bp = L.b.p;
    L.xp = L.x.p;
    MechArgs a = args();
    a.p = 1;
    a.N = 8;
    for (int d = 0; d < 3; ++d)
    {
      a.nc[d] = L.nc[d];
      a.nn[d] = L.lat.nn[d];
      a.inv_h[d] = 1.0 / L.h[d];
    }
    a.pitch = L.lat.pitch;
    a.m = L.lat.m;
    a.jxw = L.h[0] * L.h[1] * L.h[2];
    a.cells = L.cells.p;
    a.n_cells = (int)L.n_cells;
    a.node_mask = L.maskd.p;
    a.cell_coef = L.coefd.p;
    a.tab = tab1_.p;
    L.a = a;
    // diag^-1 (the diagonal kernel with these arguments; q serves as scratch)
    unsigned const nb = (unsigned)std::max<int64_t>(1, std::min<int64_t>((L.n_cells + 3) / 4, 148 * 16));
    if (L.n_cells > 0)
      elastic_diag_kernel<<<nb, 128, 0, s>>>(a, L.q.p);
    mg_invert_diag_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, L.q.p, L.dinv.p);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaMemsetAsync(L.q.p, 0, n * sizeof(double), s));
  }

  // lmax(diag^-1 A) by power iteration, then the Chebyshev coefficients
  void mg_chebyshev(MgLevel &L, int degree)
  {
    cudaStream_t const s = th_.stream_;
    int64_t const n = 3 * L.lat.m;
    mg_seed_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, L.dinv.p, L.d.p);
    ADM_CK(cudaGetLastError());
    double nv = dot_n(L.d.p, L.d.p, n, 4);
    double lmax = 0.0;
    for (int it = 0; it < kPowerSteps && nv > 0.0; ++it)
    {
      mg_apply(L, L.d.p);
      mg_power_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, L.dinv.p, L.q.p, sc_.p + 4, L.d.p);
      ADM_CK(cudaGetLastError());
      nv = dot_n(L.d.p, L.d.p, n, 4);
      lmax = std::sqrt(nv);
    }
    ADM_CK(cudaMemsetAsync(L.d.p, 0, n * sizeof(double), s));
    L.lmax = lmax;
    double const upper = 1.2 * (lmax > 0.0 ? lmax : 1.0), lower = upper / kSmoothRange;
    double const theta = 0.5 * (upper + lower), delta = 0.5 * (upper - lower), sigma = theta / delta;
    L.cd.assign(1, 0.0);
    L.cr.assign(1, 1.0 / theta);
    double rho = 1.0 / sigma;
    for (int j = 1; j < degree; ++j)
    {
      double const rn = 1.0 / (2.0 * sigma - rho);
      L.cd.push_back(rn * rho);
      L.cr.push_back(2.0 * rn / delta);
      rho = rn;
    }
  }

  // dense inverse of the coarsest FE_Q(1) level's operator on its free DoFs
  void mg_direct(MgLevel &L)
  {
    std::vector<int64_t> idx;
    std::vector<int64_t> pos(3 * L.lat.m, -1);
    for (int comp = 0; comp < 3; ++comp)
      for (int64_t g = 0; g < L.lat.m; ++g)
        if (L.mask[g] == 1)
        {
          pos[comp * L.lat.m + g] = (int64_t)idx.size();
          idx.push_back(comp * L.lat.m + g);
        }
    int const n = (int)idx.size();
    std::vector<double> K((size_t)n * n, 0.0);
    double const inv_h[3] = {1.0 / L.h[0], 1.0 / L.h[1], 1.0 / L.h[2]};
    double const jxw = L.h[0] * L.h[1] * L.h[2];
    for (int64_t c = 0; c < (int64_t)L.carry.size(); ++c)
    {
      if (!L.carry[c])
        continue;
      double const lam = L.coef[2 * c], mu = L.coef[2 * c + 1];
      int const cx = (int)(c % L.nc[0]), cy = (int)((c / L.nc[0]) % L.nc[1]), cz = (int)(c / ((int64_t)L.nc[0] * L.nc[1]));
      int64_t g[8];
      for (int a = 0; a < 8; ++a)
        g[a] = (cx + (a & 1)) + (int64_t)L.lat.pitch * ((cy + ((a >> 1) & 1)) + (int64_t)L.lat.nn[1] * (cz + (a >> 2)));
      for (int q = 0; q < 8; ++q)
      {
        double const jw = jxw * tab1_h_[kTabWq + q];
        double gr[8][3];
        for (int a = 0; a < 8; ++a)
          for (int d = 0; d < 3; ++d)
            gr[a][d] = tab1_h_[kTabGrad + (q * kMaxN + a) * 3 + d] * inv_h[d];
        for (int a = 0; a < 8; ++a)
          for (int ca = 0; ca < 3; ++ca)
          {
            int64_t const ra = pos[ca * L.lat.m + g[a]];
            if (ra < 0)
              continue;
            for (int b = 0; b < 8; ++b)
              for (int cb = 0; cb < 3; ++cb)
              {
                int64_t const rb = pos[cb * L.lat.m + g[b]];
                if (rb < 0)
                  continue;
                double v = lam * gr[a][ca] * gr[b][cb] + mu * gr[a][cb] * gr[b][ca];
                if (ca == cb)
                  v += mu * (gr[a][0] * gr[b][0] + gr[a][1] * gr[b][1] + gr[a][2] * gr[b][2]);
                K[(size_t)ra * n + rb] += jw * v;
              }
          }
      }
    }
    // Cholesky K = L L^T (lower, in place), then the inverse column by column
    for (int j = 0; j < n; ++j)
    {
      double dsum = K[(size_t)j * n + j];
      for (int k = 0; k < j; ++k)
        dsum -= K[(size_t)j * n + k] * K[(size_t)j * n + k];
      if (!(dsum > 0.0))
        throw Error(ADM_ERR_DEVICE, "the coarsest multigrid level is not positive definite");
      double const ljj = std::sqrt(dsum);
      K[(size_t)j * n + j] = ljj;
      for (int i = j + 1; i < n; ++i)
      {
        double v = K[(size_t)i * n + j];
        for (int k = 0; k < j; ++k)
          v -= K[(size_t)i * n + k] * K[(size_t)j * n + k];
        K[(size_t)i * n + j] = v / ljj;
      }
    }
    std::vector<double> inv((size_t)n * n, 0.0), col(n);
    for (int e = 0; e < n; ++e)
    {
      for (int i = 0; i < n; ++i)
      {
        double v = i == e ? 1.0 : 0.0;
        for (int k = 0; k < i; ++k)
          v -= K[(size_t)i * n + k] * col[k];
        col[i] = v / K[(size_t)i * n + i];
      }
      for (int i = n - 1; i >= 0; --i)
      {
        double v = col[i];
        for (int k = i + 1; k < n; ++k)
          v -= K[(size_t)k * n + i] * col[k];
        col[i] = v / K[(size_t)i * n + i];
      }
      for (int i = 0; i < n; ++i)
        inv[(size_t)i * n + e] = col[i];
    }
    cudaStream_t const s = th_.stream_;
    L.n_direct = n;
    L.didx.alloc(std::max(1, n));
    L.dinvm.alloc(std::max<size_t>(1, (size_t)n * n));
    if (n > 0)
    {
      ADM_CK(cudaMemcpyAsync(L.didx.p, idx.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice, s));
      ADM_CK(cudaMemcpyAsync(L.dinvm.p, inv.data(), (size_t)n * n * sizeof(double), cudaMemcpyHostToDevice, s));
    }
    ADM_CK(cudaStreamSynchronize(s));
  }

  // the level hierarchy for the current cells (built at the first
  // multigrid solve after a setup)
  void setup_multigrid()
  {
    Mesh const &M = th_.mesh_;
    release_vcycle_graph();
    mg_.clear();
    sc_.alloc(8);
    auto L0 = std::make_unique<MgLevel>();
    L0->p = p_;
    L0->N = N_;
    for (int d = 0; d < 3; ++d)
    {
      L0->nc[d] = M.nc[d];
      L0->h[d] = M.h[d];
      L0->lat.nn[d] = M.nn[d];
    }
    L0->lat.pitch = M.pitch;
    L0->lat.m = m_;
    L0->carry = carry_now_;
    L0->coef.assign(2 * carry_now_.size(), 0.0);
    for (size_t c = 0; c < carry_now_.size(); ++c)
      if (carry_now_[c])
      {
        L0->coef[2 * c] = cfg_.lame_first[th_.matid_[c]];
        L0->coef[2 * c + 1] = cfg_.lame_second[th_.matid_[c]];
      }
    L0->mask = mask_h_;
    L0->n_cells = n_cells_;
    L0->n_free = count_free(mask_h_);
    mg_device(*L0, true);
    mg_.push_back(std::move(L0));
    while (mg_.size() < 16)
    {
      MgLevel &F = *mg_.back();
      int rc[3];
      if (F.p == 2)
        rc[0] = rc[1] = rc[2] = 1; // FE_Q(1) on the same cells
      else
      {
        if (3 * F.n_free <= kDirectMax)
          break;
        for (int d = 0; d < 3; ++d)
          rc[d] = (F.nc[d] % 2 == 0) ? 2 : 1;
        if (rc[0] == 1 && rc[1] == 1 && rc[2] == 1)
          break;
      }
      auto C = std::make_unique<MgLevel>();
      for (int d = 0; d < 3; ++d)
      {
        C->nc[d] = F.nc[d] / rc[d];
        C->h[d] = F.h[d] * rc[d];
        C->lat.nn[d] = C->nc[d] + 1;
        F.r[d] = F.p == 2 ? 2 : rc[d];
      }
      C->lat.pitch = C->lat.nn[0];
      C->lat.m = (int64_t)C->lat.nn[0] * C->lat.nn[1] * C->lat.nn[2];
      int64_t const nC = (int64_t)C->nc[0] * C->nc[1] * C->nc[2];
      C->carry.assign(nC, 0);
      C->coef.assign(2 * nC, 0.0);
      double const share = 1.0 / (rc[0] * rc[1] * rc[2]);
      for (int64_t c = 0; c < (int64_t)F.carry.size(); ++c)
      {
        if (!F.carry[c])
          continue;
        int const fx = (int)(c % F.nc[0]), fy = (int)((c / F.nc[0]) % F.nc[1]), fz = (int)(c / ((int64_t)F.nc[0] * F.nc[1]));
        int64_t const cc = fx / rc[0] + (int64_t)C->nc[0] * (fy / rc[1] + (int64_t)C->nc[1] * (fz / rc[2]));
        C->carry[cc] = 1;
        C->coef[2 * cc] += share * F.coef[2 * c];
        C->coef[2 * cc + 1] += share * F.coef[2 * c + 1];
      }
      C->mask = level_mask(*C);
      C->n_free = count_free(C->mask);
      mg_device(*C, false);
      mg_.push_back(std::move(C));
    }
    // smoothers on every level but a coarsest one small enough to invert
    MgLevel &last = *mg_.back();
    bool const direct = last.p == 1 && 3 * last.n_free <= kDirectMax;
    for (size_t l = 0; l < mg_.size(); ++l)
    {
      bool const coarsest = l + 1 == mg_.size();
      if (coarsest && direct)
        mg_direct(*mg_[l]);
      else
        mg_chebyshev(*mg_[l], coarsest ? kCoarseDegree : kSmoothDegree);
    }
    ADM_CK(cudaStreamSynchronize(th_.stream_));
  }

  // sc[slot] = x . y on the device (no read-back: the CG's scalars stay
  // there; only the residual norm comes back, once per iteration)
  void dot_device(double const *x, double const *y, int slot)
  {
    cudaStream_t const s = th_.stream_;
    int64_t const n = 3 * m_;
    ADM_CK(cudaMemsetAsync(sc_.p + slot, 0, sizeof(double), s));
    dot_kernel<<<blocks_for(n), 256, 0, s>>>(n, x, y, sc_.p + slot);
    ADM_CK(cudaGetLastError());
  }

  // sc[slot] = x . y over n entries (device), also returned to the host
  double dot_n(double const *x, double const *y, int64_t n, int slot)
  {
    cudaStream_t const s = th_.stream_;
    ADM_CK(cudaMemsetAsync(sc_.p + slot, 0, sizeof(double), s));
    dot_kernel<<<blocks_for(n), 256, 0, s>>>(n, x, y, sc_.p + slot);
    ADM_CK(cudaGetLastError());
    double v = 0.0;
    ADM_CK(cudaMemcpyAsync(&v, sc_.p + slot, sizeof(double), cudaMemcpyDeviceToHost, s));
    ADM_CK(cudaStreamSynchronize(s));
    return v;
  }

  // sc[slot] = x . y (device), also returned to the host
  double dot(double const *x, double const *y, int slot)
  {
    cudaStream_t const s = th_.stream_;
    dot_device(x, y, slot);
    double v = 0.0;
    ADM_CK(cudaMemcpyAsync(&v, sc_.p + slot, sizeof(double), cudaMemcpyDeviceToHost, s));
    ADM_CK(cudaStreamSynchronize(s));
    return v;
  }

  Thermal &th_;
  adm_mech_config cfg_;
  int p_ = 1, N_ = 8;
  bool ready_ = false;
  int64_t m_ = 0, n_cells_ = 0, n_dofs_ = 0;
  std::vector<uint8_t> mask_h_;
  DevBuf<int32_t> cells_;
  DevBuf<uint8_t> mask_, matid_, melted_;
  DevBuf<double> tab_;  // reference-element tables of this handle's degree
  DevBuf<double> tab1_; // and of FE_Q(1) (multigrid levels)
  DevBuf<double> coef0_d_; // FE_Q(1): (lambda, mu) per cell
  Q1Matrices kq0_{};       // and the element matrices
  std::vector<double> tab1_h_;
  std::vector<uint8_t> carry_now_; // cells that carry displacement (last setup)
  std::vector<std::unique_ptr<MgLevel>> mg_;
  int precond_ = ADM_MECH_PRECONDITIONER_MULTIGRID;
  cudaStream_t cap_stream_ = nullptr, ls_ = nullptr;
  cudaGraphExec_t vc_exec_ = nullptr; // the captured V-cycle and the CG vectors it reads and writes
  double const *vc_r_ = nullptr;
  double *vc_z_ = nullptr;
  DevBuf<double> rhs_, diag_, r_, z_, pv_, qv_, sc_;
  // J2 state of the Gauss points and the previous displacement
  DevBuf<double> kappa_, stress_, back_, u_old_;
  DevBuf<uint8_t> carry_d_;              // [2][C]: carried before, carries now
  std::vector<uint8_t> carry_prev_;      // cells that carried displacement at the last setup
  bool has_old_ = false;                 // a solve has given a previous displacement
};

} // namespace adm

struct adm_mechanics
{
  std::unique_ptr<adm::Mechanics> m;
};

extern "C" {

int adm_mechanics_create(adm_thermal *thermal, adm_mech_config const *cfg, adm_mechanics **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(thermal && cfg && out, "null argument");
    auto h = std::make_unique<adm_mechanics>();
    h->m = std::make_unique<adm::Mechanics>(*reinterpret_cast<adm::Thermal *>(thermal), *cfg);
    *out = h.release();
  });
}

int adm_mechanics_destroy(adm_mechanics *h)
{
  delete h;
  return ADM_OK;
}

int adm_mechanics_setup(adm_mechanics *h, double const *temperature)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->m->setup(temperature);
  });
}

int adm_mechanics_vmult(adm_mechanics *h, double *dst, double const *src)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst && src, "null argument");
    h->m->vmult(dst, src);
  });
}

int adm_mechanics_rhs(adm_mechanics *h, double *dst)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst, "null argument");
    h->m->copy_rhs(dst);
  });
}

int adm_mechanics_solve(adm_mechanics *h, double *displacement, int32_t *iterations, double *residual)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && displacement, "null argument");
    h->m->solve(displacement, iterations, residual);
  });
}

int adm_mechanics_set_preconditioner(adm_mechanics *h, int32_t kind)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->m->set_preconditioner(kind);
  });
}

int adm_mechanics_multigrid_levels(adm_mechanics const *h, int32_t *n_levels, int64_t *coarsest_dofs)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->m->multigrid_levels(n_levels, coarsest_dofs);
  });
}

int adm_mechanics_n_dofs(adm_mechanics const *h, int64_t *n_dofs, int64_t *n_cells)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    if (n_dofs)
      *n_dofs = h->m->n_dofs();
    if (n_cells)
      *n_cells = h->m->n_cells();
  });
}

int adm_mechanics_node_mask(adm_mechanics const *h, uint8_t *mask)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && mask, "null argument");
    std::copy(h->m->mask().begin(), h->m->mask().end(), mask);
  });
}

int adm_mechanics_stress_state(adm_mechanics *h, double *stress, double *back_stress, double *plastic)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->m->stress_state(stress, back_stress, plastic);
  });
}

} // extern "C"
