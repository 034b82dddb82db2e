// Fused cell-tile kernel of the B200 thermal hot path.
//
// One CTA owns a tile of TX x TY x TZ hex cells (one thread per cell) and
// its brick of (DEG*TX+1) x (DEG*TY+1) x (DEG*TZ+1) nodes. Per launch the
// kernel processes the tiles of one colour (tile-index parity in x, y, z), so
// no two CTAs of a launch share a node and no atomics are needed:
//  1. the node brick of the stage input is staged in shared memory;
//  2. each thread gathers its cell's nodal values and does the sum-factorized
//     interpolation to the Gauss points and the collocation gradients in
//     registers (FP64, CUDA cores: the 2x2 and 3x3 contractions are far too
//     small for tensor cores);
//  3. at every quadrature point it updates the solid/liquid/powder ratios,
//     evaluates the temperature-dependent density, specific heat (with the
//     latent-heat term) and conductivity, and the Goldak / electron-beam /
//     cube source, then integrates back in registers;
//  4. active-boundary faces add the convective / radiative terms;
//  5. the CTA sums the per-cell results per node and writes each node: the
//     first tile (in colour order) that touches a node writes it, later ones
//     add, and the last one finalizes it -- for a time step this applies the
//     inverse lumped mass and the explicit Runge-Kutta stage update in place.
//
// The arithmetic restates source/ThermalOperator.templates.hh:227-751 and
// source/MaterialProperty.hh:529-846 of the reference (adamantine v1.1.9).
#pragma once

#include "device_types.cuh"

#include <cuda.h>
#include <cuda_runtime.h>

namespace adm
{

template <int DEG>
struct TileShape;
template <>
struct TileShape<1>
{
  static constexpr int TX = 8, TY = 4, TZ = 4;
};
template <>
struct TileShape<2>
{
  static constexpr int TX = 8, TY = 4, TZ = 2;
};

// Block dimensions of the tile kernels: the tile shape of the degree, or a
// block of TZO cell layers (FE_Q(2): 4, a z-pair of tiles, in the atomic
// schedule's 128-cell variant).
template <int DEG, int TZO = TileShape<DEG>::TZ>
struct TD
{
  static constexpr int N = DEG + 1; // nodes / Gauss points per direction
  static constexpr int TX = TileShape<DEG>::TX, TY = TileShape<DEG>::TY, TZ = TZO;
  static constexpr int NCELL = TX * TY * TZ;
  // N threads per cell: thread (slab s, cell c) owns the Gauss points and the
  // nodes of z-level s of cell c
  static constexpr int NT = NCELL * N;
  // resident CTAs per SM the register budget targets (168 registers)
  static constexpr int MINB = NT > 256 ? 1 : 2;
  static constexpr int BX = DEG * TX + 1, BY = DEG * TY + 1, BZ = DEG * TZ + 1;
  // x extent of the TMA box: a multiple of 16 bytes
  static constexpr int BXP = (BX + 1) / 2 * 2;
  static constexpr int BRICK = BX * BY * BZ;
  // one staged brick (TMA box), rounded to 128 bytes
  static constexpr int BRICKP = (BXP * BY * BZ + 15) / 16 * 16;
  static constexpr int NN = N * N * N;
  static constexpr int NQS = N * N; // Gauss points (and nodes) per slab
  static constexpr int NF = N * N;
  // nodes each thread writes back
  static constexpr int WIT = (BRICK + NT - 1) / NT;
  // dynamic shared memory: two staged bricks, the level exchange
  // [NN][NCELL], the flux exchange [2][NN][NCELL], the z-shared node sums
  // [NQS][NCELL], per-cell liquid partial sums [N][NCELL] and powder-change
  // flags [2][NCELL] (one set per item parity)
  static constexpr size_t SMEM =
      sizeof(double) * (2 * BRICKP + 3 * NN * NCELL + NQS * NCELL + N * NCELL) + sizeof(int) * 2 * NCELL;
};

// ------------------------------------------------------------ TMA + mbarrier
__device__ __forceinline__ uint32_t smem_addr(void const *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async()
{
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Barrier among the N threads (a multiple of 32) that execute it with the
// same ID (1..15; 0 is __syncthreads'); compile-time ID and count, so that
// the kernel reserves only the barriers it names.
template <int ID, int N>
__device__ __forceinline__ void named_barrier()
{
  asm volatile("bar.sync %0, %1;" ::"n"(ID), "n"(N) : "memory");
}
// The barrier of z-layer group g (warp-uniform) of a tile kernel: ID 1 + g.
template <int NG, int N>
__device__ __forceinline__ void group_barrier(int g)
{
  static_assert(NG == 2 || NG == 4, "two or four z-layer groups");
  if (g == 0)
    named_barrier<1, N>();
  else if (NG == 2 || g == 1)
    named_barrier<2, N>();
  else if (g == 2)
    named_barrier<3, N>();
  else
    named_barrier<4, N>();
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, unsigned parity)
{
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(smem_addr(bar)), "r"(parity)
               : "memory");
  return ok != 0;
}
// 4D tiled TMA load of one node brick of member m (no multicast).
__device__ __forceinline__ void tma_load_brick(void *dst, CUtensorMap const *map, int x, int y, int z,
                                               int m, uint64_t *bar)
{
  asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
               " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
               "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(m), "r"(smem_addr(bar))
               : "memory");
}
// Bounded wait on an mbarrier phase: false once limit_ns nanoseconds of the
// global timer have passed without the phase completing (or, as a backstop
// should the timer stall, after kPollCap polls); the caller then reports
// DERR_TMA_TIMEOUT instead of hanging. A brick copy lands in microseconds.
constexpr long long kWaitLimitNs = 2000000000ll; // 2 s
constexpr long long kPollCap = 1ll << 32;
__device__ __forceinline__ unsigned long long globaltimer_ns()
{
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity, long long limit_ns = kWaitLimitNs)
{
  if (mbar_try_wait(bar, parity))
    return true;
  unsigned long long const t0 = globaltimer_ns();
  for (long long i = 0; i < kPollCap; ++i)
  {
    if (mbar_try_wait(bar, parity))
      return true;
    if ((long long)(globaltimer_ns() - t0) > limit_ns)
      return false;
  }
  return false;
}

// ------------------------------------------------------------ 1D contractions
// Known entries of the FE_Q(2) one-dimensional matrices. The middle Gauss
// point 1/2 is also the middle support point, so S[1] = (0, 1, 0) and
// G[1] = (-1, 0, 1) (nodal-basis derivative at 1/2 on [0, 1]), and the
// symmetric points give D[1][1] = 0 (collocation derivative); the host checks
// these entries when it builds the rule (check_q2_structure). Contractions
// skip zero entries and add or subtract for unit ones. That is exact: an FMA
// with a zero coefficient returns its addend, and one with a unit coefficient
// rounds the same sum as the addition.
enum CoefKind
{
  K_GEN = 0,
  K_ZERO,
  K_ONE,
  K_MONE
};
enum OneDMatrix
{
  M_S = 0, // S[q][i] = phi_i(x_q)
  M_G,     // G[q][i] = phi_i'(x_q)
  M_D      // D[q][j] = l_j'(x_q), Lagrange basis through the Gauss points
};
template <int DEG, int MAT>
__device__ __forceinline__ constexpr int coef_kind(int q, int k)
{
  if (DEG != 2 || q != 1)
    return K_GEN;
  if (MAT == M_S)
    return k == 1 ? K_ONE : K_ZERO;
  if (MAT == M_G)
    return k == 1 ? K_ZERO : (k == 0 ? K_MONE : K_ONE);
  return k == 1 ? K_ZERO : K_GEN;
}
// sum_k M[q][k] u[k * st] (row contraction); q and the loop index are
// compile-time constants after unrolling, so the kinds fold away
template <int DEG, int MAT>
__device__ __forceinline__ double row_dot(double const (&M)[3][3], int q, double const *u, int st)
{
  double acc = 0.0;
  bool started = false;
#pragma unroll
  for (int k = 0; k < DEG + 1; ++k)
  {
    int const kd = coef_kind<DEG, MAT>(q, k);
    double const v = u[k * st];
    if (kd == K_ZERO)
      continue;
    if (!started)
      acc = kd == K_ONE ? v : (kd == K_MONE ? -v : M[q][k] * v);
    else
      acc = kd == K_ONE ? acc + v : (kd == K_MONE ? acc - v : fma(M[q][k], v, acc));
    started = true;
  }
  return acc;
}
// sum_q M[q][n] u[q * st] (column contraction, the transpose)
template <int DEG, int MAT>
__device__ __forceinline__ double col_dot(double const (&M)[3][3], int n, double const *u, int st)
{
  double acc = 0.0;
  bool started = false;
#pragma unroll
  for (int q = 0; q < DEG + 1; ++q)
  {
    int const kd = coef_kind<DEG, MAT>(q, n);
    double const v = u[q * st];
    if (kd == K_ZERO)
      continue;
    if (!started)
      acc = kd == K_ONE ? v : (kd == K_MONE ? -v : M[q][n] * v);
    else
      acc = kd == K_ONE ? acc + v : (kd == K_MONE ? acc - v : fma(M[q][n], v, acc));
    started = true;
  }
  return acc;
}
// acc + M[q][k] * v for one entry of known kind
template <int DEG, int MAT>
__device__ __forceinline__ double entry_mac(double const (&M)[3][3], int q, int k, double v, double acc)
{
  int const kd = coef_kind<DEG, MAT>(q, k);
  return kd == K_ZERO ? acc : (kd == K_ONE ? acc + v : (kd == K_MONE ? acc - v : fma(M[q][k], v, acc)));
}

// z direction at Gauss-point level SL: the values (S) and z-gradients (G)
// from the x/y-interpolated node levels (this thread's own level in wv, the
// others in the level exchange buffer)
template <int DEG, int SL, int NCELL>
__device__ __forceinline__ void z_interp(KernelArgs const &args, double const *wv, double const *xbuf, int cl,
                                         double *Tq, double *az)
{
  constexpr int N = DEG + 1, NQS = N * N;
#pragma unroll
  for (int i = 0; i < NQS; ++i)
  {
    double w[N];
#pragma unroll
    for (int m = 0; m < N; ++m)
      w[m] = (m == SL) ? wv[i] : xbuf[(i + NQS * m) * NCELL + cl];
    Tq[i] = row_dot<DEG, M_S>(args.S, SL, w, 1);
    az[i] = row_dot<DEG, M_G>(args.G, SL, w, 1);
  }
}
// z direction into node level SL: S^T of the values / x-y fluxes and G^T of
// the z fluxes of every Gauss-point level (this thread's own in axy / az,
// the others in the flux exchange buffer)
template <int DEG, int SL, int NCELL>
__device__ __forceinline__ void z_integrate(KernelArgs const &args, double const *axy, double const *az,
                                            double const *pzbuf, int cl, double *res)
{
  constexpr int N = DEG + 1, NQS = N * N, NN = N * NQS;
#pragma unroll
  for (int i = 0; i < NQS; ++i)
  {
    double acc = 0.0;
    bool started = false;
#pragma unroll
    for (int q = 0; q < N; ++q)
    {
      double const vp = (q == SL) ? axy[i] : pzbuf[(i + NQS * q) * NCELL + cl];
      double const vz = (q == SL) ? az[i] : pzbuf[(NN + i + NQS * q) * NCELL + cl];
      int const ks = coef_kind<DEG, M_S>(q, SL), kg = coef_kind<DEG, M_G>(q, SL);
      if (ks != K_ZERO)
      {
        acc = started ? entry_mac<DEG, M_S>(args.S, q, SL, vp, acc)
                      : (ks == K_ONE ? vp : (ks == K_MONE ? -vp : args.S[q][SL] * vp));
        started = true;
      }
      if (kg != K_ZERO)
      {
        acc = started ? entry_mac<DEG, M_G>(args.G, q, SL, vz, acc)
                      : (kg == K_ONE ? vz : (kg == K_MONE ? -vz : args.G[q][SL] * vz));
        started = true;
      }
    }
    res[i] = acc;
  }
}

struct SmemPhys
{
  double poly[kMaxMaterials][kNStateProps][kMaxStates][kMaxPoly];
  double props[kMaxMaterials][kNProps];
  double latent_term[kMaxMaterials]; // L / (T_l - T_s)
  BeamState beams[kMaxBeams];
  int prop_deg[kNStateProps];
  int n_materials, use_table, isotropic, n_beams;
  int has_rotation, sources_here;
  int member;
  int role[2][27]; // per item parity
};

// ------------------------------------------------------------ properties
__device__ __forceinline__ double table_lookup(MaterialDesc const *gm, int mat,
                                               int prop, int s, double T)
{
  // MaterialProperty::compute_property_from_table
  // (source/MaterialProperty.templates.hh:1158-1212)
  double const(*t)[2] = gm->table[mat][prop][s];
  if (T <= t[0][0])
    return t[0][1];
  int i = 0;
  for (; i < kTableSize; ++i)
    if (T < t[i][0])
      break;
  if (i >= kTableSize - 1)
    return t[kTableSize - 1][1];
  return t[i - 1][1] + (T - t[i - 1][0]) * (t[i][1] - t[i - 1][1]) /
                           (t[i][0] - t[i - 1][0]);
}

// Horner evaluation of sum_i c[i] T^i up to degree deg (uniform branch).
__device__ __forceinline__ double horner(double const *c, int deg, double T)
{
  switch (deg)
  {
  case 0:
    return c[0];
  case 1:
    return fma(c[1], T, c[0]);
  case 2:
    return fma(fma(c[2], T, c[1]), T, c[0]);
  case 3:
    return fma(fma(fma(c[3], T, c[2]), T, c[1]), T, c[0]);
  default:
    return fma(fma(fma(fma(c[4], T, c[3]), T, c[2]), T, c[1]), T, c[0]);
  }
}

// Horner evaluation with a compile-time degree (higher coefficients are zero).
template <int P>
__device__ __forceinline__ double horner_fixed(double const *c, double T)
{
  double acc = c[P];
#pragma unroll
  for (int i = P - 1; i >= 0; --i)
    acc = fma(acc, T, c[i]);
  return acc;
}

// 1/x by Newton-Raphson iteration on the hardware reciprocal estimate
// (PTX rcp.approx.ftz.f64). Each step y <- y + y (1 - x y) squares the
// relative error of the estimate, so two steps bring it to the rounding
// level of double precision for normal, finite x.
__device__ __forceinline__ double recip(double x)
{
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// MaterialProperty::compute_material_property (source/MaterialProperty.hh:529-800):
// sum over states of ratio_s * property_s(T). pure >= 0 names the only state
// with a nonzero ratio (that ratio is exactly 1).
template <int NS>
__device__ __forceinline__ double property(SmemPhys const &sp,
                                           MaterialDesc const *gm, int prop,
                                           int mat, double const *r, int pure,
                                           double T)
{
  if (sp.use_table)
  {
    double v = 0.0;
#pragma unroll
    for (int s = 0; s < NS; ++s)
      v += r[s] * table_lookup(gm, mat, prop, s, T);
    return v;
  }
  int const deg = sp.prop_deg[prop];
  double const *c = &sp.poly[mat][prop][0][0];
  if (NS == 1 || pure >= 0)
    return horner(c + (NS == 1 ? 0 : pure) * kMaxPoly, deg, T);
  double m[kMaxPoly];
#pragma unroll
  for (int i = 0; i < kMaxPoly; ++i)
  {
    double a = r[0] * c[i];
#pragma unroll
    for (int s = 1; s < NS; ++s)
      a = fma(r[s], c[s * kMaxPoly + i], a);
    m[i] = a;
  }
  return horner(m, deg, T);
}

// update_state_ratios (source/ThermalOperator.templates.hh:227-317), scalar
// semantics for every quadrature point. Returns the pure state or -1.
template <int NS>
__device__ __forceinline__ int state_ratios(SmemPhys const &sp, int mat,
                                            double T, double p_old, double *r,
                                            double &liquid, double &p_new)
{
  if (NS == 1)
  {
    r[0] = 1.0;
    liquid = 0.0;
    return 0;
  }
  double const solidus = sp.props[mat][Q_SOLIDUS];
  double const liquidus = sp.props[mat][Q_LIQUIDUS];
  double l;
  if (T < solidus)
    l = 0.0;
  else if (T > liquidus)
    l = 1.0;
  else
    l = (T - solidus) / (liquidus - solidus);
  liquid = l;
  r[1] = l;
  if (NS == 2)
  {
    r[0] = 1.0 - l;
    if (l == 0.0)
      return 0;
    if (l == 1.0)
      return 1;
    return -1;
  }
  double const one_minus_l = 1.0 - l;
  double const p = (p_old < one_minus_l) ? p_old : one_minus_l; // std::min
  p_new = p;
  r[2] = p;
  r[0] = 1.0 - l - p;
  if (l == 0.0)
  {
    if (p == 0.0)
      return 0;
    if (p == 1.0)
      return 2;
    return -1;
  }
  if (l == 1.0)
    return 1; // p = min(0, p_old) = 0, s = 0
  return -1;
}

// get_inv_rho_cp (source/ThermalOperator.templates.hh:415-477), CPU latent
// heat rule liquid * solid > 0.
template <int NS>
__device__ __forceinline__ double inv_rho_cp(SmemPhys const &sp,
                                             MaterialDesc const *gm, int mat,
                                             double const *r, int pure,
                                             double T)
{
  double const rho = property<NS>(sp, gm, P_DENSITY, mat, r, pure, T);
  double cp = property<NS>(sp, gm, P_SPECIFIC_HEAT, mat, r, pure, T);
  if (NS > 1 && pure < 0)
    if (r[1] * r[0] > 0.0)
      cp += sp.latent_term[mat];
  return 1.0 / (rho * cp);
}

// Conductivity tensor and 1/(rho c_p) at one Gauss point.
struct QpCoef
{
  double inv, kxx, kxy, kyy, kzz;
};

// General material evaluation (tables, mixed states, anisotropy, rotation);
// kept out of line so that the common path stays compact.
template <int NS>
__device__ __noinline__ void qp_general(SmemPhys const &sp, MaterialDesc const *gm, int mat, double r0,
                                        double r1, double r2, int pure, double T, double cs, double sn,
                                        QpCoef &out)
{
  double const rat[3] = {r0, r1, r2};
  out.inv = inv_rho_cp<NS>(sp, gm, mat, rat, pure, T);
  double const kx = property<NS>(sp, gm, P_KX, mat, rat, pure, T);
  double const ky = sp.isotropic ? kx : property<NS>(sp, gm, P_KY, mat, rat, pure, T);
  double const kz = sp.isotropic ? kx : property<NS>(sp, gm, P_KZ, mat, rat, pure, T);
  // rotation by the deposition angle (source/ThermalOperator.templates.hh:552-594)
  out.kxx = kx * cs * cs + ky * sn * sn;
  out.kxy = (kx - ky) * sn * cs;
  out.kyy = kx * sn * sn + ky * cs * cs;
  out.kzz = kz;
}

// Scalar GoldakHeatSource::value / ElectronBeamHeatSource::value /
// CubeHeatSource::value (source/GoldakHeatSource.cc:46-89,
// source/ElectronBeamHeatSource.cc:47-93, source/CubeHeatSource.cc:51-71).
__device__ __forceinline__ double beam_value(BeamState const &b, double px,
                                             double py, double pz)
{
  if (b.type == 2)
  {
    if (!b.on)
      return 0.0;
    if (px < b.cube_min[0] || px > b.cube_max[0] || py < b.cube_min[1] ||
        py > b.cube_max[1] || pz < b.cube_min[2] || pz > b.cube_max[2])
      return 0.0;
    return b.cube_value;
  }
  double const z = pz - b.center[2];
  if (z + b.depth < 0.0)
    return 0.0;
  double const dx = px - b.center[0], dy = py - b.center[1];
  double const xpy = dx * dx + dy * dy;
  if (xpy > b.five_r2)
    return 0.0;
  if (b.type == 0)
    return b.alpha * exp(-3.0 * xpy * b.inv_r2 + -3.0 * (z * z) * b.inv_d2);
  double const z_rel = z * b.inv_d;
  double const dist_z = -3.0 * (z_rel * z_rel) - 2.0 * z_rel + 1.0;
  return b.alpha * exp(b.log01 * xpy * b.inv_r2) * dist_z;
}

// Sum of all heat sources at a point (out of line: only tiles near a beam
// call it).
static __device__ __noinline__ double beam_sum(SmemPhys const &sp, double px, double py, double pz)
{
  double qs = 0.0;
  for (int b = 0; b < sp.n_beams; ++b)
    qs += beam_value(sp.beams[b], px, py, pz);
  return qs;
}

// The quadrature points of one node level of a cell on the general path
// (update_state_ratios, get_inv_rho_cp and the conductivity of
// source/ThermalOperator.templates.hh:227-617): per point the phase-state
// update with its history write, the material evaluation (pure-state
// polynomials inline, everything else in qp_general), the fluxes and their
// collocation D^T in x/y, and the source. Tq holds the level's temperatures,
// az its z-gradients on entry and the z fluxes on return; axy accumulates.
template <int DEG, int NS, int P>
__device__ __noinline__ void general_level(SmemPhys const &sp, MaterialDesc const *gm, MemberData const &md,
                                           KernelArgs const &args, int mat, int slab, int cold, int pmode,
                                           double pu, size_t pbase, double cs, double sn, bool fast_ok,
                                           bool do_src, int cx, int cy, int cz, double const *__restrict__ Tq,
                                           double *__restrict__ az, double *__restrict__ axy,
                                           double *__restrict__ liquid_out, uint32_t *__restrict__ changed_out)
{
  constexpr int N = DEG + 1, NQS = N * N;
  constexpr int PS = kMaxStates * kMaxPoly; // stride between properties
  double const solidus = sp.props[mat][Q_SOLIDUS];
  double const *cold_c = &sp.poly[mat][0][cold < 0 ? 0 : cold][0];
  double const *cw = &args.cw[NQS * slab][0];
  double liquid_acc = 0.0;
  uint32_t changed_mask = 0;
#pragma unroll
  for (int i = 0; i < NQS; ++i)
  {
    int const qa = i % N, qb = i / N;
    double const T = Tq[i];
    double const gx = row_dot<DEG, M_D>(args.D, qa, &Tq[N * qb], 1);
    double const gy = row_dot<DEG, M_D>(args.D, qb, &Tq[qa], N);
    double const gz = az[i];
    double inv, fx, fy, fz;
    if (cold >= 0 && (NS == 1 || T < solidus))
    {
      // one state, polynomial, isotropic: Horner in that state only; cw
      // holds W_q * vol / h_d^2 and W_q * vol for this point
      double const rho = horner_fixed<P>(cold_c + P_DENSITY * PS, T);
      double const cp = horner_fixed<P>(cold_c + P_SPECIFIC_HEAT * PS, T);
      inv = recip(rho * cp);
      double const cf = -inv * horner_fixed<P>(cold_c + P_KX * PS, T);
      fx = (cf * cw[4 * i + 0]) * gx;
      fy = (cf * cw[4 * i + 1]) * gy;
      fz = (cf * cw[4 * i + 2]) * gz;
    }
    else
    {
      double p_old = 0.0;
      if (NS == 3)
        p_old = (pmode == 2) ? md.powder_q[pbase + i] : pu;
      double r0, r1 = 0.0, r2 = 0.0;
      double liquid = 0.0, p_new = p_old;
      int pure;
      {
        double rat[NS > 1 ? NS : 1];
        pure = state_ratios<NS>(sp, mat, T, p_old, rat, liquid, p_new);
        r0 = rat[0];
        if (NS > 1)
          r1 = rat[1];
        if (NS > 2)
          r2 = rat[NS > 2 ? 2 : 0];
      }
      if (NS > 1)
        liquid_acc += liquid;
      if (NS == 3 && p_new != p_old)
      {
        md.powder_q[pbase + i] = p_new;
        changed_mask |= 1u << i;
      }
      double kxx, kxy, kyy, kzz;
      if (fast_ok && pure >= 0)
      {
        double const *cc = &sp.poly[mat][0][NS == 1 ? 0 : pure][0];
        double const rho = horner_fixed<P>(cc + P_DENSITY * PS, T);
        double const cp = horner_fixed<P>(cc + P_SPECIFIC_HEAT * PS, T);
        inv = recip(rho * cp);
        kxx = horner_fixed<P>(cc + P_KX * PS, T);
        kyy = kxx;
        kzz = kxx;
        kxy = 0.0;
      }
      else
      {
        QpCoef kk;
        qp_general<NS>(sp, gm, mat, r0, r1, r2, pure, T, cs, sn, kk);
        inv = kk.inv;
        kxx = kk.kxx;
        kxy = kk.kxy;
        kyy = kk.kyy;
        kzz = kk.kzz;
      }
      double const W = args.qw[qa] * args.qw[qb] * args.qw[slab];
      double const grx = gx * args.inv_h[0], gry = gy * args.inv_h[1];
      double const cf = -inv * W;
      fx = cf * (kxx * grx + kxy * gry) * args.vol_over_h[0];
      fy = cf * (kxy * grx + kyy * gry) * args.vol_over_h[1];
      fz = cf * kzz * gz * args.vol_over_h2[2];
    }
    az[i] = fz;
#pragma unroll
    for (int m = 0; m < N; ++m)
    {
      axy[m + N * qb] = entry_mac<DEG, M_D>(args.D, qa, m, fx, axy[m + N * qb]);
      axy[qa + N * m] = entry_mac<DEG, M_D>(args.D, qb, m, fy, axy[qa + N * m]);
    }
    if (do_src)
    {
      double const px = (args.origin[0] + cx * args.h[0]) + args.qx[qa] * args.h[0];
      double const py = (args.origin[1] + cy * args.h[1]) + args.qx[qb] * args.h[1];
      double const pz = (args.origin[2] + cz * args.h[2]) + args.qx[slab] * args.h[2];
      axy[i] += beam_sum(sp, px, py, pz) * inv * cw[4 * i + 3];
    }
  }
  *liquid_out = liquid_acc;
  *changed_out = changed_mask;
}

// Convective / radiative face terms of one cell (face_local_apply,
// source/ThermalOperator.templates.hh:619-751) for the node level `slab`:
// every level thread of a cell evaluates the face quadrature and keeps the
// test functions of its own level; out[e] receives the contribution to the
// level's node e.
template <int DEG, int NS>
__device__ __noinline__ void face_terms(SmemPhys const &sp, MaterialDesc const *gm, MemberData const &md,
                                        KernelArgs const &args, double const *brick, int lx, int ly, int lz,
                                        int slab, uint32_t info, int mat, size_t c, double *out)
{
  constexpr int N = DEG + 1, NQS = N * N;
  constexpr int BXP = TD<DEG>::BXP, BY = TD<DEG>::BY;
  for (int e = 0; e < NQS; ++e)
    out[e] = 0.0;
  int const slot = (NS == 3) ? md.face_slot[c] : -1;
  for (int f = 0; f < 6; ++f)
  {
    if (!((info >> (CI_FACE_SHIFT + f)) & 1u))
      continue;
    int const d = f / 2, side = f % 2;
    if (d == 2 && slab != (side ? N - 1 : 0))
      continue; // a z face only touches one node level
    int const t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
    int const btype =
        ((info >> (CI_INTERFACE_SHIFT + f)) & 1u) ? args.interface_type : args.boundary_type[f];
    double const ht0 = args.h[t0], ht1 = args.h[t1];
    for (int fq = 0; fq < N * N; ++fq)
    {
      int const qa = fq % N, qb = fq / N;
      double T = 0.0;
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
        {
          int loc[3];
          loc[d] = side ? N - 1 : 0;
          loc[t0] = i;
          loc[t1] = j;
          double const u = brick[(DEG * lx + loc[0]) + BXP * ((DEG * ly + loc[1]) + BY * (DEG * lz + loc[2]))];
          T += args.S[qa][i] * args.S[qb][j] * u;
        }
      double rat[NS > 1 ? NS : 1];
      double liquid = 0.0, p_old = 0.0, p_new = 0.0;
      double *ph = nullptr;
      if (NS == 3 && slot >= 0)
      {
        ph = &md.face_powder[((size_t)slot * 6 + f) * (N * N) + fq];
        p_old = *ph;
      }
      int const pure = state_ratios<NS>(sp, mat, T, p_old, rat, liquid, p_new);
      // p_new = min(1 - l, p_old) is idempotent, so the other level threads
      // of this cell compute the same value whether they read the history
      // before or after this store
      if (ph && (d == 2 || slab == 0) && p_new != p_old)
        *ph = p_new;
      double const inv = inv_rho_cp<NS>(sp, gm, mat, rat, pure, T);
      double conv_tinf = 0.0, conv_h = 0.0, rad_tinf = 0.0, rad_h = 0.0;
      if (btype & B_CONVECTIVE)
      {
        conv_tinf = sp.props[mat][Q_CONV_TINF];
        conv_h = property<NS>(sp, gm, P_CONV_COEF, mat, rat, pure, T);
      }
      if (btype & B_RADIATIVE)
      {
        rad_tinf = sp.props[mat][Q_RAD_TINF];
        rad_h = property<NS>(sp, gm, P_EMISSIVITY, mat, rat, pure, T) * 5.670374419e-8 * (T + rad_tinf) *
                (T * T + rad_tinf * rad_tinf);
      }
      double const bval = -inv * (conv_h * (T - conv_tinf) + rad_h * (T - rad_tinf));
      double const JxW = args.qw[qa] * ht0 * args.qw[qb] * ht1;
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
        {
          // node (la, lb, lc) of this face; kept if it is on level `slab`
          int const la = d == 0 ? (side ? N - 1 : 0) : i;
          int const lb = d == 0 ? i : (d == 1 ? (side ? N - 1 : 0) : j);
          int const lc = d == 2 ? (side ? N - 1 : 0) : j;
          if (lc != slab)
            continue;
          out[la + N * lb] += bval * (args.S[qa][i] * args.S[qb][j]) * JxW;
        }
    }
  }
}

// Role of a node class of a tile whose sharing state per direction is
// (s0, s1, s2) (0 not shared, 1 shared with the lower neighbour tile, 2 with
// the upper one), from the tile's neighbour-activity mask nbr and colour.
// Coloured schedule: bit 1 first and bit 2 last toucher in colour order.
__device__ __forceinline__ int node_role(uint32_t nbr, int colour, int s0, int s1, int s2)
{
  int cmin = 8, cmax = -1;
#pragma unroll
  for (int m = 0; m < 8; ++m)
  {
    int const b0 = m & 1, b1 = (m >> 1) & 1, b2 = (m >> 2) & 1;
    if ((b0 && s0 == 0) || (b1 && s1 == 0) || (b2 && s2 == 0))
      continue;
    int const o0 = b0 ? (s0 == 1 ? -1 : 1) : 0;
    int const o1 = b1 ? (s1 == 1 ? -1 : 1) : 0;
    int const o2 = b2 ? (s2 == 1 ? -1 : 1) : 0;
    int const bit = (o0 + 1) + 3 * (o1 + 1) + 9 * (o2 + 1);
    if (!((nbr >> bit) & 1u))
      continue;
    int const c = colour ^ (b0 | (b1 << 1) | (b2 << 2));
    cmin = c < cmin ? c : cmin;
    cmax = c > cmax ? c : cmax;
  }
  return (colour == cmin ? 1 : 0) | (colour == cmax ? 2 : 0);
}

// Two-pass schedule: the halo array of a tile holds one partial sum per node
// on its upper brick faces that an upper neighbour tile owns, in three full
// faces: z (x = 0..BX-1, y = 0..BY-1), y (x, z) and x (y, z). A node shared
// with the upper z neighbour sits in the z face, else one shared with the
// upper y neighbour in the y face, else in the x face -- a rule both the
// writing tile (from its sharing state) and the gather (from the offset of
// the lower neighbour it reads) apply without looking at coordinates.
template <int BX, int BY, int BZ>
struct HaloLayout
{
  static constexpr int RZ = 0, RY = BX * BY, RX = BX * BY + BX * BZ;
  static constexpr int SIZE = BX * BY + BX * BZ + BY * BZ;
  // brick-local node (X, Y, Z), shared upward in z (uz), else y (uy), else x
  __host__ __device__ static int index(bool uz, bool uy, int X, int Y, int Z)
  {
    return uz ? RZ + X + BX * Y : (uy ? RY + X + BX * Z : RX + Y + BY * Z);
  }
};
template <int DEG>
using HaloOf = HaloLayout<TD<DEG>::BX, TD<DEG>::BY, TD<DEG>::BZ>;

// Launch schedules of the tile kernels (template parameter SC).
enum Schedule : int
{
  SC_COLOURED = 0,
  SC_ATOMIC = 1,
  SC_TWO_PASS = 2
};

// Two-pass role and halo slot of a node this thread writes, from its
// brick-local coordinates and sharing state per direction (2: shared with
// the upper neighbour tile, which owns it). Returns 8 (partial sum into the
// halo array at *slot) or 4 (the tile's own node).
template <class HL>
__device__ __forceinline__ int two_pass_slot(int X, int Y, int Z, int sx, int sy, int sz, int *slot)
{
  if (sx != 2 && sy != 2 && sz != 2)
    return 4;
  *slot = HL::index(sz == 2, sy == 2, X, Y, Z);
  return 8;
}

// Two-pass write-out (rl[i]: 4 own node, 8 halo node at slot[i], 0 none):
// stores only (vmult mode 1 adds to dst). The owner's partial sum goes to
// dst (vmult) or to the stage accumulator; the gather pass completes it.
template <class HL, int NV>
__device__ __forceinline__ void write_nodes_two_pass(KernelArgs const &args, MemberData const &md, int tile,
                                                     double const *res, int const *rl, size_t const *gidx,
                                                     int const *slot)
{
  double *const tgt = args.mode == 2 ? md.acc : args.vdst;
  double *const halo = md.halo + (size_t)tile * HL::SIZE;
  uint64_t const pol = l2_policy_evict_last(); // the gather pass reads the halo next
  double old[NV];
#pragma unroll
  for (int i = 0; i < NV; ++i)
    old[i] = (args.mode == 1 && rl[i] == 4) ? tgt[gidx[i]] : 0.0;
#pragma unroll
  for (int i = 0; i < NV; ++i)
  {
    if (rl[i] == 8)
      st_keep(halo + slot[i], res[i], pol);
    else if (rl[i] == 4)
      tgt[gidx[i]] = old[i] + res[i];
  }
}

// Write-out of the node sums res[i] of one thread (rl[i]: bit 4 the thread
// owns the node, bit 1 / 2 first / last toucher in colour order; gidx[i]:
// its index in the node vector). Atomic schedule: added into the zeroed
// target. Coloured schedule: the first toucher writes, later ones add (acc),
// the last one finalizes -- vmult writes dst, a stage applies the inverse
// lumped mass and the explicit Runge-Kutta update. All loads, then stores.
template <bool AT, int NV>
__device__ __forceinline__ void write_nodes(KernelArgs const &args, MemberData const &md, double *y,
                                            double const *res, int const *rl, size_t const *gidx)
{
  if constexpr (AT)
  {
    double *const tgt = args.mode == 2 ? md.acc : args.vdst;
#pragma unroll
    for (int i = 0; i < NV; ++i)
      if (rl[i] & 4)
        atomicAdd(&tgt[gidx[i]], res[i]);
  }
  else if (args.mode == 0 || args.mode == 1)
  {
    double old[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i)
      old[i] = ((rl[i] & 4) && (args.mode == 1 || !(rl[i] & 1))) ? args.vdst[gidx[i]] : 0.0;
#pragma unroll
    for (int i = 0; i < NV; ++i)
      if (rl[i] & 4)
        args.vdst[gidx[i]] = old[i] + res[i];
  }
  else
  {
    double const dt = md.clock[1];
    double *const znext = args.dst_sel == 1 ? md.za : md.zb;
    double pa[NV], im[NV], yv[NV], sv[NV], fv[NV];
#pragma unroll
    for (int i = 0; i < NV; ++i)
    {
      bool const valid = rl[i] & 4, first = rl[i] & 1, last = rl[i] & 2;
      size_t const g = gidx[i];
      pa[i] = (valid && !first) ? md.acc[g] : 0.0;
      im[i] = (valid && last) ? md.inv_mass[g] : 0.0;
      yv[i] = (valid && last) ? y[g] : 0.0;
      sv[i] = (valid && last && args.n_stages > 1 && (args.stage > 0)) ? md.s[g] : 0.0;
      fv[i] = (valid && last && args.has_f0) ? md.f0[g] : 0.0;
    }
#pragma unroll
    for (int i = 0; i < NV; ++i)
    {
      if (!(rl[i] & 4))
        continue;
      size_t const g = gidx[i];
      double const total = pa[i] + res[i];
      if (!(rl[i] & 2))
      {
        md.acc[g] = total;
        continue;
      }
      double const f = im[i] * total;
      if (!isfinite(f))
        atomicCAS(md.error, 0, (int)DERR_NONFINITE);
      if (args.n_stages == 1)
      {
        y[g] = yv[i] + dt * f;
      }
      else if (!args.last)
      {
        double zn = yv[i];
        if (args.has_f0)
          zn = zn + (dt * args.a_next_f0) * fv[i];
        zn = zn + (dt * args.a_next) * f;
        znext[g] = zn;
        double const sb = (dt * args.b_i) * f;
        md.s[g] = args.stage == 0 ? sb : sv[i] + sb;
        if (args.store_f0)
          md.f0[g] = f;
      }
      else
      {
        y[g] = yv[i] + (sv[i] + (dt * args.b_i) * f);
      }
    }
  }
}

// ------------------------------------------------------------ the kernel
// Loads the physics constants of a member into shared memory.
template <int NT>
__device__ __forceinline__ void load_member_constants(SmemPhys &sp, MemberData const &md, int tid)
{
  MaterialDesc const *gm = md.mat;
  int const nm = gm->n_materials;
  double const *gp = &gm->poly[0][0][0][0];
  double *spp = &sp.poly[0][0][0][0];
  int const npoly = nm * kNStateProps * kMaxStates * kMaxPoly;
  for (int i = tid; i < npoly; i += NT)
    spp[i] = gp[i];
  for (int i = tid; i < nm * kNProps; i += NT)
    (&sp.props[0][0])[i] = (&gm->props[0][0])[i];
  if (tid < nm)
  {
    double const Tl = gm->props[tid][Q_LIQUIDUS], Ts = gm->props[tid][Q_SOLIDUS];
    sp.latent_term[tid] = gm->props[tid][Q_LATENT] / (Tl - Ts);
  }
  if (tid < kNStateProps)
    sp.prop_deg[tid] = gm->prop_deg[tid];
  if (tid < md.n_beams)
    sp.beams[tid] = md.beam_state[tid];
  if (tid == 0)
  {
    sp.n_materials = nm;
    sp.use_table = gm->use_table;
    sp.isotropic = gm->isotropic;
    sp.n_beams = md.n_beams;
    sp.has_rotation = md.has_rotation;
  }
}

// The persistent tile loop: CTA b processes work items b, b + grid, ... of
// one colour. The node brick of the next item is fetched by TMA into the
// other buffer while the current item is computed.
// FC: the problem has convective / radiative faces (instantiated apart so
// that adiabatic problems carry no face code).
template <int DEG, int NS, int P, int SC, bool FC, int TZO = TileShape<DEG>::TZ>
__global__ void __launch_bounds__(TD<DEG, TZO>::NT, TD<DEG, TZO>::MINB)
    tile_kernel(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ KernelArgs args, int n_items)
{
  using T_ = TD<DEG, TZO>;
  constexpr int N = T_::N, NN = T_::NN, NT = T_::NT, NCELL = T_::NCELL, NQS = T_::NQS;
  constexpr int TX = T_::TX, TY = T_::TY, TZ = T_::TZ;
  constexpr int BX = T_::BX, BY = T_::BY, BZ = T_::BZ, BXP = T_::BXP;
  constexpr int WIT = T_::WIT;
  constexpr unsigned kBoxBytes = sizeof(double) * BXP * BY * BZ;
  extern __shared__ __align__(128) double smem[];
  double *const xbuf = smem + 2 * T_::BRICKP;  // [NN][NCELL]: level exchange
  double *const pzbuf = xbuf + NN * NCELL;     // [2][NN][NCELL]: flux exchange
  double *const mbuf = pzbuf + 2 * NN * NCELL; // [NQS][NCELL]: z-shared node sums
  double *const lsum = mbuf + NQS * NCELL;     // [N][NCELL]
  int *const changed_p = reinterpret_cast<int *>(lsum + N * NCELL); // [2][NCELL]
  __shared__ SmemPhys sp;
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int src_on_g[T_::TZ]; // per z-layer group: the item's tile meets a source

  int const tid = threadIdx.x;
  int const slab = tid / NCELL, cl = tid % NCELL;
  int const lx = cl % TX, ly = (cl / TX) % TY, lz = cl / (TX * TY);
  int const nt0 = args.nt[0], nt1 = args.nt[1];
  int const pitch = args.pitch, nn1 = args.nn[1];

  auto issue = [&](int buf, int item) {
    TileWork const wi = args.work[item];
    int const tix = wi.xyz & 2047u, tiy = (wi.xyz >> 11) & 2047u, tiz = wi.xyz >> 22;
    mbar_arrive_expect_tx(&bars[buf], kBoxBytes);
    tma_load_brick(smem + buf * T_::BRICKP, &tmap, DEG * TX * tix, DEG * TY * tiy, DEG * TZ * tiz,
                   wi.member, &bars[buf]);
  };

  // work distribution: with args.claim (and a list that is not blocked),
  // dynamic -- CTA b starts with item b and claims each further item from
  // the launch's counter, one item ahead (a CTA held up by a slow tile, near
  // the melt pool, takes fewer; the lists put the top tile layers first); else
  // strided (CTA b takes items b, b + grid, ...) or, with args.blocked, one
  // contiguous run of items per CTA (consecutive items of a member-major
  // list then share the member's constants)
  bool const dyn = args.claim != nullptr && !args.blocked;
  __shared__ int claimed[2]; // dynamic: the item after the current one, by item parity
  int first, last, step;
  if (dyn || !args.blocked)
  {
    first = blockIdx.x;
    last = n_items;
    step = gridDim.x;
  }
  else
  {
    int const per = (n_items + (int)gridDim.x - 1) / (int)gridDim.x;
    first = (int)blockIdx.x * per;
    last = min(first + per, n_items);
    step = 1;
  }
  if (tid == 0)
  {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
    sp.member = -1;
    if (dyn)
      claimed[1] = first < last ? atomicAdd(args.claim, 1) + (int)gridDim.x : last;
  }
  __syncthreads();
  if (tid == 0 && first < last)
    issue(0, first);

  // The work item and this thread's cell data (info word, powder mode and
  // uniform powder value) are loaded one item ahead, so that their
  // dependent global loads overlap the previous item's arithmetic.
  TileWork nx_w{0, 0, 0u};
  uint32_t nx_info = 0u;
  int nx_pmode = 0;
  double nx_pu = 0.0;
  auto load_item = [&](int item2) {
    nx_w = args.work[item2];
    MemberData const &mk = args.members[nx_w.member];
    int const kx = TX * (int)(nx_w.xyz & 2047u) + lx, ky = TY * (int)((nx_w.xyz >> 11) & 2047u) + ly,
              kz = TZ * (int)(nx_w.xyz >> 22) + lz;
    nx_info = 0u;
    nx_pmode = 0;
    nx_pu = 0.0;
    if (kx < args.nc[0] && ky < args.nc[1] && kz < args.nc[2])
    {
      size_t const kc = kx + (size_t)args.nc[0] * (ky + (size_t)args.nc[1] * kz);
      nx_info = mk.cell_info[kc];
      if (NS == 3)
      {
        // both loaded unconditionally: a load that waited for the mode
        // would stall the thread here
        nx_pmode = mk.powder_mode[kc];
        nx_pu = mk.powder_cell[kc];
      }
    }
  };
  if (first < last)
    load_item(first);

  int it = 0;
  for (int item = first; item < last; ++it)
  {
    int const buf = it & 1;
    // the next item: claimed during the previous one (published by its
    // barriers), or the next of the static distribution
    int const next = dyn ? claimed[(it + 1) & 1] : item + step;
    double const *brick = smem + buf * T_::BRICKP;
    TileWork const w = nx_w;
    uint32_t const cur_info = nx_info;
    int const cur_pmode = nx_pmode;
    double const cur_pu = nx_pu;
    if (next < last)
      load_item(next);
    MemberData const &md = args.members[w.member];
    MaterialDesc const *gm = md.mat;
    int const tile = w.tile;
    int const tix = w.xyz & 2047u, tiy = (w.xyz >> 11) & 2047u, tiz = w.xyz >> 22;
    int const colour = (tix & 1) | ((tiy & 1) << 1) | ((tiz & 1) << 2);
    int const ncx0 = TX * tix, ncy0 = TY * tiy, ncz0 = TZ * tiz;      // first cell
    int const nx0 = DEG * ncx0, ny0 = DEG * ncy0, nz0 = DEG * ncz0; // first node
    double *const y = args.y_override ? args.y_override : md.y;
    // Three CTA barriers per item: the level exchange (which also publishes
    // this item's roles and cleared flags and carries the brick-timeout
    // vote), the flux exchange and the z-shared node sums. Per-item shared
    // state that a thread still finishing the previous item may read (roles,
    // powder-change flags) alternates between two copies by item parity;
    // the next brick is requested after the first barrier, when every
    // thread has finished the previous item and no longer reads its buffer.
    int *const changed = changed_p + buf * NCELL;
    if (sp.member != w.member)
    {
      load_member_constants<NT>(sp, md, tid);
      __syncthreads();
      if (tid == 0)
        sp.member = w.member;
    }
    if (SC == SC_COLOURED && tid < 27)
    {
      // the role of the node class (tid % 3, tid / 3 % 3, tid / 9): sharing
      // state per direction, 0 not shared, 1 with the lower neighbour tile,
      // 2 with the upper one
      sp.role[buf][tid] = node_role(md.tile_nbr[tile], colour, tid % 3, (tid / 3) % 3, tid / 9);
    }
    if (slab == 0)
      changed[cl] = 0;
    // wait for this item's brick (bounded; every thread polls); a thread
    // whose wait gave up computes on whatever the buffer holds and the vote
    // at the level-exchange barrier ends the CTA before anything is written
    bool const arrived = mbar_wait(&bars[buf], (unsigned)((it >> 1) & 1));

    // Tile-level source culling (exact: it skips only points where every
    // source is zero by its own cutoff rules), evaluated by the first warp
    // of each z-layer group (slab 0) for its group and published through
    // the group's level-exchange barrier. A warp that writes its group's
    // flag for the next item has passed the node barrier of this one, after
    // which nobody reads it.
    if (slab == 0)
    {
      bool do_src = false;
      double const x0 = args.origin[0] + ncx0 * args.h[0];
      double const y0 = args.origin[1] + ncy0 * args.h[1];
      double const z0 = args.origin[2] + ncz0 * args.h[2];
      double const x1 = x0 + TX * args.h[0], y1 = y0 + TY * args.h[1], z1 = z0 + TZ * args.h[2];
      for (int b = 0; b < sp.n_beams; ++b)
      {
        BeamState const &bs = sp.beams[b];
        if (!bs.on)
          continue;
        if (bs.type == 2)
        {
          if (x1 >= bs.cube_min[0] && x0 <= bs.cube_max[0] && y1 >= bs.cube_min[1] &&
              y0 <= bs.cube_max[1] && z1 >= bs.cube_min[2] && z0 <= bs.cube_max[2])
            do_src = true;
          continue;
        }
        if ((z1 - bs.center[2]) + bs.depth < 0.0)
          continue;
        double const qx = fmin(fmax(bs.center[0], x0), x1);
        double const qy = fmin(fmax(bs.center[1], y0), y1);
        double const dx = qx - bs.center[0], dy = qy - bs.center[1];
        if (dx * dx + dy * dy > bs.five_r2 * (1.0 + 1e-9))
          continue;
        do_src = true;
      }
      if ((tid & 31) == 0)
        src_on_g[lz] = do_src;
    }

    // ---- the cell: thread (slab, cl) handles Gauss-point level qc = slab
    int const cx = ncx0 + lx, cy = ncy0 + ly, cz = ncz0 + lz;
    bool const in_domain = cx < args.nc[0] && cy < args.nc[1] && cz < args.nc[2];
    size_t const c = in_domain ? cx + (size_t)args.nc[0] * (cy + (size_t)args.nc[1] * cz) : 0;
    uint32_t const info = cur_info;
    bool const active = (info & CI_ACTIVE) != 0;
    int const mat = (info >> CI_MAT_SHIFT) & 15;
    // 1. x/y interpolation of the nodes of z-level `slab` (in registers)
    double wv[NQS];
    {
#pragma unroll
      for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = 0; i < N; ++i)
          wv[i + N * j] = brick[(DEG * lx + i) + BXP * ((DEG * ly + j) + BY * (DEG * lz + slab))];
#pragma unroll
      for (int j = 0; j < N; ++j)
      {
        double t[N];
#pragma unroll
        for (int q = 0; q < N; ++q)
          t[q] = row_dot<DEG, M_S>(args.S, q, &wv[N * j], 1);
#pragma unroll
        for (int q = 0; q < N; ++q)
          wv[q + N * j] = t[q];
      }
#pragma unroll
      for (int i = 0; i < N; ++i)
      {
        double t[N];
#pragma unroll
        for (int q = 0; q < N; ++q)
          t[q] = row_dot<DEG, M_S>(args.S, q, &wv[i], N);
#pragma unroll
        for (int q = 0; q < N; ++q)
          wv[i + N * q] = t[q];
      }
    }
    // 2. exchange the levels: values T and z-gradients gz (G = D S) at this
    //    thread's Gauss-point level. The N level threads of a cell are in
    //    the cell's z-layer group (its N warps), so the exchange needs only
    //    that group's barrier; the other group goes on.
#pragma unroll
    for (int i = 0; i < NQS; ++i)
      xbuf[(i + NQS * slab) * NCELL + cl] = wv[i];
    group_barrier<TZ, NT / TZ>(lz);
    // prefetch the next item's brick into the other buffer, and claim the
    // item after it (read at the start of the next item, after this item's
    // flux and node barriers; the slot's previous value was read at the
    // start of the previous item)
    if (tid == 0)
    {
      if (next < last)
      {
        fence_proxy_async();
        issue(buf ^ 1, next);
      }
      if (dyn)
        claimed[it & 1] = next < last ? atomicAdd(args.claim, 1) + (int)gridDim.x : last;
    }
    bool const do_src = src_on_g[lz] != 0;
    double Tq[NQS], az[NQS];
    // (a warp-uniform branch: a warp's threads share the level)
    if (slab == 0)
      z_interp<DEG, 0, NCELL>(args, wv, xbuf, cl, Tq, az);
    else if (DEG == 1 || slab == 1)
      z_interp<DEG, 1, NCELL>(args, wv, xbuf, cl, Tq, az);
    else
      z_interp<DEG, DEG, NCELL>(args, wv, xbuf, cl, Tq, az);
    // 3. physics at the NQS Gauss points of this level; axy accumulates the
    //    x/y flux contributions (collocation D^T) and the source, az ends
    //    up holding the z fluxes
    double axy[NQS];
#pragma unroll
    for (int i = 0; i < NQS; ++i)
      axy[i] = 0.0;
    double liquid_acc = 0.0;
    uint32_t changed_mask = 0;
    int pmode = 0;
    double pu = 0.0;
    if (active)
    {
      size_t const pbase = c * NN + (size_t)NQS * slab;
      if (NS == 3)
      {
        pmode = cur_pmode;
        if (pmode == 1)
          pu = cur_pu;
      }
      double cs = 1.0, sn = 0.0;
      if (sp.has_rotation)
      {
        cs = md.cosv[c];
        sn = md.sinv[c];
      }
      bool const fast_ok = !sp.use_table && sp.isotropic && !sp.has_rotation;
      // Below the solidus the liquid ratio is 0 and the powder ratio keeps
      // its value (min(1, p) = p), so a cell whose powder ratio is uniformly
      // 0 or 1 is in one pure state there: `cold` names it (or -1).
      double const solidus = sp.props[mat][Q_SOLIDUS];
      int cold = -1;
      if (fast_ok)
      {
        if (NS == 1)
          cold = 0;
        else if (NS == 2)
          cold = 0;
        else if (pmode == 0)
          cold = 0;
        else if (pmode == 1 && pu == 1.0)
          cold = 2;
      }
      constexpr int PS = kMaxStates * kMaxPoly; // stride between properties
      double const *cold_c = &sp.poly[mat][0][cold < 0 ? 0 : cold][0];
      double const *cw = &args.cw[NQS * slab][0];
      // every point of this level cold: one straight-line pass (no branch
      // per point, so the points' dependency chains interleave)
      bool all_cold = cold >= 0;
      if (NS > 1)
      {
#pragma unroll
        for (int i = 0; i < NQS; ++i)
          all_cold &= Tq[i] < solidus;
      }
      if (all_cold)
      {
        double crho[P + 1], ccp[P + 1], ck[P + 1];
#pragma unroll
        for (int k = 0; k <= P; ++k)
        {
          crho[k] = cold_c[P_DENSITY * PS + k];
          ccp[k] = cold_c[P_SPECIFIC_HEAT * PS + k];
          ck[k] = cold_c[P_KX * PS + k];
        }
#pragma unroll
        for (int i = 0; i < NQS; ++i)
        {
          int const qa = i % N, qb = i / N;
          double const T = Tq[i];
          double const gx = row_dot<DEG, M_D>(args.D, qa, &Tq[N * qb], 1);
          double const gy = row_dot<DEG, M_D>(args.D, qb, &Tq[qa], N);
          double const inv = recip(horner_fixed<P>(crho, T) * horner_fixed<P>(ccp, T));
          double const cf = -inv * horner_fixed<P>(ck, T);
          double const fx = (cf * cw[4 * i + 0]) * gx;
          double const fy = (cf * cw[4 * i + 1]) * gy;
          az[i] = (cf * cw[4 * i + 2]) * az[i];
#pragma unroll
          for (int m = 0; m < N; ++m)
          {
            axy[m + N * qb] = entry_mac<DEG, M_D>(args.D, qa, m, fx, axy[m + N * qb]);
            axy[qa + N * m] = entry_mac<DEG, M_D>(args.D, qb, m, fy, axy[qa + N * m]);
          }
        }
        if (do_src)
        {
#pragma unroll
          for (int i = 0; i < NQS; ++i)
          {
            int const qa = i % N, qb = i / N;
            double const T = Tq[i];
            double const inv = recip(horner_fixed<P>(crho, T) * horner_fixed<P>(ccp, T));
            double const px = (args.origin[0] + cx * args.h[0]) + args.qx[qa] * args.h[0];
            double const py = (args.origin[1] + cy * args.h[1]) + args.qx[qb] * args.h[1];
            double const pz = (args.origin[2] + cz * args.h[2]) + args.qx[slab] * args.h[2];
            axy[i] += beam_sum(sp, px, py, pz) * inv * cw[4 * i + 3];
          }
        }
      }
      else
      {
        // mixed states, the mushy range, tables, anisotropy or rotation: an
        // out-of-line pass over the level's points on copies of the arrays
        // (only threads near the melt or in partly melted powder take it)
        double tq_l[NQS], az_l[NQS], axy_l[NQS];
#pragma unroll
        for (int i = 0; i < NQS; ++i)
        {
          tq_l[i] = Tq[i];
          az_l[i] = az[i];
          axy_l[i] = axy[i];
        }
        double lacc = 0.0;
        uint32_t cmask = 0;
        general_level<DEG, NS, P>(sp, gm, md, args, mat, slab, cold, pmode, pu, c * NN + (size_t)NQS * slab, cs, sn,
                                  fast_ok, do_src, cx, cy, cz, tq_l, az_l, axy_l, &lacc, &cmask);
#pragma unroll
        for (int i = 0; i < NQS; ++i)
        {
          az[i] = az_l[i];
          axy[i] = axy_l[i];
        }
        liquid_acc = lacc;
        changed_mask = cmask;
      }
      if (NS == 3 && pmode != 2 && changed_mask)
        changed[cl] = 1;
    }
    // 4. in-slab S^T in x and y of both contributions
#pragma unroll
    for (int pass = 0; pass < 2; ++pass)
    {
      double *a = pass == 0 ? axy : az;
#pragma unroll
      for (int j = 0; j < N; ++j)
      {
        double t[N];
#pragma unroll
        for (int n = 0; n < N; ++n)
          t[n] = col_dot<DEG, M_S>(args.S, n, &a[N * j], 1);
#pragma unroll
        for (int n = 0; n < N; ++n)
          a[n + N * j] = t[n];
      }
#pragma unroll
      for (int i = 0; i < N; ++i)
      {
        double t[N];
#pragma unroll
        for (int n = 0; n < N; ++n)
          t[n] = col_dot<DEG, M_S>(args.S, n, &a[i], N);
#pragma unroll
        for (int n = 0; n < N; ++n)
          a[i + N * n] = t[n];
      }
    }
    if (NS > 1)
      lsum[slab * NCELL + cl] = liquid_acc;
    // 5. z-direction: node level `slab` gathers S^T (values, x/y fluxes) and
    //    G^T (z fluxes) from every Gauss-point level
#pragma unroll
    for (int i = 0; i < NQS; ++i)
    {
      pzbuf[(i + NQS * slab) * NCELL + cl] = axy[i];
      pzbuf[(NN + i + NQS * slab) * NCELL + cl] = az[i];
    }
    group_barrier<TZ, NT / TZ>(lz); // the flux exchange: the z-layer group
    double res[NQS];
    if (slab == 0)
      z_integrate<DEG, 0, NCELL>(args, axy, az, pzbuf, cl, res);
    else if (DEG == 1 || slab == 1)
      z_integrate<DEG, 1, NCELL>(args, axy, az, pzbuf, cl, res);
    else
      z_integrate<DEG, DEG, NCELL>(args, axy, az, pzbuf, cl, res);
    if (!active)
    {
#pragma unroll
      for (int i = 0; i < NQS; ++i)
        res[i] = 0.0;
    }

    // ---- face terms of this node level (face_local_apply,
    // source/ThermalOperator.templates.hh:619-751), out of line: only cells
    // with active-boundary faces take them
    if (FC && active && ((info >> CI_FACE_SHIFT) & 63u))
    {
      double fres[NQS];
      face_terms<DEG, NS>(sp, gm, md, args, brick, lx, ly, lz, slab, info, mat, c, fres);
#pragma unroll
      for (int e = 0; e < NQS; ++e)
        res[e] += fres[e];
    }
    // ---- per-node sums: a warp holds one 8 x 4 layer of cells (lane =
    // lx + 8 ly), so the nodes shared in x and y are summed with shuffles
    // into the cell that owns them (the lower one); nodes shared in z go
    // through one shared-memory exchange between the level threads.
    static_assert(TX == 8 && TY == 4, "the node merge assumes 8 x 4 cell layers per warp");
    unsigned const full = 0xffffffffu;
#pragma unroll
    for (int j = 0; j < N; ++j)
    {
      double const v = __shfl_down_sync(full, res[0 + N * j], 1);
      if (lx < TX - 1)
        res[DEG + N * j] += v;
    }
#pragma unroll
    for (int i = 0; i < N; ++i)
    {
      double const v = __shfl_down_sync(full, res[i], TX);
      if (ly < TY - 1)
        res[i + N * DEG] += v;
    }
    if (slab == 0 && lz > 0)
    {
#pragma unroll
      for (int i = 0; i < NQS; ++i)
        mbuf[i * NCELL + cl] = res[i];
    }
    // the node barrier (the whole CTA) carries the brick-timeout vote: a
    // thread whose wait gave up computed on whatever the buffer held, and
    // the CTA ends here, before anything is written
    if (__syncthreads_or(!arrived))
    {
      if (tid == 0)
      {
        atomicCAS(md.error, 0, (int)DERR_TMA_TIMEOUT);
        // let the late copy, and the one requested for the next item, land
        // before the CTA leaves (bounded as well)
        mbar_wait(&bars[buf], (unsigned)((it >> 1) & 1));
        if (next < last)
          mbar_wait(&bars[buf ^ 1], (unsigned)(((it + 1) >> 1) & 1));
      }
      return;
    }
    if (slab == DEG && lz < TZ - 1)
    {
#pragma unroll
      for (int i = 0; i < NQS; ++i)
        res[i] += mbuf[i * NCELL + cl + TX * TY];
    }

    // ---- state write-back (the liquid sum is read only by the state
    // queries, which see the last evaluation: written by a vmult and by a
    // step's last stage)
    if (slab == 0 && active)
    {
      if (NS > 1 && (args.mode != 2 || args.last))
      {
        double l = 0.0;
        for (int s = 0; s < N; ++s)
          l += lsum[s * NCELL + cl];
        md.liquid_sum[c] = l;
      }
      if (NS == 3 && changed[cl])
        md.powder_mode[c] = 2;
    }
    if (NS == 3 && active && pmode != 2 && changed[cl])
    {
      // the cell switches to per-point powder storage: write this level's
      // points that kept the uniform value
      size_t const pbase = c * NN + (size_t)NQS * slab;
      for (int i = 0; i < NQS; ++i)
        if (!((changed_mask >> i) & 1u))
          md.powder_q[pbase + i] = pu;
    }

    // ---- colour-ordered write-out of the nodes this thread owns: the
    // first tile (in colour order) that touches a node writes it, later
    // ones add, the last one finalizes it. All loads first, then stores.
    bool const own_k = slab > 0 || lz == 0;
    int const Z = DEG * lz + slab;
    int const gz = nz0 + Z;
    int const sz = (Z == 0 && tiz > 0) ? 1 : ((Z == DEG * TZ && tiz < args.nt[2] - 1) ? 2 : 0);
    int rl[NQS], slot[NQS];
    size_t gidx[NQS];
    // the thread's first node and how many of its N x N nodes per row and
    // column lie inside the mesh: one 64-bit index per thread, the nodes at
    // constant offsets from it
    int const gx0 = nx0 + DEG * lx, gy0 = ny0 + DEG * ly;
    int const xin = args.nn[0] - gx0, yin = nn1 - gy0;
    bool const zin = gz < args.nn[2];
    size_t const g0 = gx0 + (size_t)pitch * (gy0 + (size_t)nn1 * gz);
#pragma unroll
    for (int i = 0; i < NQS; ++i)
    {
      int const a = i % N, bb = i / N;
      int const X = DEG * lx + a, Y = DEG * ly + bb;
      bool const own = own_k && (a > 0 || lx == 0) && (bb > 0 || ly == 0);
      bool const inside = a < xin && bb < yin && zin;
      int const sx = (X == 0 && tix > 0) ? 1 : ((X == DEG * TX && tix < nt0 - 1) ? 2 : 0);
      int const sy = (Y == 0 && tiy > 0) ? 1 : ((Y == DEG * TY && tiy < nt1 - 1) ? 2 : 0);
      slot[i] = 0;
      if constexpr (SC == SC_TWO_PASS)
        rl[i] = (own && inside) ? two_pass_slot<HaloOf<DEG>>(X, Y, Z, sx, sy, sz, &slot[i]) : 0;
      else
        rl[i] = (own && inside) ? (SC == SC_ATOMIC ? 4 : (sp.role[buf][sx + 3 * sy + 9 * sz] | 4)) : 0;
      gidx[i] = g0 + a + (size_t)pitch * bb;
    }
    if constexpr (SC == SC_TWO_PASS)
      write_nodes_two_pass<HaloOf<DEG>, NQS>(args, md, tile, res, rl, gidx, slot);
    else
      write_nodes<SC == SC_ATOMIC, NQS>(args, md, y, res, rl, gidx);
    // vmult writes zeros into the row padding of the node layout (the
    // two-pass gather does that itself)
    if (SC == SC_COLOURED && args.mode == 0 && tix == nt0 - 1 && pitch > args.nn[0])
    {
      int const npad = pitch - args.nn[0];
      for (int i = tid; i < npad * BY * BZ; i += NT)
      {
        int const X = i % npad, Y = (i / npad) % BY, Z = i / (npad * BY);
        int const gy = ny0 + Y, gz = nz0 + Z;
        if (gy < nn1 && gz < args.nn[2])
          args.vdst[args.nn[0] + X + (size_t)pitch * (gy + (size_t)nn1 * gz)] = 0.0;
      }
    }
    item = next;
  }
}

// Launches the persistent tile kernel over n_items work items with at most
// the number of CTAs that are resident at once on the device.
template <int DEG, int NS, int P, int SC, bool FC, int TZO = TileShape<DEG>::TZ>
void launch_tile_f(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  using T_ = TD<DEG, TZO>;
  static int grid_cap = 0;
  if (grid_cap == 0)
  {
    cudaFuncSetAttribute(tile_kernel<DEG, NS, P, SC, FC, TZO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)T_::SMEM);
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, tile_kernel<DEG, NS, P, SC, FC, TZO>, T_::NT, T_::SMEM);
    grid_cap = (per_sm > 0 ? per_sm : 1) * (sms > 0 ? sms : 1);
  }
  int const grid = n_items < grid_cap ? n_items : grid_cap;
  tile_kernel<DEG, NS, P, SC, FC, TZO><<<grid, T_::NT, T_::SMEM, stream>>>(map, a, n_items);
}

template <int DEG, int NS, int P, int SC, int TZO = TileShape<DEG>::TZ>
void launch_tile_s(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  if (a.faces)
    launch_tile_f<DEG, NS, P, SC, true, TZO>(map, a, n_items, stream);
  else
    launch_tile_f<DEG, NS, P, SC, false, TZO>(map, a, n_items, stream);
}

// The schedule of a launch: a.atomic, else a.two_pass, else coloured; an
// atomic launch with a.tile_pairs runs 128-cell blocks over z-pairs of tiles
// (FE_Q(2)).
template <int DEG, int NS, int P>
void launch_tile_t(CUtensorMap const &map, KernelArgs const &a, int n_items, cudaStream_t stream)
{
  if (a.atomic)
  {
    if constexpr (DEG == 2)
      if (a.tile_pairs)
      {
        launch_tile_s<DEG, NS, P, SC_ATOMIC, 2 * TileShape<DEG>::TZ>(map, a, n_items, stream);
        return;
      }
    launch_tile_s<DEG, NS, P, SC_ATOMIC>(map, a, n_items, stream);
  }
  else if (a.two_pass)
    launch_tile_s<DEG, NS, P, SC_TWO_PASS>(map, a, n_items, stream);
  else
    launch_tile_s<DEG, NS, P, SC_COLOURED>(map, a, n_items, stream);
}

} // namespace adm

namespace adm
{
// Two-pass schedule, second pass: one CTA per (tile, member) over the nodes
// the tile owns -- its half-open node box, the last tile per direction
// taking the upper end too. A node's sum is the owner's partial sum (when
// the owner is active) plus, in a fixed order, the halo partial sums of the
// lower neighbour tiles that touch it -- no atomics, bit-reproducible. The
// halo arrays of inactive tiles hold zeros (cleared whenever the active set
// changes), so a halo load waits for nothing but the node's position; the
// neighbour mask only decides what is written. An active owner has written
// all its nodes (dst for a vmult, the stage accumulator for a stage), so only
// the nodes on the box's lower faces are visited; an inactive owner's whole
// box is written (its nodes that no active tile touches get zero, except in
// a vmult that adds to dst). A stage then runs the streaming update over all
// nodes (stage_finalize_kernel), as the atomic schedule does.
template <int DEG>
__device__ __forceinline__ void two_pass_gather_node(double *tgt, uint32_t w, bool keep, bool fill, bool const *lower,
                                                     double const *hbase, size_t const *hstride, size_t g, int X,
                                                     int Y, int Z)
{
  using HL = HaloOf<DEG>;
  constexpr int SX = DEG * TD<DEG>::TX, SY = DEG * TD<DEG>::TY;
  constexpr int BX = TD<DEG>::BX, BY = TD<DEG>::BY;
  bool const fx = lower[0] && X == 0, fy = lower[1] && Y == 0, fz = lower[2] && Z == 0;
  double h = 0.0;
  bool any = false;
#pragma unroll
  for (int m = 1; m < 8; ++m)
  {
    int const dx = m & 1, dy = (m >> 1) & 1, dz = m >> 2;
    if ((!dx || fx) && (!dy || fy) && (!dz || fz))
    {
      // the node in the lower neighbour at -(dx, dy, dz) and its halo slot
      // (shared upward in z if dz, else in y if dy, else in x)
      int const slot = dz ? HL::RZ + (X + dx * SX) + BX * (Y + dy * SY)
                          : (dy ? HL::RY + (X + dx * SX) + BX * Z : HL::RX + Y + BY * Z);
      double const *const hp = hbase - (dx ? hstride[0] : 0) - (dy ? hstride[1] : 0) - (dz ? hstride[2] : 0);
      h += hp[slot];
      // its activity: bit (1 - dx) + 3 (1 - dy) + 9 (1 - dz) of the owner's mask
      any = any || ((w >> ((1 - dx) + 3 * (1 - dy) + 9 * (1 - dz))) & 1u);
    }
  }
  double const b = (keep && (fx || fy || fz)) ? tgt[g] : 0.0;
  if (any || fill)
    tgt[g] = b + h;
}

// Grid: x over the tiles, y over the members; 128 threads.
template <int DEG>
__global__ void __launch_bounds__(128) two_pass_gather_kernel(KernelArgs a)
{
  constexpr int SX = DEG * TD<DEG>::TX, SY = DEG * TD<DEG>::TY, SZ = DEG * TD<DEG>::TZ;
  constexpr int NT = 128;
  MemberData const &md = a.members[blockIdx.y];
  int const nt0 = a.nt[0], nt1 = a.nt[1];
  size_t const owner = blockIdx.x;
  int const tx = (int)(owner % (size_t)nt0);
  int const ty = (int)((owner / (size_t)nt0) % (size_t)nt1);
  int const tz = (int)(owner / ((size_t)nt0 * (size_t)nt1));
  uint32_t const w = md.tile_nbr[owner];
  bool const owner_active = (w >> 13) & 1u;
  // the owner's node box, which lower neighbours exist, the owner's halo
  // array and the distances to its lower neighbours' arrays, its first node
  int const ex = tx == nt0 - 1 ? a.nn[0] - SX * tx : SX;
  int const ey = ty == nt1 - 1 ? a.nn[1] - SY * ty : SY;
  int const ez = tz == a.nt[2] - 1 ? a.nn[2] - SZ * tz : SZ;
  bool const lower[3] = {tx > 0, ty > 0, tz > 0};
  constexpr size_t HS = HaloOf<DEG>::SIZE;
  size_t const hstride[3] = {HS, HS * nt0, HS * nt0 * nt1};
  double const *const hbase = md.halo + owner * HS;
  size_t const pitch = (size_t)a.pitch, plane = (size_t)a.pitch * (size_t)a.nn[1];
  size_t const rbase0 = (size_t)SX * tx + pitch * (size_t)(SY * ty) + plane * (size_t)(SZ * tz);
  double *const tgt = a.mode == 2 ? md.acc : a.vdst;
  // the target keeps its value where the owner wrote it, or where a vmult adds
  bool const keep = owner_active || a.mode == 1;
  if (owner_active)
  {
    // the nodes on the lower faces: first those that only one lower
    // neighbour touches (inside the z = 0, y = 0 and x = 0 faces: one halo
    // load each), then the edges and the corner where faces meet
    int const x0 = lower[0] ? 1 : 0, y0 = lower[1] ? 1 : 0, z0 = lower[2] ? 1 : 0;
    int const wx = ex - x0, wy = ey - y0, wz = ez - z0;
    int const nZ = lower[2] ? wx * wy : 0, nY = lower[1] ? wx * wz : 0, nX = lower[0] ? wy * wz : 0;
    int const eXY = lower[0] && lower[1] ? wz : 0, eYZ = lower[1] && lower[2] ? wx : 0;
    int const eXZ = lower[0] && lower[2] ? wy : 0, eC = lower[0] && lower[1] && lower[2] ? 1 : 0;
    int const n1 = nZ + nY + nX, n = n1 + eXY + eYZ + eXZ + eC;
    constexpr int BX = TD<DEG>::BX, BY = TD<DEG>::BY;
    using HL = HaloOf<DEG>;
    for (int k = threadIdx.x; k < n; k += NT)
    {
      if (k < n1)
      {
        int X, Y, Z, slot;
        double const *hp;
        uint32_t bit;
        if (k < nZ)
        {
          int const r = k / wx;
          X = x0 + (k - r * wx);
          Y = y0 + r;
          Z = 0;
          slot = HL::RZ + X + BX * Y;
          hp = hbase - hstride[2];
          bit = 1u << (1 + 3 * 1 + 9 * 0);
        }
        else if (k < nZ + nY)
        {
          int const j = k - nZ, r = j / wx;
          X = x0 + (j - r * wx);
          Y = 0;
          Z = z0 + r;
          slot = HL::RY + X + BX * Z;
          hp = hbase - hstride[1];
          bit = 1u << (1 + 3 * 0 + 9 * 1);
        }
        else
        {
          int const j = k - nZ - nY, r = j / wy;
          X = 0;
          Y = y0 + (j - r * wy);
          Z = z0 + r;
          slot = HL::RX + Y + BY * Z;
          hp = hbase - hstride[0];
          bit = 1u << (0 + 3 * 1 + 9 * 1);
        }
        size_t const g = rbase0 + X + pitch * Y + plane * Z;
        double const h = hp[slot];
        double const b = tgt[g];
        if (w & bit)
          tgt[g] = b + h;
      }
      else
      {
        // edges: X = Y = 0 (along z), Y = Z = 0 (along x), X = Z = 0
        // (along y), then the corner
        int const j = k - n1;
        int X, Y, Z;
        if (j < eXY)
        {
          X = 0;
          Y = 0;
          Z = z0 + j;
        }
        else if (j < eXY + eYZ)
        {
          X = x0 + (j - eXY);
          Y = 0;
          Z = 0;
        }
        else if (j < eXY + eYZ + eXZ)
        {
          X = 0;
          Y = y0 + (j - eXY - eYZ);
          Z = 0;
        }
        else
        {
          X = 0;
          Y = 0;
          Z = 0;
        }
        two_pass_gather_node<DEG>(tgt, w, keep, false, lower, hbase, hstride, rbase0 + X + pitch * Y + plane * Z, X,
                                  Y, Z);
      }
    }
  }
  else
  {
    // the whole box: no active owner wrote it
    bool const fill = a.mode != 1;
    int const exy = ex * ey;
    for (int k = threadIdx.x; k < exy * ez; k += NT)
    {
      int const Z = k / exy, r = k - Z * exy, Y = r / ex, X = r - Y * ex;
      two_pass_gather_node<DEG>(tgt, w, keep, fill, lower, hbase, hstride, rbase0 + X + pitch * Y + plane * Z, X,
                                Y, Z);
    }
  }
  // vmult writes zeros into the row padding of the node layout
  if (a.mode == 0 && tx == nt0 - 1 && a.pitch > a.nn[0])
  {
    int const npad = a.pitch - a.nn[0];
    for (int i = threadIdx.x; i < npad * ey * ez; i += NT)
    {
      int const row = i / npad, Z = row / ey, Y = row - Z * ey;
      a.vdst[rbase0 + ex + (i - row * npad) + pitch * Y + plane * Z] = 0.0;
    }
  }
}
} // namespace adm
