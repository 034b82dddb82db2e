// Transpose (adjoint) of one operator application, for the hand-written
// adjoint of the explicit time step.
//
// One stage of the forward step evaluates, per Gauss point q of every active
// cell, the phase update s' = min(1 - l(T_q), s) and the residual
//   r_i = sum_q JxW_q [ -sum_d a_d(T_q, s'_q) dT/dx_d dphi_i/dx_d + b(T_q, s'_q) phi_i ]
// with a_d = k_d / (rho c_p), b = Q / (rho c_p) (the cell term of
// source/ThermalOperator.templates.hh:479-617). Given mu = M^-1 lambda_k and
// the adjoint lambda_s' of the updated phase state, this kernel adds
//   (dr/dT)^T mu + (ds'/dT)^T g          to lambda_T (node vector),
//   (ds'/ds)^T g                          to lambda_s (per Gauss point),
// with g = lambda_s' + (dr/ds')^T mu, and accumulates the derivatives of
// mu . r with respect to the logarithms of the conductivity scale, the
// specific-heat scale and the source strength (absorptivity or power):
//   d/dlog k_scale   = sum_q JxW [ -sum_d a_d (dT/dx_d)(dmu/dx_d) ]
//   d/dlog cp_scale  = -(c_p / c_p,eff) (that + JxW b mu)
//   d/dlog Q         = sum_q JxW b mu   (b from the Goldak and electron beams)
// The derivative of the temperature dependence covers the polynomials of
// every state, the liquid ratio (dl/dT = 1 / (T_l - T_s) inside the mushy
// range) and the mixing with the powder history; the latent-heat indicator
// l * solid > 0 is piecewise constant and contributes nothing.
//
// Properties are polynomials or 12-point tables (the derivative of a table
// is the slope of its segment, 0 where it is clamped). A deposition angle
// rotates the conductivity tensor in x-y: the gradients are rotated into the
// frame of (k_x, k_y) before the point evaluation and the fluxes rotated
// back. Convective / radiative faces (source/ThermalOperator.templates.hh:
// 619-751) add the transpose of their flux density
// B = -(1/(rho c_p)) [h_conv (T - T_conv) + h_rad (T - T_rad)] at the face
// points, with the face points' own powder history (adj_face_terms).
//
// Same tiles and thread layout as the forward tile kernel (one thread per
// cell and z-level); one launch covers the tiles of every colour, CTAs loop
// over them, the two node bricks (T and mu) are staged with plain loads and
// the per-node results are added with atomics (a node is shared by at most
// eight tiles).
#pragma once

#include "tile_kernel.cuh"

namespace adm
{

struct AdjArgs
{
  KernelArgs k;            // mesh, 1D rules, work list, member table
  double const *yv;        // stage input (node vector)
  double const *mu;        // M^-1 lambda_k (node vector)
  double const *s_in;      // [C][NN] powder ratio before the stage (3 states)
  double *lam_s_out;       // [C][NN] adjoint of the powder ratio after the stage (cleared where a tile drops out)
  double *lam_s_in;        // [C][NN] adjoint of the powder ratio before the stage
  uint8_t const *powder_start; // [C] powder mode of the run's initial state (0: none), or null
  double *lam_y;           // node vector: += the transpose applied to mu
  double *grad;            // [3] += log-derivatives: k scale, c_p scale, source
  double const *mu_max;    // max |mu| of the stage, or null (no flush)
  double flush;            // tiles with |mu| <= flush * *mu_max and no powder adjoint are skipped
  int const *n_items_dev;  // number of work items (a selected list) in device memory, or null
  uint8_t *act_next;       // per tile: may hold a non-negligible adjoint next stage (set here), or null
  // faces of three-state problems: [slot][6][NF] as MemberData::face_powder
  double const *sf_in;     // powder ratio of the face points before the stage
  double *lam_sf_out;      // adjoint of the face points' powder ratio after the stage
  double *lam_sf_in;       // adjoint of the face points' powder ratio before the stage
};

// Horner value and derivative of sum_i c[i] T^i up to degree deg.
__device__ __forceinline__ void poly_vd(double const *c, int deg, double T, double &v, double &d)
{
  double vv = c[deg], dd = 0.0;
  for (int i = deg - 1; i >= 0; --i)
  {
    dd = fma(dd, T, vv);
    vv = fma(vv, T, c[i]);
  }
  v = vv;
  d = dd;
}

// Value and derivative of MaterialProperty::compute_property_from_table
// (source/MaterialProperty.templates.hh:1158-1212; the value as
// table_lookup computes it): the slope of the segment holding T, 0 where
// the table is clamped (below the first point, from the next-to-last on).
__device__ __forceinline__ void table_vd(MaterialDesc const *gm, int mat, int prop, int s, double T, double &v,
                                         double &d)
{
  double const(*t)[2] = gm->table[mat][prop][s];
  d = 0.0;
  if (T <= t[0][0])
  {
    v = t[0][1];
    return;
  }
  int i = 0;
  for (; i < kTableSize; ++i)
    if (T < t[i][0])
      break;
  if (i >= kTableSize - 1)
  {
    v = t[kTableSize - 1][1];
    return;
  }
  v = t[i - 1][1] + (T - t[i - 1][0]) * (t[i][1] - t[i - 1][1]) / (t[i][0] - t[i - 1][0]);
  d = (t[i][1] - t[i - 1][1]) / (t[i][0] - t[i - 1][0]);
}

// Value and T-derivative of one state's property (polynomial or table).
__device__ __forceinline__ void prop_vd(SmemPhys const &sp, MaterialDesc const *gm, int mat, int prop, int s,
                                        double T, double &v, double &d)
{
  if (sp.use_table)
    table_vd(gm, mat, prop, s, T, v, d);
  else
    poly_vd(&sp.poly[mat][prop][s][0], sp.prop_deg[prop], T, v, d);
}

// Mixture value, T-derivative and s'-derivative of one state property.
template <int NS>
__device__ __forceinline__ void mix_prop(SmemPhys const &sp, MaterialDesc const *gm, int mat, int prop, double T,
                                         double const *r, double ld, double &v, double &dT, double &ds)
{
  double pv[NS], pd[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s)
    prop_vd(sp, gm, mat, prop, s, T, pv[s], pd[s]);
  double a = 0.0, b = 0.0;
#pragma unroll
  for (int s = 0; s < NS; ++s)
  {
    a = fma(r[s], pv[s], a);
    b = fma(r[s], pd[s], b);
  }
  ds = 0.0;
  if (NS > 1)
    b = fma(ld, pv[1] - pv[0], b); // d r_liquid / dT = ld, d r_solid / dT = -ld
  if (NS == 3)
    ds = pv[NS == 3 ? 2 : 0] - pv[0]; // d r_powder / ds' = 1, d r_solid / ds' = -1
  v = a;
  dT = b;
}

struct AdjQp
{
  double fx, fy, fz, val, lsin, gk, gq, gc;
};

// The transposed coefficients at one Gauss point. Inputs: the field T and mu
// with their reference gradients, the powder ratio before the stage, the
// adjoint of the powder ratio after it, JxW, the source value Q and the
// squared inverse cell sizes. Outputs: the reference-space fluxes and the
// value term of the transposed operator, the adjoint of the powder ratio
// before the stage and the three log-derivative contributions.
// State ratios exactly as update_state_ratios computes them
// (source/ThermalOperator.templates.hh:227-317), with dl/dT (ld) and which
// side of s' = min(1 - l, s) is taken (br: s' = 1 - l).
template <int NS>
__device__ __forceinline__ void adj_ratios(SmemPhys const &sp, int mat, double T, double s_in, double *r,
                                           double &ld, bool &br)
{
  r[0] = 1.0;
  r[1] = r[2] = 0.0;
  ld = 0.0;
  br = false;
  if (NS > 1)
  {
    double const Ts = sp.props[mat][Q_SOLIDUS], Tl = sp.props[mat][Q_LIQUIDUS];
    double l;
    if (T < Ts)
      l = 0.0;
    else if (T > Tl)
      l = 1.0;
    else
      l = (T - Ts) / (Tl - Ts);
    if (T > Ts && T < Tl)
      ld = 1.0 / (Tl - Ts);
    r[1] = l;
    if (NS == 2)
      r[0] = 1.0 - l;
    else
    {
      double const one_minus_l = 1.0 - l;
      br = !(s_in < one_minus_l);
      double const sp_new = br ? one_minus_l : s_in;
      r[2] = sp_new;
      r[0] = 1.0 - l - sp_new;
    }
  }
}

// 1/(rho c_p,eff) with its T- and s'-derivatives (get_inv_rho_cp,
// source/ThermalOperator.templates.hh:415-477; the latent-heat indicator is
// piecewise constant); cp / cp_eff for the specific-heat log-derivative.
template <int NS>
__device__ __forceinline__ void adj_inv_rho_cp(SmemPhys const &sp, MaterialDesc const *gm, int mat, double T,
                                               double const *r, double ld, double &inv, double &inv_T,
                                               double &inv_s, double &cp_frac)
{
  double rho, rho_T, rho_s, cp, cp_T, cp_s;
  mix_prop<NS>(sp, gm, mat, P_DENSITY, T, r, ld, rho, rho_T, rho_s);
  mix_prop<NS>(sp, gm, mat, P_SPECIFIC_HEAT, T, r, ld, cp, cp_T, cp_s);
  double cp_eff = cp;
  if (NS > 1 && r[1] * r[0] > 0.0)
    cp_eff += sp.latent_term[mat];
  inv = recip(rho * cp_eff);
  inv_T = -inv * inv * (rho_T * cp_eff + rho * cp_T);
  inv_s = -inv * inv * (rho_s * cp_eff + rho * cp_s);
  cp_frac = cp / cp_eff;
}

template <int NS>
__device__ __forceinline__ AdjQp adj_qp(SmemPhys const &sp, MaterialDesc const *gm, int mat, double T, double mu,
                                     double gx, double gy, double gz, double mx, double my, double mz,
                                     double s_in, double lam_out, double JxW, double Q, double hx2, double hy2,
                                     double hz2)
{
  double r[3], ld;
  bool br;
  adj_ratios<NS>(sp, mat, T, s_in, r, ld, br);
  double inv, inv_T, inv_s, cp_frac;
  adj_inv_rho_cp<NS>(sp, gm, mat, T, r, ld, inv, inv_T, inv_s, cp_frac);
  double kd[3], kd_T[3], kd_s[3];
  mix_prop<NS>(sp, gm, mat, P_KX, T, r, ld, kd[0], kd_T[0], kd_s[0]);
  if (sp.isotropic)
  {
    kd[1] = kd[2] = kd[0];
    kd_T[1] = kd_T[2] = kd_T[0];
    kd_s[1] = kd_s[2] = kd_s[0];
  }
  else
  {
    mix_prop<NS>(sp, gm, mat, P_KY, T, r, ld, kd[1], kd_T[1], kd_s[1]);
    mix_prop<NS>(sp, gm, mat, P_KZ, T, r, ld, kd[2], kd_T[2], kd_s[2]);
  }
  // physical gradient products (reference gradients / h)
  double const uv[3] = {gx * mx * hx2, gy * my * hy2, gz * mz * hz2};
  double dot_a = 0.0, dot_aT = 0.0, dot_as = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    double const a = kd[d] * inv;
    dot_a = fma(a, uv[d], dot_a);
    dot_aT = fma(fma(kd_T[d], inv, kd[d] * inv_T), uv[d], dot_aT);
    dot_as = fma(fma(kd_s[d], inv, kd[d] * inv_s), uv[d], dot_as);
  }
  AdjQp o;
  double const b = Q * inv;
  o.val = JxW * (-dot_aT + Q * inv_T * mu);
  o.lsin = 0.0;
  if (NS == 3)
  {
    double const gs = lam_out + JxW * (-dot_as + Q * inv_s * mu);
    if (br)
      o.val -= ld * gs;
    else
      o.lsin = gs;
  }
  o.gk = JxW * (-dot_a);
  o.gq = JxW * b * mu;
  o.gc = -cp_frac * (o.gk + o.gq);
  // fluxes of the transposed diffusion term in reference coordinates
  double const cf = -inv * JxW;
  o.fx = cf * kd[0] * mx * hx2;
  o.fy = cf * kd[1] * my * hy2;
  o.fz = cf * kd[2] * mz * hz2;
  return o;
}

// adj_qp at a point in one pure state st below the solidus: ratios 1 for st
// and 0 elsewhere, no liquid-ratio derivative, no latent heat, and a
// powder adjoint that does not propagate (the point is solid without powder
// history, or untouched powder, whose s' = 1 - l follows T with
// dl/dT = 0). One polynomial per property, inline.
__device__ __forceinline__ AdjQp adj_qp_pure(SmemPhys const &sp, MaterialDesc const *gm, int mat, int st, double T,
                                             double mu, double gx, double gy, double gz, double mx, double my,
                                             double mz, double JxW, double Q, double hx2, double hy2, double hz2)
{
  double rho, rho_T, cp, cp_T;
  prop_vd(sp, gm, mat, P_DENSITY, st, T, rho, rho_T);
  prop_vd(sp, gm, mat, P_SPECIFIC_HEAT, st, T, cp, cp_T);
  double const inv = recip(rho * cp);
  double const inv_T = -inv * inv * (rho_T * cp + rho * cp_T);
  double kd[3], kd_T[3];
  prop_vd(sp, gm, mat, P_KX, st, T, kd[0], kd_T[0]);
  if (sp.isotropic)
  {
    kd[1] = kd[2] = kd[0];
    kd_T[1] = kd_T[2] = kd_T[0];
  }
  else
  {
    prop_vd(sp, gm, mat, P_KY, st, T, kd[1], kd_T[1]);
    prop_vd(sp, gm, mat, P_KZ, st, T, kd[2], kd_T[2]);
  }
  double const uv[3] = {gx * mx * hx2, gy * my * hy2, gz * mz * hz2};
  double dot_a = 0.0, dot_aT = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    dot_a = fma(kd[d] * inv, uv[d], dot_a);
    dot_aT = fma(fma(kd_T[d], inv, kd[d] * inv_T), uv[d], dot_aT);
  }
  AdjQp o;
  o.val = JxW * (-dot_aT + Q * inv_T * mu);
  o.lsin = 0.0;
  o.gk = JxW * (-dot_a);
  o.gq = JxW * (Q * inv) * mu;
  o.gc = -(o.gk + o.gq);
  double const cf = -inv * JxW;
  o.fx = cf * kd[0] * mx * hx2;
  o.fy = cf * kd[1] * my * hy2;
  o.fz = cf * kd[2] * mz * hz2;
  return o;
}

// One Gauss point of the adjoint kernel: the pure-state path, the cells
// without powder at the start (solid/liquid mixtures: the powder adjoint
// never reaches the temperature or the parameters there) or the full
// mixture. Out of line: the kernel calls it for the 9 or 4 points of a
// thread's level, and one copy of the code keeps the instruction footprint
// small.
template <int NS>
__device__ __noinline__ AdjQp adj_point(SmemPhys const &sp, MaterialDesc const *gm, int mat, int pure,
                                        bool no_powder, double T, double mu, double gx, double gy, double gz,
                                        double mx, double my, double mz, double s_in, double lam_out, double JxW,
                                        double Q, double hx2, double hy2, double hz2)
{
  if (pure >= 0)
    return adj_qp_pure(sp, gm, mat, pure, T, mu, gx, gy, gz, mx, my, mz, JxW, Q, hx2, hy2, hz2);
  if (NS == 3 && no_powder)
    return adj_qp<NS == 3 ? 2 : NS>(sp, gm, mat, T, mu, gx, gy, gz, mx, my, mz, 0.0, 0.0, JxW, Q, hx2, hy2, hz2);
  return adj_qp<NS>(sp, gm, mat, T, mu, gx, gy, gz, mx, my, mz, s_in, lam_out, JxW, Q, hx2, hy2, hz2);
}

// Transposed face terms of one cell for the node level `slab` (the
// transpose of face_terms in tile_kernel.cuh, which every level thread of
// a cell evaluates, keeping its own level's test functions). At a face
// point with trace values T_f and mu_f, powder ratio s' = min(1 - l(T_f), s)
// and flux density B(T_f, s') = -(1/(rho c_p)) [h_conv (T_f - T_conv) +
// h_rad (T_f - T_rad)], h_rad = eps sigma (T_f + T_rad)(T_f^2 + T_rad^2):
//   out[e]          += JxW mu_f dB/dT phi_e        (node e of this level)
//   g                = lam_sf' + JxW mu_f dB/ds'   (to s, or -g dl/dT to T where s' = 1 - l)
//   return value    += -(c_p / c_p,eff) JxW mu_f B (specific-heat log-derivative)
// The powder adjoint and the return value come from one thread per face
// point (the one that updates the face powder in the forward kernel).
template <int DEG, int NS>
__device__ __noinline__ double adj_face_terms(SmemPhys const &sp, MaterialDesc const *gm, AdjArgs const &A,
                                              MemberData const &md, double const *yb, double const *mb, int lx,
                                              int ly, int lz, int slab, uint32_t info, int mat, size_t c,
                                              bool no_powder, double *out)
{
  constexpr int N = DEG + 1, NQS = N * N, NF = N * N;
  constexpr int BXP = TD<DEG>::BXP, BY = TD<DEG>::BY;
  KernelArgs const &args = A.k;
  for (int e = 0; e < NQS; ++e)
    out[e] = 0.0;
  double gc = 0.0;
  int const slot = (NS == 3 && !no_powder) ? md.face_slot[c] : -1;
  for (int f = 0; f < 6; ++f)
  {
    if (!((info >> (CI_FACE_SHIFT + f)) & 1u))
      continue;
    int const d = f / 2, side = f % 2;
    if (d == 2 && slab != (side ? N - 1 : 0))
      continue; // a z face only touches one node level
    bool const writer = d == 2 || slab == 0;
    int const t0 = d == 0 ? 1 : 0, t1 = d == 2 ? 1 : 2;
    int const btype =
        ((info >> (CI_INTERFACE_SHIFT + f)) & 1u) ? args.interface_type : args.boundary_type[f];
    double const ht0 = args.h[t0], ht1 = args.h[t1];
    for (int fq = 0; fq < NF; ++fq)
    {
      int const qa = fq % N, qb = fq / N;
      double T = 0.0, M = 0.0;
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
        {
          int loc[3];
          loc[d] = side ? N - 1 : 0;
          loc[t0] = i;
          loc[t1] = j;
          int const e = (DEG * lx + loc[0]) + BXP * ((DEG * ly + loc[1]) + BY * (DEG * lz + loc[2]));
          double const phi = args.S[qa][i] * args.S[qb][j];
          T += phi * yb[e];
          M += phi * mb[e];
        }
      size_t const fi = ((size_t)(slot < 0 ? 0 : slot) * 6 + f) * NF + fq;
      double const s_in = (slot >= 0 && A.sf_in) ? A.sf_in[fi] : 0.0;
      double r[3], ld;
      bool br;
      adj_ratios<NS>(sp, mat, T, s_in, r, ld, br);
      double inv, inv_T, inv_s, cp_frac;
      adj_inv_rho_cp<NS>(sp, gm, mat, T, r, ld, inv, inv_T, inv_s, cp_frac);
      double F = 0.0, F_T = 0.0, F_s = 0.0;
      if (btype & B_CONVECTIVE)
      {
        double const Tc = sp.props[mat][Q_CONV_TINF];
        double hc, hc_T, hc_s;
        mix_prop<NS>(sp, gm, mat, P_CONV_COEF, T, r, ld, hc, hc_T, hc_s);
        F += hc * (T - Tc);
        F_T += hc_T * (T - Tc) + hc;
        F_s += hc_s * (T - Tc);
      }
      if (btype & B_RADIATIVE)
      {
        double const Tr = sp.props[mat][Q_RAD_TINF];
        double em, em_T, em_s;
        mix_prop<NS>(sp, gm, mat, P_EMISSIVITY, T, r, ld, em, em_T, em_s);
        double const sigma = 5.670374419e-8;
        double const p = (T + Tr) * (T * T + Tr * Tr);
        double const p_T = (T * T + Tr * Tr) + 2.0 * T * (T + Tr);
        F += em * sigma * p * (T - Tr);
        F_T += sigma * (em_T * p * (T - Tr) + em * (p_T * (T - Tr) + p));
        F_s += em_s * sigma * p * (T - Tr);
      }
      double const B = -inv * F;
      double const B_T = -(inv_T * F + inv * F_T);
      double const w = args.qw[qa] * ht0 * args.qw[qb] * ht1 * M;
      double val = w * B_T;
      if (NS == 3 && slot >= 0)
      {
        double const lam_out = A.lam_sf_out ? A.lam_sf_out[fi] : 0.0;
        double const gs = lam_out + w * (-(inv_s * F + inv * F_s));
        if (br)
          val -= ld * gs;
        if (writer && A.lam_sf_in)
          A.lam_sf_in[fi] = br ? 0.0 : gs;
      }
      if (writer)
        gc -= cp_frac * w * B;
      for (int j = 0; j < N; ++j)
        for (int i = 0; i < N; ++i)
        {
          int const la = d == 0 ? (side ? N - 1 : 0) : i;
          int const lb = d == 0 ? i : (d == 1 ? (side ? N - 1 : 0) : j);
          int const lc = d == 2 ? (side ? N - 1 : 0) : j;
          if (lc != slab)
            continue;
          out[la + N * lb] += val * (args.S[qa][i] * args.S[qb][j]);
        }
    }
  }
  return gc;
}

// The source at a point from the Goldak and electron beams only (the
// beams the source-strength parameter scales; cube sources keep their
// value).
static __device__ __noinline__ double scaled_beam_sum(SmemPhys const &sp, double px, double py, double pz)
{
  double qs = 0.0;
  for (int b = 0; b < sp.n_beams; ++b)
    if (sp.beams[b].type != 2)
      qs += beam_value(sp.beams[b], px, py, pz);
  return qs;
}

// GEN: the problem has a deposition-angle rotation, boundary faces or a
// cube source (instantiated apart so that the common case carries none of
// that code).
template <int DEG, int NS, bool GEN>
__global__ void __launch_bounds__(TD<DEG>::NT, 2)
    adjoint_kernel(const __grid_constant__ CUtensorMap ymap, const __grid_constant__ CUtensorMap mmap,
                   const __grid_constant__ AdjArgs A, int n_items_max)
{
  int const n_items = A.n_items_dev ? min(n_items_max, *A.n_items_dev) : n_items_max;
  using T_ = TD<DEG>;
  constexpr int N = T_::N, NN = T_::NN, NT = T_::NT, NCELL = T_::NCELL, NQS = T_::NQS;
  constexpr int TX = T_::TX, TY = T_::TY, TZ = T_::TZ;
  constexpr int BXP = T_::BXP, BY = T_::BY;
  constexpr unsigned kBoxBytes = sizeof(double) * T_::BXP * T_::BY * T_::BZ;
  extern __shared__ __align__(128) double smem[];
  // [buffer][field T, mu][BRICKP]: the next item's bricks arrive by TMA while
  // the current item is computed
  double *const xbuf = smem + 4 * T_::BRICKP;   // [2][NN][NCELL]
  double *const pzbuf = xbuf + 2 * NN * NCELL;  // [2][NN][NCELL]
  __shared__ SmemPhys sp;
  __shared__ double red[3][NT / 32];
  __shared__ __align__(8) uint64_t bars[2];

  KernelArgs const &args = A.k;
  int const tid = threadIdx.x;
  int const slab = tid / NCELL, cl = tid % NCELL;
  int const lx = cl % TX, ly = (cl / TX) % TY, lz = cl / (TX * TY);
  int const nt0 = args.nt[0], nt1 = args.nt[1];
  int const pitch = args.pitch, nn1 = args.nn[1];

  auto issue = [&](int buf, int item) {
    TileWork const wi = args.work[item];
    int const x = DEG * TX * (int)(wi.xyz & 2047u), y = DEG * TY * (int)((wi.xyz >> 11) & 2047u),
              z = DEG * TZ * (int)(wi.xyz >> 22);
    mbar_arrive_expect_tx(&bars[buf], 2 * kBoxBytes);
    tma_load_brick(smem + (2 * buf) * T_::BRICKP, &ymap, x, y, z, 0, &bars[buf]);
    tma_load_brick(smem + (2 * buf + 1) * T_::BRICKP, &mmap, x, y, z, 0, &bars[buf]);
  };
  if (tid == 0)
  {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0 && (int)blockIdx.x < n_items)
    issue(0, blockIdx.x);

  double g_k = 0.0, g_c = 0.0, g_q = 0.0;
  int cur_member = -1;
  int it = 0;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x, ++it)
  {
    int const buf = it & 1;
    double const *const yb = smem + (2 * buf) * T_::BRICKP;
    double const *const mb = smem + (2 * buf + 1) * T_::BRICKP;
    TileWork const w = args.work[item];
    MemberData const &md = args.members[w.member];
    int const tix = w.xyz & 2047u, tiy = (w.xyz >> 11) & 2047u, tiz = w.xyz >> 22;
    int const ncx0 = TX * tix, ncy0 = TY * tiy, ncz0 = TZ * tiz;
    int const nx0 = DEG * ncx0, ny0 = DEG * ncy0, nz0 = DEG * ncz0;

    // prefetch the next item's bricks into the other buffer (consumed before
    // the barrier that ended the previous item)
    if (tid == 0 && item + (int)gridDim.x < n_items)
    {
      fence_proxy_async();
      issue(buf ^ 1, item + gridDim.x);
    }
    if (w.member != cur_member)
    {
      // the previous item ended with a barrier, so nobody reads sp now
      load_member_constants<NT>(sp, md, tid);
      cur_member = w.member;
    }
    // bounded wait for this item's bricks; the barrier also publishes sp
    bool const arrived = mbar_wait(&bars[buf], (unsigned)((it >> 1) & 1));
    if (__syncthreads_or(!arrived))
    {
      if (tid == 0)
      {
        atomicCAS(md.error, 0, (int)DERR_TMA_TIMEOUT);
        if (item + (int)gridDim.x < n_items)
          mbar_wait(&bars[buf ^ 1], (unsigned)(((it + 1) >> 1) & 1));
      }
      return;
    }

    // A tile on whose nodes mu is zero, and whose cells carry no powder
    // adjoint, contributes nothing: every output is a multiple of mu or of
    // lam_s_out (the transposed fluxes and values, the powder adjoint
    // passed on, the parameter derivatives). The explicit stencil spreads
    // the adjoint of a misfit at a few points by about one cell per stage,
    // with values falling by orders of magnitude per cell, so "zero" is
    // |mu| <= flush * max |mu| (flush 0: exactly zero; the default 1e-30
    // drops terms some 14 orders of magnitude below double rounding). Such
    // tiles only clear the powder adjoint they hand on.
    {
      double const thr = A.mu_max ? A.flush * *A.mu_max : 0.0;
      bool nz = false;
      for (int e = tid; e < BXP * BY * T_::BZ; e += NT)
        nz |= fabs(mb[e]) > thr;
      int const sx = ncx0 + lx, sy = ncy0 + ly, sz = ncz0 + lz;
      size_t const sc = (sx < args.nc[0] && sy < args.nc[1] && sz < args.nc[2])
                            ? sx + (size_t)args.nc[0] * (sy + (size_t)args.nc[1] * sz)
                            : (size_t)-1;
      bool const powder_cell = NS == 3 && sc != (size_t)-1 && (md.cell_info[sc] & CI_ACTIVE) &&
                               !(A.powder_start && A.powder_start[sc] == 0);
      size_t const sbase = powder_cell ? sc * NN + (size_t)NQS * slab : 0;
      if (powder_cell)
        for (int i = 0; i < NQS; ++i)
          nz |= A.lam_s_out[sbase + i] != 0.0;
      // the face points of the cell (level thread 0 of each cell)
      int const fslot = (GEN && powder_cell && slab == 0 && A.lam_sf_out) ? md.face_slot[sc] : -1;
      constexpr int NFS = 6 * (DEG + 1) * (DEG + 1);
      if (fslot >= 0)
        for (int i = 0; i < NFS; ++i)
          nz |= A.lam_sf_out[(size_t)fslot * NFS + i] != 0.0;
      if (!__syncthreads_or(nz))
      {
        // the tile drops out of the list: both powder-adjoint buffers of
        // its cells are left clean for when it comes back (only this
        // tile's threads read them)
        if (powder_cell)
          for (int i = 0; i < NQS; ++i)
          {
            A.lam_s_in[sbase + i] = 0.0;
            A.lam_s_out[sbase + i] = 0.0;
          }
        if (fslot >= 0)
          for (int i = 0; i < NFS; ++i)
          {
            A.lam_sf_in[(size_t)fslot * NFS + i] = 0.0;
            A.lam_sf_out[(size_t)fslot * NFS + i] = 0.0;
          }
        continue;
      }
      // the adjoint spreads by at most one cell per stage: this tile and its
      // neighbours are visited next stage
      if (A.act_next && tid < 27)
      {
        int const ox = tix + tid % 3 - 1, oy = tiy + (tid / 3) % 3 - 1, oz = tiz + tid / 9 - 1;
        if (ox >= 0 && ox < args.nt[0] && oy >= 0 && oy < args.nt[1] && oz >= 0 && oz < args.nt[2])
          A.act_next[ox + (size_t)args.nt[0] * (oy + (size_t)args.nt[1] * oz)] = 1;
      }
    }

    // tile-level source culling (as in the forward kernel)
    bool do_src = false, has_cube = false;
    {
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
          if (x1 >= bs.cube_min[0] && x0 <= bs.cube_max[0] && y1 >= bs.cube_min[1] && y0 <= bs.cube_max[1] &&
              z1 >= bs.cube_min[2] && z0 <= bs.cube_max[2])
          {
            do_src = true;
            has_cube = GEN;
          }
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
    }

    int const cx = ncx0 + lx, cy = ncy0 + ly, cz = ncz0 + lz;
    bool const in_domain = cx < args.nc[0] && cy < args.nc[1] && cz < args.nc[2];
    size_t const c = in_domain ? cx + (size_t)args.nc[0] * (cy + (size_t)args.nc[1] * cz) : 0;
    uint32_t const info = in_domain ? md.cell_info[c] : 0u;
    bool const active = (info & CI_ACTIVE) != 0;
    int const mat = (info >> CI_MAT_SHIFT) & 15;

    // 1. x/y interpolation of node level `slab` of both fields
    double wv[2][NQS];
  #pragma unroll
    for (int f = 0; f < 2; ++f)
    {
      double const *brick = f == 0 ? yb : mb;
      double *v = wv[f];
  #pragma unroll
      for (int j = 0; j < N; ++j)
  #pragma unroll
        for (int i = 0; i < N; ++i)
          v[i + N * j] = brick[(DEG * lx + i) + BXP * ((DEG * ly + j) + BY * (DEG * lz + slab))];
  #pragma unroll
      for (int j = 0; j < N; ++j)
      {
        double t[N];
  #pragma unroll
        for (int q = 0; q < N; ++q)
        {
          double acc = args.S[q][0] * v[N * j];
  #pragma unroll
          for (int k = 1; k < N; ++k)
            acc = fma(args.S[q][k], v[k + N * j], acc);
          t[q] = acc;
        }
  #pragma unroll
        for (int q = 0; q < N; ++q)
          v[q + N * j] = t[q];
      }
  #pragma unroll
      for (int i = 0; i < N; ++i)
      {
        double t[N];
  #pragma unroll
        for (int q = 0; q < N; ++q)
        {
          double acc = args.S[q][0] * v[i];
  #pragma unroll
          for (int k = 1; k < N; ++k)
            acc = fma(args.S[q][k], v[i + N * k], acc);
          t[q] = acc;
        }
  #pragma unroll
        for (int q = 0; q < N; ++q)
          v[i + N * q] = t[q];
      }
  #pragma unroll
      for (int i = 0; i < NQS; ++i)
        xbuf[(f * NN + i + NQS * slab) * NCELL + cl] = v[i];
    }
    __syncthreads();
    // 2. values and z-gradients at this thread's Gauss-point level
    double Tq[NQS], Tz[NQS], Mq[NQS], Mz[NQS];
  #pragma unroll
    for (int i = 0; i < NQS; ++i)
    {
      double tv = 0.0, tz = 0.0, mv = 0.0, mz = 0.0;
  #pragma unroll
      for (int m = 0; m < N; ++m)
      {
        double const a = (m == slab) ? wv[0][i] : xbuf[(i + NQS * m) * NCELL + cl];
        double const b = (m == slab) ? wv[1][i] : xbuf[(NN + i + NQS * m) * NCELL + cl];
        tv = fma(args.S[slab][m], a, tv);
        tz = fma(args.G[slab][m], a, tz);
        mv = fma(args.S[slab][m], b, mv);
        mz = fma(args.G[slab][m], b, mz);
      }
      Tq[i] = tv;
      Tz[i] = tz;
      Mq[i] = mv;
      Mz[i] = mz;
    }

    // 3. per Gauss point: the transposed coefficients
    double axy[NQS], az[NQS];
  #pragma unroll
    for (int i = 0; i < NQS; ++i)
    {
      axy[i] = 0.0;
      az[i] = 0.0;
    }
    MaterialDesc const *const gm = md.mat;
    bool const no_powder = NS == 3 && A.powder_start && A.powder_start[c] == 0;
    if (active)
    {
      size_t const qbase = c * NN + (size_t)NQS * slab;
      double const hz2 = args.inv_h[2] * args.inv_h[2];
      // a deposition angle rotates (k_x, k_y) (source/ThermalOperator.templates.hh:552-594):
      // the point sees physical gradients in the frame of (k_x, k_y)
      bool const rot = GEN && sp.has_rotation && !sp.isotropic;
      double cs = 1.0, sn = 0.0;
      if (rot)
      {
        cs = md.cosv[c];
        sn = md.sinv[c];
      }
      double const hx2 = rot ? 1.0 : args.inv_h[0] * args.inv_h[0];
      double const hy2 = rot ? 1.0 : args.inv_h[1] * args.inv_h[1];
  #pragma unroll
      for (int i = 0; i < NQS; ++i)
      {
        int const qa = i % N, qb = i / N;
        double const T = Tq[i], mu = Mq[i];
        double gx = 0.0, gy = 0.0, mx = 0.0, my = 0.0;
  #pragma unroll
        for (int k = 0; k < N; ++k)
        {
          gx = fma(args.D[qa][k], Tq[k + N * qb], gx);
          gy = fma(args.D[qb][k], Tq[qa + N * k], gy);
          mx = fma(args.D[qa][k], Mq[k + N * qb], mx);
          my = fma(args.D[qb][k], Mq[qa + N * k], my);
        }
        double const gz = Tz[i], mz = Mz[i];
        if (rot)
        {
          double const gxp = gx * args.inv_h[0], gyp = gy * args.inv_h[1];
          double const mxp = mx * args.inv_h[0], myp = my * args.inv_h[1];
          gx = cs * gxp + sn * gyp;
          gy = cs * gyp - sn * gxp;
          mx = cs * mxp + sn * myp;
          my = cs * myp - sn * mxp;
        }
        double Q = 0.0, Qp = 0.0; // all sources; the scaled beams
        if (do_src)
        {
          double const px = (args.origin[0] + cx * args.h[0]) + args.qx[qa] * args.h[0];
          double const py = (args.origin[1] + cy * args.h[1]) + args.qx[qb] * args.h[1];
          double const pz = (args.origin[2] + cz * args.h[2]) + args.qx[slab] * args.h[2];
          Q = beam_sum(sp, px, py, pz);
          Qp = has_cube ? scaled_beam_sum(sp, px, py, pz) : Q;
        }
        double const JxW = args.qw[qa] * args.qw[qb] * args.qw[slab] * args.vol;
        AdjQp o;
        bool const with_powder = NS == 3 && !no_powder;
        double const s_in = with_powder ? A.s_in[qbase + i] : 0.0;
        // one pure state below the solidus (see adj_qp_pure)
        int pure = -1;
        if (NS == 1)
          pure = 0;
        else if (T < sp.props[mat][Q_SOLIDUS])
          pure = !with_powder ? 0 : (s_in == 1.0 ? 2 : -1);
        double const lam_out = (with_powder && pure < 0) ? A.lam_s_out[qbase + i] : 0.0;
        o = adj_point<NS>(sp, gm, mat, pure, no_powder, T, mu, gx, gy, gz, mx, my, mz, s_in, lam_out, JxW, Q,
                          hx2, hy2, hz2);
        if (with_powder)
          A.lam_s_in[qbase + i] = o.lsin;
        g_k += o.gk;
        g_q += (!GEN || Qp == Q) ? o.gq : (Q != 0.0 ? o.gq * (Qp / Q) : 0.0);
        g_c += o.gc;
        double fx = o.fx, fy = o.fy;
        if (rot)
        {
          // back to the mesh frame, then to reference coordinates
          double const fxp = cs * fx - sn * fy, fyp = sn * fx + cs * fy;
          fx = fxp * args.inv_h[0];
          fy = fyp * args.inv_h[1];
        }
        double const val = o.val;
        az[i] = o.fz;
  #pragma unroll
        for (int m = 0; m < N; ++m)
        {
          axy[m + N * qb] = fma(args.D[qa][m], fx, axy[m + N * qb]);
          axy[qa + N * m] = fma(args.D[qb][m], fy, axy[qa + N * m]);
        }
        axy[i] += val;
      }
    }
    // 4. S^T in x and y
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
        {
          double acc = args.S[0][n] * a[N * j];
  #pragma unroll
          for (int q = 1; q < N; ++q)
            acc = fma(args.S[q][n], a[q + N * j], acc);
          t[n] = acc;
        }
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
        {
          double acc = args.S[0][n] * a[i];
  #pragma unroll
          for (int q = 1; q < N; ++q)
            acc = fma(args.S[q][n], a[i + N * q], acc);
          t[n] = acc;
        }
  #pragma unroll
        for (int n = 0; n < N; ++n)
          a[i + N * n] = t[n];
      }
    }
    // 5. z direction: S^T of values and x/y fluxes, G^T of z fluxes
  #pragma unroll
    for (int i = 0; i < NQS; ++i)
    {
      pzbuf[(i + NQS * slab) * NCELL + cl] = axy[i];
      pzbuf[(NN + i + NQS * slab) * NCELL + cl] = az[i];
    }
    __syncthreads();
    double res[NQS];
  #pragma unroll
    for (int i = 0; i < NQS; ++i)
    {
      double acc = 0.0;
  #pragma unroll
      for (int q = 0; q < N; ++q)
      {
        double const vp = (q == slab) ? axy[i] : pzbuf[(i + NQS * q) * NCELL + cl];
        double const vz = (q == slab) ? az[i] : pzbuf[(NN + i + NQS * q) * NCELL + cl];
        acc = fma(args.S[q][slab], vp, acc);
        acc = fma(args.G[q][slab], vz, acc);
      }
      res[i] = active ? acc : 0.0;
    }
    // transposed face terms of the cells with active-boundary faces
    if (GEN && args.faces && active && ((info >> CI_FACE_SHIFT) & 63u))
    {
      double fres[NQS];
      g_c += adj_face_terms<DEG, NS>(sp, gm, A, md, yb, mb, lx, ly, lz, slab, info, mat, c, no_powder, fres);
  #pragma unroll
      for (int e = 0; e < NQS; ++e)
        res[e] += fres[e];
    }
    // 6. per-node sums inside the tile (as in the forward kernel)
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
        xbuf[i * NCELL + cl] = res[i];
    }
    __syncthreads();
    if (slab == DEG && lz < TZ - 1)
    {
  #pragma unroll
      for (int i = 0; i < NQS; ++i)
        res[i] += xbuf[i * NCELL + cl + TX * TY];
    }
    // 7. owned nodes: lambda_y += result
    bool const own_k = slab > 0 || lz == 0;
    int const gz = nz0 + DEG * lz + slab;
  #pragma unroll
    for (int i = 0; i < NQS; ++i)
    {
      int const a = i % N, bb = i / N;
      int const gx = nx0 + DEG * lx + a, gy = ny0 + DEG * ly + bb;
      bool const own = own_k && (a > 0 || lx == 0) && (bb > 0 || ly == 0);
      if (own && gx < args.nn[0] && gy < nn1 && gz < args.nn[2])
      {
        size_t const g = gx + (size_t)pitch * (gy + (size_t)nn1 * gz);
        atomicAdd(&A.lam_y[g], res[i]);
      }
    }
    // the bricks and exchange buffers are reused by the next item
    __syncthreads();
  }
  // 8. parameter derivatives: warp sums, then one atomic per CTA
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
  {
    g_k += __shfl_xor_sync(0xffffffffu, g_k, o);
    g_c += __shfl_xor_sync(0xffffffffu, g_c, o);
    g_q += __shfl_xor_sync(0xffffffffu, g_q, o);
  }
  if ((tid & 31) == 0)
  {
    red[0][tid >> 5] = g_k;
    red[1][tid >> 5] = g_c;
    red[2][tid >> 5] = g_q;
  }
  __syncthreads();
  if (tid < 3)
  {
    double s = 0.0;
    for (int wi = 0; wi < NT / 32; ++wi)
      s += red[tid][wi];
    if (s != 0.0)
      atomicAdd(&A.grad[tid], s);
  }
}

} // namespace adm
