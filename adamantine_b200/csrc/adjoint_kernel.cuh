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
//   d/dlog Q         = sum_q JxW b mu
// The derivative of the temperature dependence covers the polynomials of
// every state, the liquid ratio (dl/dT = 1 / (T_l - T_s) inside the mushy
// range) and the mixing with the powder history; the latent-heat indicator
// l * solid > 0 is piecewise constant and contributes nothing.
//
// Same tiles and thread layout as the forward tile kernel (one thread per
// cell and z-level); one launch covers the tiles of every colour, CTAs loop
// over them, the two node bricks (T and mu) are staged with plain loads and
// the per-node results are added with atomics (a node is shared by at most
// eight tiles). Adiabatic faces only; polynomial properties; no
// deposition-angle rotation.
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

// Mixture value, T-derivative and s'-derivative of one state property.
template <int NS>
__device__ __forceinline__ void mix_prop(SmemPhys const &sp, int mat, int prop, double T, double const *r,
                                         double ld, double &v, double &dT, double &ds)
{
  int const deg = sp.prop_deg[prop];
  double pv[NS], pd[NS];
#pragma unroll
  for (int s = 0; s < NS; ++s)
    poly_vd(&sp.poly[mat][prop][s][0], deg, T, pv[s], pd[s]);
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
template <int NS>
__device__ __forceinline__ AdjQp adj_qp(SmemPhys const &sp, int mat, double T, double mu, double gx, double gy,
                                     double gz, double mx, double my, double mz, double s_in, double lam_out,
                                     double JxW, double Q, double hx2, double hy2, double hz2)
{
  // ratios exactly as update_state_ratios computes them
  double r[3] = {1.0, 0.0, 0.0};
  double ld = 0.0;
  bool br = false; // s' = 1 - l (true) or s' = s (false)
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
  double rho, rho_T, rho_s, cp, cp_T, cp_s;
  mix_prop<NS>(sp, mat, P_DENSITY, T, r, ld, rho, rho_T, rho_s);
  mix_prop<NS>(sp, mat, P_SPECIFIC_HEAT, T, r, ld, cp, cp_T, cp_s);
  double cp_eff = cp;
  if (NS > 1 && r[1] * r[0] > 0.0)
    cp_eff += sp.latent_term[mat];
  double const inv = recip(rho * cp_eff);
  double const inv_T = -inv * inv * (rho_T * cp_eff + rho * cp_T);
  double const inv_s = -inv * inv * (rho_s * cp_eff + rho * cp_s);
  double kd[3], kd_T[3], kd_s[3];
  mix_prop<NS>(sp, mat, P_KX, T, r, ld, kd[0], kd_T[0], kd_s[0]);
  if (sp.isotropic)
  {
    kd[1] = kd[2] = kd[0];
    kd_T[1] = kd_T[2] = kd_T[0];
    kd_s[1] = kd_s[2] = kd_s[0];
  }
  else
  {
    mix_prop<NS>(sp, mat, P_KY, T, r, ld, kd[1], kd_T[1], kd_s[1]);
    mix_prop<NS>(sp, mat, P_KZ, T, r, ld, kd[2], kd_T[2], kd_s[2]);
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
  o.gc = -(cp / cp_eff) * (o.gk + o.gq);
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
__device__ __forceinline__ AdjQp adj_qp_pure(SmemPhys const &sp, int mat, int st, double T, double mu, double gx,
                                             double gy, double gz, double mx, double my, double mz, double JxW,
                                             double Q, double hx2, double hy2, double hz2)
{
  double rho, rho_T, cp, cp_T;
  poly_vd(&sp.poly[mat][P_DENSITY][st][0], sp.prop_deg[P_DENSITY], T, rho, rho_T);
  poly_vd(&sp.poly[mat][P_SPECIFIC_HEAT][st][0], sp.prop_deg[P_SPECIFIC_HEAT], T, cp, cp_T);
  double const inv = recip(rho * cp);
  double const inv_T = -inv * inv * (rho_T * cp + rho * cp_T);
  double kd[3], kd_T[3];
  poly_vd(&sp.poly[mat][P_KX][st][0], sp.prop_deg[P_KX], T, kd[0], kd_T[0]);
  if (sp.isotropic)
  {
    kd[1] = kd[2] = kd[0];
    kd_T[1] = kd_T[2] = kd_T[0];
  }
  else
  {
    poly_vd(&sp.poly[mat][P_KY][st][0], sp.prop_deg[P_KY], T, kd[1], kd_T[1]);
    poly_vd(&sp.poly[mat][P_KZ][st][0], sp.prop_deg[P_KZ], T, kd[2], kd_T[2]);
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
__device__ __noinline__ AdjQp adj_point(SmemPhys const &sp, int mat, int pure, bool no_powder, double T,
                                        double mu, double gx, double gy, double gz, double mx, double my,
                                        double mz, double s_in, double lam_out, double JxW, double Q, double hx2,
                                        double hy2, double hz2)
{
  if (pure >= 0)
    return adj_qp_pure(sp, mat, pure, T, mu, gx, gy, gz, mx, my, mz, JxW, Q, hx2, hy2, hz2);
  if (NS == 3 && no_powder)
    return adj_qp<NS == 3 ? 2 : NS>(sp, mat, T, mu, gx, gy, gz, mx, my, mz, 0.0, 0.0, JxW, Q, hx2, hy2, hz2);
  return adj_qp<NS>(sp, mat, T, mu, gx, gy, gz, mx, my, mz, s_in, lam_out, JxW, Q, hx2, hy2, hz2);
}

template <int DEG, int NS>
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
    bool do_src = false;
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
    if (active)
    {
      size_t const qbase = c * NN + (size_t)NQS * slab;
      bool const no_powder = NS == 3 && A.powder_start && A.powder_start[c] == 0;
      double const hx2 = args.inv_h[0] * args.inv_h[0], hy2 = args.inv_h[1] * args.inv_h[1],
                   hz2 = args.inv_h[2] * args.inv_h[2];
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
        double Q = 0.0;
        if (do_src)
        {
          double const px = (args.origin[0] + cx * args.h[0]) + args.qx[qa] * args.h[0];
          double const py = (args.origin[1] + cy * args.h[1]) + args.qx[qb] * args.h[1];
          double const pz = (args.origin[2] + cz * args.h[2]) + args.qx[slab] * args.h[2];
          Q = beam_sum(sp, px, py, pz);
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
        o = adj_point<NS>(sp, mat, pure, no_powder, T, mu, gx, gy, gz, mx, my, mz, s_in, lam_out, JxW, Q, hx2,
                          hy2, hz2);
        if (with_powder)
          A.lam_s_in[qbase + i] = o.lsin;
        g_k += o.gk;
        g_q += o.gq;
        g_c += o.gc;
        double const fx = o.fx, fy = o.fy, val = o.val;
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
