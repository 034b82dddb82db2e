/*
 * CPU oracle for the adamantine thermal hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C++17/OpenMP restatement of the reference's CPU (Host memory space)
 * matrix-free heat operator, material model, heat sources and explicit time
 * stepping, on a structured box mesh with a fixed full-grid node numbering.
 * Each block cites the reference code it follows (paths inside adamantine
 * v1.1.9). Only tests/, the smoke check and the benchmark's CPU-baseline leg
 * may load this library; the product never does.
 *
 * Restatement choices (each differs from the reference only where the
 * reference result depends on SIMD batch composition or on a lookup bug):
 *  R1 heat-source cutoff: the scalar semantics of GoldakHeatSource::value /
 *     ElectronBeamHeatSource::value (both the depth mask and the r^2 > 5R^2
 *     cutoff); the vectorized reference paths apply only the depth mask once
 *     any lane of a batch is inside the cutoff.
 *  R2 powder history: every quadrature point's powder ratio is updated and
 *     stored (the vectorized reference loop in update_state_ratios reloads the
 *     stored vector inside the lane loop, so only the last SIMD lane keeps its
 *     update).
 *  R3 set_state: FE_Nothing cells keep their state (the host reference reads
 *     cell (0,0) of the MatrixFree through std::map::operator[] for them; the
 *     device reference skips them, as here).
 *  R4 latent heat in the operator uses the CPU rule liquid*solid > 0
 *     (ThermalOperator.templates.hh:466-473).
 *  R5 RK2 is deal.II's explicit midpoint tableau (the reference offers only
 *     forward Euler, RK3 and RK4).
 */
#include "thermal_oracle.h"

#include <omp.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

namespace
{
constexpr double kStefanBoltzmann = 5.670374419e-8; // types.hh:158
constexpr double kPi = 3.14159265358979323846;
enum StateProperty
{
  DENSITY = 0,
  SPECIFIC_HEAT,
  KX,
  KY,
  KZ,
  EMISSIVITY,
  RAD_COEF,
  CONV_COEF,
  N_STATE_PROPS
};
enum Property
{
  LIQUIDUS = 0,
  SOLIDUS,
  LATENT,
  RAD_TINF,
  CONV_TINF
};
enum BoundaryBits
{
  B_ADIABATIC = 1,
  B_RADIATIVE = 2,
  B_CONVECTIVE = 4
};
enum State
{
  SOLID = 0,
  LIQUID = 1,
  POWDER = 2
};

struct Rule1D
{
  std::vector<double> x, w;
};

long double legendre(int n, long double x, long double *dp)
{
  long double p0 = 1.0L, p1 = x;
  if (n == 0)
  {
    *dp = 0;
    return 1;
  }
  for (int k = 2; k <= n; ++k)
  {
    long double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
    p0 = p1;
    p1 = p2;
  }
  *dp = n * (x * p1 - p0) / (x * x - 1.0L);
  return p1;
}

// Gauss-Legendre rule with n points on [0,1] (deal.II QGauss<1>(n)).
Rule1D gauss_rule(int n)
{
  Rule1D r;
  std::vector<long double> xs(n), ws(n);
  for (int i = 0; i < n; ++i)
  {
    long double x = std::cos(kPi * (i + 0.75L) / (n + 0.5L));
    for (int it = 0; it < 100; ++it)
    {
      long double dp;
      long double p = legendre(n, x, &dp);
      long double dx = p / dp;
      x -= dx;
      if (std::fabs((double)dx) < 1e-30)
        break;
    }
    long double dp;
    legendre(n, x, &dp);
    xs[i] = x;
    ws[i] = 2.0L / ((1.0L - x * x) * dp * dp);
  }
  for (int i = n - 1; i >= 0; --i)
  {
    r.x.push_back((double)((1.0L - xs[i]) / 2.0L));
    r.w.push_back((double)(ws[i] / 2.0L));
  }
  std::vector<int> idx(n);
  for (int i = 0; i < n; ++i)
    idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&](int a, int b) { return r.x[a] < r.x[b]; });
  Rule1D s;
  for (int i : idx)
  {
    s.x.push_back(r.x[i]);
    s.w.push_back(r.w[i]);
  }
  return s;
}

// Gauss-Lobatto rule with n points on [0,1] (deal.II QGaussLobatto<1>(n)).
Rule1D gauss_lobatto_rule(int n)
{
  Rule1D r;
  std::vector<long double> xs;
  xs.push_back(-1.0L);
  // interior points: roots of P'_{n-1}
  for (int i = 1; i < n - 1; ++i)
  {
    long double x = -std::cos(kPi * i / (n - 1));
    for (int it = 0; it < 200; ++it)
    {
      // f = P'_{n-1}(x); f' = P''_{n-1}(x) via (1-x^2)P'' = 2xP' - m(m+1)P
      long double dp;
      long double p = legendre(n - 1, x, &dp);
      long double m = n - 1;
      long double d2p = (2 * x * dp - m * (m + 1) * p) / (1 - x * x);
      long double dx = dp / d2p;
      x -= dx;
      if (std::fabs((double)dx) < 1e-30)
        break;
    }
    xs.push_back(x);
  }
  xs.push_back(1.0L);
  for (long double x : xs)
  {
    long double dp;
    long double p = legendre(n - 1, x, &dp);
    long double w = 2.0L / (n * (n - 1) * p * p);
    r.x.push_back((double)((x + 1.0L) / 2.0L));
    r.w.push_back((double)(w / 2.0L));
  }
  return r;
}

struct Beam
{
  int type = 0;
  bool on = false;
  double center[3] = {0, 0, 0};
  double alpha = 0;
  double depth = 0, radius_squared = 0, inv_r2 = 0, inv_d2 = 0, inv_d = 0;
};

} // namespace

struct orc_oracle
{
  orc_config cfg;
  std::vector<std::vector<double>> segments;
  int dim, deg, np, nq, nqc, ndc, nfq, nfaces;
  int64_t nc[3], nn[3], ncells, nnodes;
  double h[3], cell_volume;
  std::vector<double> qx, qw;                 // 1D quadrature on [0,1]
  std::vector<double> S, G;                   // [nq][np]
  std::vector<double> glw;                    // 1D lumped mass weights
  std::vector<double> hq;                     // QGauss(deg+1) for averages
  std::vector<double> hqw, Sh;                // weights, values [nh][np]
  std::vector<uint8_t> active, matid, node_active, has_melted;
  // cells whose region carries material (level grid of a refined mesh:
  // the active cells are that level's leaves); empty: the active cells
  std::vector<uint8_t> domain;
  std::vector<double> cosv, sinv;
  std::vector<double> state;                  // [n_states][C]
  // mutable like the reference's tables (ThermalOperator.hh:210-226):
  // vmult updates them as a side effect
  mutable std::vector<double> liquid_q, powder_q; // [C][Q]
  mutable std::vector<double> face_powder;        // [C][2*dim][nfq]
  std::vector<double> inv_mass;
  std::vector<Beam> beams;
  bool sources_on = false;
  bool adiabatic_only = true;

  // ---------------------------------------------------------------- helpers
  void cell_coords(int64_t c, int64_t *cc) const
  {
    cc[0] = c % nc[0];
    int64_t r = c / nc[0];
    cc[1] = r % nc[1];
    cc[2] = r / nc[1];
  }
  int64_t cell_index(int64_t const *cc) const
  {
    return cc[0] + nc[0] * (cc[1] + nc[1] * cc[2]);
  }
  int64_t node_index(int64_t const *ni) const
  {
    return ni[0] + nn[0] * (ni[1] + nn[1] * ni[2]);
  }
  // Global node indices of the cell's (deg+1)^dim local nodes (x fastest).
  void cell_nodes(int64_t c, int64_t *out) const
  {
    int64_t cc[3];
    cell_coords(c, cc);
    int idx = 0;
    int const n2 = dim == 3 ? np : 1;
    for (int k = 0; k < n2; ++k)
      for (int j = 0; j < np; ++j)
        for (int i = 0; i < np; ++i)
        {
          int64_t ni[3] = {deg * cc[0] + i, deg * cc[1] + j,
                           dim == 3 ? deg * cc[2] + k : 0};
          out[idx++] = node_index(ni);
        }
  }

  int boundary_type_for_id(int id) const
  {
    // Boundary::get_boundary_type (Boundary.hh:120-126)
    int const n = cfg.n_boundary_types;
    if (id >= 0 && id < n - 1 && id < 8)
      return cfg.boundary_types[id];
    return cfg.boundary_types[n - 1];
  }

  // Tensor sweep: apply M (rows x cols) along direction d of a tensor whose
  // extents are all n (np == nq). transpose applies M^T.
  void sweep(double const *M, bool transpose, int d, double const *in,
             double *out) const
  {
    int const n = np;
    int stride = 1;
    for (int e = 0; e < d; ++e)
      stride *= n;
    int const total = dim == 3 ? n * n * n : n * n;
    for (int base = 0; base < total; ++base)
    {
      if ((base / stride) % n != 0)
        continue;
      for (int r = 0; r < n; ++r)
      {
        double acc = 0;
        for (int k = 0; k < n; ++k)
        {
          double const m = transpose ? M[k * n + r] : M[r * n + k];
          acc += m * in[base + k * stride];
        }
        out[base + r * stride] = acc;
      }
    }
  }

  // -------------------------------------------------------- material model
  double table_lookup(int mat, int prop, int s, double T) const
  {
    // MaterialProperty::compute_property_from_table
    // (MaterialProperty.templates.hh:1158-1212)
    auto const &t = cfg.table[mat][prop][s];
    if (T <= t[0][0])
      return t[0][1];
    unsigned i = 0;
    unsigned const size = 12;
    for (; i < size; ++i)
      if (T < t[i][0])
        break;
    if (i >= size - 1)
      return t[size - 1][1];
    double const ti = t[i][0], tim1 = t[i - 1][0];
    double const pi = t[i][1], pim1 = t[i - 1][1];
    return pim1 + (T - tim1) * (pi - pim1) / (ti - tim1);
  }

  // MaterialProperty::compute_material_property (MaterialProperty.hh:529-800)
  double property(int prop, int mat, double const *ratios, double T,
                  double const *Tpow) const
  {
    double value = 0.0;
    int const ns = cfg.n_states;
    if (cfg.use_table)
    {
      for (int s = 0; s < ns; ++s)
        value += ratios[s] * table_lookup(mat, prop, s, T);
    }
    else if (cfg.n_materials == 1)
    {
      for (int i = 0; i <= cfg.p_order; ++i)
        for (int s = 0; s < ns; ++s)
          value += ratios[s] * cfg.poly[mat][prop][s][i] * Tpow[i];
    }
    else
    {
      for (int s = 0; s < ns; ++s)
        for (int i = 0; i <= cfg.p_order; ++i)
          value += ratios[s] * cfg.poly[mat][prop][s][i] * Tpow[i];
    }
    return value;
  }

  // ThermalOperator::update_state_ratios, scalar semantics (R2)
  // (ThermalOperator.templates.hh:227-317)
  void state_ratios(int mat, double T, double *powder_hist, double *liquid_out,
                    double *r) const
  {
    int const ns = cfg.n_states;
    if (ns == 1)
    {
      r[SOLID] = 1.;
      return;
    }
    double const solidus = cfg.props[mat][SOLIDUS];
    double const liquidus = cfg.props[mat][LIQUIDUS];
    double l;
    if (T < solidus)
      l = 0.;
    else if (T > liquidus)
      l = 1.;
    else
      l = (T - solidus) / (liquidus - solidus);
    r[LIQUID] = l;
    if (ns == 2)
    {
      r[SOLID] = 1. - l;
    }
    else
    {
      double const p = std::min(1. - l, *powder_hist);
      r[POWDER] = p;
      r[SOLID] = 1. - l - p;
      *powder_hist = p;
    }
    if (liquid_out)
      *liquid_out = l;
  }

  // ThermalOperator::get_inv_rho_cp (ThermalOperator.templates.hh:415-477)
  double inv_rho_cp(int mat, double const *r, double T, double const *Tpow) const
  {
    double const density = property(DENSITY, mat, r, T, Tpow);
    double specific_heat = property(SPECIFIC_HEAT, mat, r, T, Tpow);
    if (cfg.n_states > 1)
    {
      double const is_mushy = r[LIQUID] * r[SOLID];
      if (is_mushy > 0.0)
        specific_heat += cfg.props[mat][LATENT] /
                         (cfg.props[mat][LIQUIDUS] - cfg.props[mat][SOLIDUS]);
    }
    return 1.0 / (density * specific_heat);
  }

  void powers(double T, double *Tpow) const
  {
    Tpow[0] = 1.0;
    for (int i = 1; i <= cfg.p_order; ++i)
      Tpow[i] = Tpow[i - 1] * T;
  }

  // ------------------------------------------------------------ sources
  // ScanPath::value / get_power_modifier (ScanPath.cc:197-275)
  void scan_path(int b, double t, double *pos, double *pmod) const
  {
    auto const &sg = segments[b];
    int const n = (int)(sg.size() / 5);
    if (n == 0 || t > sg[(n - 1) * 5 + 0])
    {
      double const low = std::numeric_limits<double>::lowest();
      pos[0] = pos[1] = pos[2] = low;
      *pmod = 0.0;
      return;
    }
    int cur = 0;
    while (t > sg[cur * 5 + 0])
      ++cur;
    double st, sp[3];
    if (cur > 0)
    {
      st = sg[(cur - 1) * 5 + 0];
      for (int d = 0; d < 3; ++d)
        sp[d] = sg[(cur - 1) * 5 + 2 + d];
    }
    else
    {
      st = 0.0;
      for (int d = 0; d < 3; ++d)
        sp[d] = sg[cur * 5 + 2 + d];
    }
    double const et = sg[cur * 5 + 0];
    for (int d = 0; d < 3; ++d)
      pos[d] = sp[d] + (sg[cur * 5 + 2 + d] - sp[d]) / (et - st) * (t - st);
    *pmod = sg[cur * 5 + 1];
  }

  // ThermalOperator::set_time (ThermalOperator.hh:296-308) with
  // GoldakHeatSource::update_time (GoldakHeatSource.cc:24-44),
  // ElectronBeamHeatSource::update_time (ElectronBeamHeatSource.cc:24-45),
  // CubeHeatSource::update_time (CubeHeatSource.cc:45-49).
  void set_time(double t)
  {
    sources_on = false;
    for (int b = 0; b < cfg.n_sources; ++b)
    {
      orc_source const &src = cfg.sources[b];
      Beam &bm = beams[b];
      bm.type = src.type;
      if (src.type == 2)
      {
        bm.on = (t > src.cube_start_time) && (t < src.cube_end_time);
      }
      else
      {
        double pos[3], pmod;
        scan_path(b, t, pos, &pmod);
        bm.on = pmod > 0.0;
        for (int d = 0; d < 3; ++d)
          bm.center[d] = pos[d];
        bm.depth = src.depth;
        bm.radius_squared = src.radius_squared;
        if (src.type == 0)
        {
          double const pi_over_3_to_1p5 = std::pow(kPi / 3.0, 1.5);
          bm.alpha = 2.0 * src.absorption_efficiency * src.max_power * pmod /
                     (bm.radius_squared * bm.depth * pi_over_3_to_1p5);
          bm.inv_r2 = 1.0 / bm.radius_squared;
          bm.inv_d2 = 1.0 / (bm.depth * bm.depth);
        }
        else
        {
          double const log_01 = std::log(0.1);
          bm.alpha = -src.absorption_efficiency * src.max_power * pmod *
                     log_01 / (kPi * src.radius_squared * src.depth);
          bm.inv_d = 1.0 / bm.depth;
          bm.inv_r2 = 1.0 / bm.radius_squared;
        }
      }
      if (bm.on)
        sources_on = true;
    }
  }

  // Scalar HeatSource::value (R1).
  double source_value(int b, double const *p) const
  {
    Beam const &bm = beams[b];
    orc_source const &src = cfg.sources[b];
    if (bm.type == 2)
    {
      // CubeHeatSource::value (CubeHeatSource.cc:51-71)
      if (bm.on)
      {
        for (int i = 0; i < dim; ++i)
          if (p[i] < src.cube_min[i] || p[i] > src.cube_max[i])
            return 0.;
        return src.cube_value;
      }
      return 0.;
    }
    int const zax = dim - 1;
    double const z = p[zax] - bm.center[zax];
    if (z + bm.depth < 0.)
      return 0.;
    double xpy = (p[0] - bm.center[0]) * (p[0] - bm.center[0]);
    if (dim == 3)
      xpy += (p[1] - bm.center[1]) * (p[1] - bm.center[1]);
    if (xpy > 5. * bm.radius_squared)
      return 0.;
    if (bm.type == 0)
    {
      // GoldakHeatSource::value (GoldakHeatSource.cc:46-89)
      return bm.alpha *
             std::exp(-3.0 * xpy * bm.inv_r2 + -3.0 * (z * z) * bm.inv_d2);
    }
    // ElectronBeamHeatSource::value (ElectronBeamHeatSource.cc:47-93)
    double const z_rel = z * bm.inv_d;
    double const dist_z = -3. * (z_rel * z_rel) - 2. * z_rel + 1.;
    double const log_01 = std::log(0.1);
    return bm.alpha * std::exp(log_01 * xpy * bm.inv_r2) * dist_z;
  }

  // ------------------------------------------------------------ operator
  bool face_is_boundary(int64_t const *cc, int f, bool *outer) const
  {
    int const d = f / 2, side = f % 2;
    int64_t nb[3] = {cc[0], cc[1], cc[2]};
    nb[d] += side ? 1 : -1;
    if (nb[d] < 0 || nb[d] >= nc[d])
    {
      *outer = true;
      return true;
    }
    *outer = false;
    return domain.empty() ? !active[cell_index(nb)] : !domain[cell_index(nb)];
  }

  // cell_local_apply (ThermalOperator.templates.hh:479-617) plus
  // face_local_apply (ThermalOperator.templates.hh:619-751) for this cell.
  void cell_apply(int64_t c, double const *src, double *dst,
                  std::vector<double> &scratch) const
  {
    int const Q = nqc;
    double *u = scratch.data();
    double *t0 = u + Q;
    double *t1 = t0 + Q;
    double *val = t1 + Q;
    double *grad = val + Q;      // dim * Q
    double *fg = grad + 3 * Q;   // dim * Q
    double *fv = fg + 3 * Q;
    double *r = fv + Q;
    double *acc = r + Q;
    int64_t nodes[125];
    cell_nodes(c, nodes);
    for (int i = 0; i < ndc; ++i)
      u[i] = src[nodes[i]];

    // values: S in every direction; gradients: G in direction d, S elsewhere
    auto eval = [&](int gdir, double *out) {
      double const *cur = u;
      double *bufs[2] = {t0, t1};
      for (int d = 0; d < dim; ++d)
      {
        double *o = (d == dim - 1) ? out : bufs[d % 2];
        sweep(d == gdir ? G.data() : S.data(), false, d, cur, o);
        cur = o;
      }
    };
    eval(-1, val);
    for (int d = 0; d < dim; ++d)
      eval(d, grad + d * Q);

    int64_t cc[3];
    cell_coords(c, cc);
    int const mat = matid[c];
    double const cs = cosv[c], sn = sinv[c];
    double Tpow[5];
    double ratios[3];
    for (int q = 0; q < Q; ++q)
    {
      int qi[3] = {q % nq, (q / nq) % nq, q / (nq * nq)};
      double JxW = cell_volume;
      for (int d = 0; d < dim; ++d)
        JxW *= qw[qi[d]];
      double const T = val[q];
      powers(T, Tpow);
      double *ph = cfg.n_states == 3 ? &powder_q[c * Q + q] : nullptr;
      double *lq = cfg.n_states > 1 ? &liquid_q[c * Q + q] : nullptr;
      state_ratios(mat, T, ph, lq, ratios);
      double const inv = inv_rho_cp(mat, ratios, T, Tpow);
      double g[3];
      for (int d = 0; d < dim; ++d)
        g[d] = grad[d * Q + q] / h[d];
      double kg[3];
      if (dim == 2)
      {
        kg[0] = g[0] * property(KX, mat, ratios, T, Tpow);
        kg[1] = g[1] * property(KZ, mat, ratios, T, Tpow);
      }
      else
      {
        double const kx = property(KX, mat, ratios, T, Tpow);
        double const ky = property(KY, mat, ratios, T, Tpow);
        kg[0] = (kx * cs * cs + ky * sn * sn) * g[0] +
                ((kx - ky) * sn * cs) * g[1];
        kg[1] = ((kx - ky) * sn * cs) * g[0] +
                (kx * sn * sn + ky * cs * cs) * g[1];
        kg[2] = g[2] * property(KZ, mat, ratios, T, Tpow);
      }
      for (int d = 0; d < dim; ++d)
        fg[d * Q + q] = (-inv * kg[d]) / h[d] * JxW;
      if (sources_on)
      {
        double pt[3];
        for (int d = 0; d < dim; ++d)
          pt[d] = (cfg.origin[d] + cc[d] * h[d]) + qx[qi[d]] * h[d];
        double qs = 0.0;
        for (int b = 0; b < cfg.n_sources; ++b)
          qs += source_value(b, pt);
        fv[q] = qs * inv * JxW;
      }
    }

    // integrate: r = sum_d (G_d^T S^T..) fg_d [+ S^T.. fv]
    for (int i = 0; i < Q; ++i)
      acc[i] = 0.;
    auto integ = [&](int gdir, double const *in) {
      double const *cur = in;
      double *bufs[2] = {t0, t1};
      for (int d = dim - 1; d >= 0; --d)
      {
        double *o = (d == 0) ? r : bufs[d % 2];
        sweep(d == gdir ? G.data() : S.data(), true, d, cur, o);
        cur = o;
      }
      for (int i = 0; i < Q; ++i)
        acc[i] += r[i];
    };
    for (int d = 0; d < dim; ++d)
      integ(d, fg + d * Q);
    if (sources_on)
      integ(-1, fv);

    if (!adiabatic_only)
      face_terms(c, cc, u, acc);

    for (int i = 0; i < ndc; ++i)
      dst[nodes[i]] += acc[i];
  }

  void face_terms(int64_t c, int64_t const *cc, double const *u,
                  double *acc) const
  {
    int const mat = matid[c];
    for (int f = 0; f < nfaces; ++f)
    {
      bool outer;
      if (!face_is_boundary(cc, f, &outer))
        continue;
      int const btype = outer ? boundary_type_for_id(f)
                              : boundary_type_for_id(255);
      int const d = f / 2, side = f % 2;
      int tdirs[2], nt = 0;
      for (int e = 0; e < dim; ++e)
        if (e != d)
          tdirs[nt++] = e;
      int const fnq = nfq;
      for (int fq = 0; fq < fnq; ++fq)
      {
        int qa = fq % nq, qb = dim == 3 ? fq / nq : 0;
        // trace value: sum over the face's nodes of the tangential basis
        double T = 0.0;
        double phi[125];
        double JxW = 1.0;
        JxW *= qw[qa] * h[tdirs[0]];
        if (dim == 3)
          JxW *= qw[qb] * h[tdirs[1]];
        for (int i = 0; i < ndc; ++i)
        {
          int li[3] = {i % np, (i / np) % np, i / (np * np)};
          if (li[d] != (side ? np - 1 : 0))
          {
            phi[i] = 0.;
            continue;
          }
          double v = S[qa * np + li[tdirs[0]]];
          if (dim == 3)
            v *= S[qb * np + li[tdirs[1]]];
          phi[i] = v;
          T += v * u[i];
        }
        double Tpow[5], ratios[3];
        powers(T, Tpow);
        double *ph = cfg.n_states == 3
                         ? &face_powder[(c * nfaces + f) * nfq + fq]
                         : nullptr;
        state_ratios(mat, T, ph, nullptr, ratios);
        double const inv = inv_rho_cp(mat, ratios, T, Tpow);
        double conv_tinf = 0., conv_h = 0., rad_tinf = 0., rad_h = 0.;
        if (btype & B_CONVECTIVE)
        {
          conv_tinf = cfg.props[mat][CONV_TINF];
          conv_h = property(CONV_COEF, mat, ratios, T, Tpow);
        }
        if (btype & B_RADIATIVE)
        {
          rad_tinf = cfg.props[mat][RAD_TINF];
          rad_h = property(EMISSIVITY, mat, ratios, T, Tpow) *
                  kStefanBoltzmann * (T + rad_tinf) *
                  (T * T + rad_tinf * rad_tinf);
        }
        double const bval =
            -inv * (conv_h * (T - conv_tinf) + rad_h * (T - rad_tinf));
        for (int i = 0; i < ndc; ++i)
          if (phi[i] != 0.)
            acc[i] += bval * phi[i] * JxW;
      }
    }
  }

  void vmult_add(double *dst, double const *src) const
  {
    int const ncol = 1 << dim;
    int64_t const sz = 3 * nqc * 12 + 64;
    for (int col = 0; col < ncol; ++col)
    {
      int const px = col & 1, py = (col >> 1) & 1, pz = (col >> 2) & 1;
      int64_t const mx = (nc[0] - px + 1) / 2, my = (nc[1] - py + 1) / 2;
      int64_t const mz = dim == 3 ? (nc[2] - pz + 1) / 2 : 1;
      int64_t const total = mx * my * mz;
#pragma omp parallel num_threads(cfg.n_threads > 0 ? cfg.n_threads : omp_get_max_threads())
      {
        std::vector<double> scratch(sz);
#pragma omp for schedule(static)
        for (int64_t w = 0; w < total; ++w)
        {
          int64_t cc[3] = {2 * (w % mx) + px, 2 * ((w / mx) % my) + py,
                           dim == 3 ? 2 * (w / (mx * my)) + pz : 0};
          int64_t const c = cell_index(cc);
          if (!active[c])
            continue;
          cell_apply(c, src, dst, scratch);
        }
      }
    }
  }

  // ------------------------------------------------------------ setup
  void update_node_active()
  {
    std::fill(node_active.begin(), node_active.end(), 0);
    std::vector<int64_t> nodes(ndc);
    for (int64_t c = 0; c < ncells; ++c)
    {
      if (!active[c])
        continue;
      cell_nodes(c, nodes.data());
      for (int i = 0; i < ndc; ++i)
        node_active[nodes[i]] = 1;
    }
  }

  // compute_inverse_mass_matrix (ThermalOperator.templates.hh:118-164):
  // Gauss-Lobatto lumped mass on active cells, inverted on active DoFs.
  void compute_inverse_mass()
  {
    std::vector<double> m(nnodes, 0.0);
    std::vector<int64_t> nodes(ndc);
    for (int64_t c = 0; c < ncells; ++c)
    {
      if (!active[c])
        continue;
      cell_nodes(c, nodes.data());
      for (int i = 0; i < ndc; ++i)
      {
        int li[3] = {i % np, (i / np) % np, i / (np * np)};
        double w = cell_volume;
        for (int d = 0; d < dim; ++d)
          w *= glw[li[d]];
        m[nodes[i]] += w;
      }
    }
    for (int64_t n = 0; n < nnodes; ++n)
      inv_mass[n] = node_active[n] ? 1. / m[n] : 0.;
  }

  // get_state_from_material_properties (ThermalOperator.templates.hh:753-884)
  void get_state_from_material_properties()
  {
    int const ns = cfg.n_states;
    for (int64_t c = 0; c < ncells; ++c)
    {
      if (!active[c])
        continue;
      for (int q = 0; q < nqc; ++q)
      {
        if (ns > 1)
          liquid_q[c * nqc + q] = state[LIQUID * ncells + c];
        if (ns == 3)
          powder_q[c * nqc + q] = state[POWDER * ncells + c];
      }
      if (ns == 3 && !adiabatic_only)
        for (int f = 0; f < nfaces; ++f)
          for (int q = 0; q < nfq; ++q)
            face_powder[(c * nfaces + f) * nfq + q] = state[POWDER * ncells + c];
    }
  }

  // set_state_to_material_properties -> MaterialProperty::set_state
  // (MaterialProperty.templates.hh:537-621), R3 for FE_Nothing cells.
  void set_state_to_material_properties()
  {
    int const ns = cfg.n_states;
    for (int64_t c = 0; c < ncells; ++c)
    {
      if (ns == 1)
      {
        state[c] = 1.;
        continue;
      }
      if (!active[c])
        continue;
      double ls = 0., ps = 0.;
      for (int q = 0; q < nqc; ++q)
      {
        ls += liquid_q[c * nqc + q];
        if (ns == 3)
          ps += powder_q[c * nqc + q];
      }
      state[LIQUID * ncells + c] = ls / nqc;
      if (ns == 2)
        state[SOLID * ncells + c] = 1. - state[LIQUID * ncells + c];
      else
      {
        state[POWDER * ncells + c] = ps / nqc;
        state[SOLID * ncells + c] =
            1. - state[LIQUID * ncells + c] - state[POWDER * ncells + c];
      }
    }
  }

  // Cell average with QGauss(deg+1): compute_average
  // (MaterialProperty.templates.hh:33-73), also mark_has_melted
  // (ThermalPhysics.templates.hh:537-593).
  double cell_average(int64_t c, double const *T) const
  {
    int64_t nodes[125];
    cell_nodes(c, nodes);
    int const nh = (int)hqw.size();
    int const nhq = dim == 3 ? nh * nh * nh : nh * nh;
    double volume = 0., avg = 0.;
    for (int q = 0; q < nhq; ++q)
    {
      int qi[3] = {q % nh, (q / nh) % nh, q / (nh * nh)};
      double JxW = cell_volume;
      for (int d = 0; d < dim; ++d)
        JxW *= hqw[qi[d]];
      for (int i = 0; i < ndc; ++i)
      {
        int li[3] = {i % np, (i / np) % np, i / (np * np)};
        double phi = 1.;
        for (int d = 0; d < dim; ++d)
          phi *= Sh[qi[d] * np + li[d]];
        volume += phi * JxW;
        avg += phi * T[nodes[i]] * JxW;
      }
    }
    return avg / volume;
  }
};

namespace
{
void build_basis(orc_oracle *o)
{
  int const np = o->np;
  // FE_Q support points = Gauss-Lobatto points
  Rule1D gl = gauss_lobatto_rule(np);
  std::vector<double> const &nodes = gl.x;
  o->glw = gl.w;
  Rule1D q = o->cfg.quadrature == 1 ? gauss_lobatto_rule(np) : gauss_rule(np);
  o->qx = q.x;
  o->qw = q.w;
  auto lag = [&](int i, double x, double *dval) {
    double v = 1.0, dv = 0.0;
    for (int j = 0; j < np; ++j)
    {
      if (j == i)
        continue;
      double const den = nodes[i] - nodes[j];
      // product rule accumulation
      dv = dv * (x - nodes[j]) / den + v / den;
      v *= (x - nodes[j]) / den;
    }
    *dval = dv;
    return v;
  };
  o->S.assign(np * np, 0.);
  o->G.assign(np * np, 0.);
  for (int qq = 0; qq < np; ++qq)
    for (int i = 0; i < np; ++i)
    {
      double dv;
      double v = lag(i, o->qx[qq], &dv);
      o->S[qq * np + i] = v;
      o->G[qq * np + i] = dv;
    }
  Rule1D hq = gauss_rule(np);
  o->hqw = hq.w;
  o->Sh.assign(np * np, 0.);
  for (int qq = 0; qq < np; ++qq)
    for (int i = 0; i < np; ++i)
    {
      double dv;
      o->Sh[qq * np + i] = lag(i, hq.x[qq], &dv);
    }
}
} // namespace

extern "C" {

orc_oracle *orc_create(orc_config const *cfg)
{
  auto *o = new orc_oracle();
  o->cfg = *cfg;
  o->dim = cfg->dim;
  o->deg = cfg->degree;
  o->np = o->deg + 1;
  o->nq = o->np;
  o->nqc = o->dim == 3 ? o->nq * o->nq * o->nq : o->nq * o->nq;
  o->ndc = o->dim == 3 ? o->np * o->np * o->np : o->np * o->np;
  o->nfq = o->dim == 3 ? o->nq * o->nq : o->nq;
  o->nfaces = 2 * o->dim;
  for (int d = 0; d < 3; ++d)
  {
    o->nc[d] = d < o->dim ? cfg->n_cells[d] : 1;
    o->nn[d] = d < o->dim ? o->deg * o->nc[d] + 1 : 1;
    o->h[d] = d < o->dim ? cfg->extent[d] / cfg->n_cells[d] : 1.0;
  }
  o->ncells = o->nc[0] * o->nc[1] * o->nc[2];
  o->nnodes = o->nn[0] * o->nn[1] * o->nn[2];
  o->cell_volume = 1.0;
  for (int d = 0; d < o->dim; ++d)
    o->cell_volume *= o->h[d];
  build_basis(o);
  o->segments.resize(4);
  for (int b = 0; b < cfg->n_sources; ++b)
  {
    orc_source const &s = cfg->sources[b];
    if (s.segments && s.n_segments > 0)
      o->segments[b].assign(s.segments, s.segments + 5 * s.n_segments);
    o->cfg.sources[b].segments = nullptr;
  }
  o->beams.resize(4);
  int n_adiabatic = 0;
  for (int i = 0; i < cfg->n_boundary_types; ++i)
    if (cfg->boundary_types[i] & B_ADIABATIC)
      ++n_adiabatic;
  o->adiabatic_only = n_adiabatic == cfg->n_boundary_types;
  o->active.assign(o->ncells, 1);
  o->matid.assign(o->ncells, 0);
  o->cosv.assign(o->ncells, 1.0);
  o->sinv.assign(o->ncells, 0.0);
  o->has_melted.assign(o->ncells, 0);
  o->node_active.assign(o->nnodes, 0);
  o->inv_mass.assign(o->nnodes, 0.0);
  o->state.assign((size_t)cfg->n_states * o->ncells, 0.0);
  for (int64_t c = 0; c < o->ncells; ++c)
    o->state[c] = 1.0;
  if (cfg->n_states > 1)
    o->liquid_q.assign((size_t)o->ncells * o->nqc, 0.0);
  if (cfg->n_states == 3)
  {
    o->powder_q.assign((size_t)o->ncells * o->nqc, 0.0);
    if (!o->adiabatic_only)
      o->face_powder.assign((size_t)o->ncells * o->nfaces * o->nfq, 0.0);
  }
  return o;
}

void orc_destroy(orc_oracle *o) { delete o; }
int64_t orc_n_nodes(orc_oracle const *o) { return o->nnodes; }
int64_t orc_n_cells(orc_oracle const *o) { return o->ncells; }
int32_t orc_n_qp(orc_oracle const *o) { return o->nqc; }

void orc_set_cells(orc_oracle *o, uint8_t const *active,
                   uint8_t const *material_id, uint8_t const *initial_state,
                   double const *deposition_cos, double const *deposition_sin)
{
  int const ns = o->cfg.n_states;
  for (int64_t c = 0; c < o->ncells; ++c)
  {
    o->active[c] = active ? active[c] : 1;
    o->matid[c] = material_id ? material_id[c] : 0;
    o->cosv[c] = deposition_cos ? deposition_cos[c] : 1.0;
    o->sinv[c] = deposition_sin ? deposition_sin[c] : 0.0;
    // MaterialProperty::set_initial_state (MaterialProperty.templates.hh:755-794)
    int const s = initial_state ? initial_state[c] : 0;
    for (int k = 0; k < ns; ++k)
      o->state[(size_t)k * o->ncells + c] = (k == s) ? 1.0 : 0.0;
  }
}

void orc_set_domain(orc_oracle *o, uint8_t const *domain)
{
  o->domain.clear();
  if (domain)
    o->domain.assign(domain, domain + o->ncells);
}

void orc_setup(orc_oracle *o)
{
  o->update_node_active();
  o->compute_inverse_mass();
  o->get_state_from_material_properties();
}

void orc_set_time(orc_oracle *o, double t) { o->set_time(t); }

void orc_vmult(orc_oracle *o, double *dst, double const *src)
{
  std::fill(dst, dst + o->nnodes, 0.0);
  o->vmult_add(dst, src);
}

void orc_vmult_add(orc_oracle *o, double *dst, double const *src)
{
  o->vmult_add(dst, src);
}

void orc_inverse_mass(orc_oracle const *o, double *out)
{
  std::copy(o->inv_mass.begin(), o->inv_mass.end(), out);
}

void orc_node_active(orc_oracle const *o, uint8_t *out)
{
  std::copy(o->node_active.begin(), o->node_active.end(), out);
}

// evaluate_thermal_physics_impl (ThermalPhysics.templates.hh:43-124) and
// evolve_one_time_step (ThermalPhysics.templates.hh:854-888) with the
// deal.II ExplicitRungeKutta tableaux.
static void evaluate(orc_oracle *o, double t, double const *y, double *f)
{
  o->set_time(t);
  std::fill(f, f + o->nnodes, 0.0);
  o->vmult_add(f, y);
  for (int64_t i = 0; i < o->nnodes; ++i)
    f[i] *= o->inv_mass[i];
}

double orc_evolve_one_time_step(orc_oracle *o, double t, double dt,
                                double *y)
{
  int64_t const n = o->nnodes;
  int const method = o->cfg.time_method;
  if (method == 0)
  {
    std::vector<double> f(n);
    evaluate(o, t, y, f.data());
    for (int64_t i = 0; i < n; ++i)
      y[i] = y[i] + dt * f[i];
    return t + dt;
  }
  std::vector<double> b, c;
  std::vector<std::vector<double>> a;
  if (method == 1)
  {
    b = {0.0, 1.0};
    c = {0.0, 0.5};
    a = {{}, {0.5}};
  }
  else if (method == 2)
  {
    b = {1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0};
    c = {0.0, 0.5, 1.0};
    a = {{}, {0.5}, {-1.0, 2.0}};
  }
  else
  {
    b = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};
    c = {0.0, 0.5, 0.5, 1.0};
    a = {{}, {0.5}, {0.0, 0.5}, {0.0, 0.0, 1.0}};
  }
  int const ns = (int)b.size();
  std::vector<std::vector<double>> fs(ns, std::vector<double>(n));
  std::vector<double> Y(n);
  for (int i = 0; i < ns; ++i)
  {
    std::copy(y, y + n, Y.begin());
    for (int j = 0; j < i; ++j)
    {
      double const s = dt * a[i][j];
      for (int64_t k = 0; k < n; ++k)
        Y[k] = Y[k] + s * fs[j][k];
    }
    evaluate(o, t + c[i] * dt, Y.data(), fs[i].data());
  }
  for (int i = 0; i < ns; ++i)
  {
    double const s = dt * b[i];
    for (int64_t k = 0; k < n; ++k)
      y[k] = y[k] + s * fs[i][k];
  }
  return t + dt;
}

void orc_set_state_to_material_properties(orc_oracle *o)
{
  o->set_state_to_material_properties();
}

void orc_get_state_from_material_properties(orc_oracle *o)
{
  o->get_state_from_material_properties();
}

void orc_get_cell_state(orc_oracle const *o, double *out)
{
  std::copy(o->state.begin(), o->state.end(), out);
}

void orc_set_cell_state(orc_oracle *o, double const *in)
{
  std::copy(in, in + o->state.size(), o->state.begin());
}

void orc_get_qp_powder(orc_oracle const *o, double *out)
{
  std::copy(o->powder_q.begin(), o->powder_q.end(), out);
}

void orc_get_qp_liquid(orc_oracle const *o, double *out)
{
  std::copy(o->liquid_q.begin(), o->liquid_q.end(), out);
}

// MaterialProperty::update (MaterialProperty.templates.hh:244-437)
void orc_evaluate_material_properties(orc_oracle *o, double const *T,
                                      double *pv)
{
  int64_t const C = o->ncells;
  int const ns = o->cfg.n_states;
  std::fill(pv, pv + N_STATE_PROPS * C, 0.0);
  for (int64_t c = 0; c < C; ++c)
  {
    double const Tavg = o->active[c] ? o->cell_average(c, T) : 0.0;
    int const mat = o->matid[c];
    double const solidus = o->cfg.props[mat][SOLIDUS];
    double const liquidus = o->cfg.props[mat][LIQUIDUS];
    double solid_ratio = 1., liquid_ratio = 0.;
    auto st = [&](int s) -> double & { return o->state[(size_t)s * C + c]; };
    if (ns > 1)
    {
      if (Tavg < solidus)
        liquid_ratio = 0.;
      else if (Tavg > liquidus)
        liquid_ratio = 1.;
      else
        liquid_ratio = (Tavg - solidus) / (liquidus - solidus);
      if (ns == 2)
        solid_ratio = 1. - liquid_ratio;
      else
      {
        double const powder_ratio = std::min(1. - liquid_ratio, st(POWDER));
        solid_ratio = 1. - liquid_ratio - powder_ratio;
        st(POWDER) = powder_ratio;
      }
      st(LIQUID) = liquid_ratio;
    }
    st(SOLID) = solid_ratio;
    for (int p = 0; p < N_STATE_PROPS; ++p)
      for (int s = 0; s < ns; ++s)
      {
        if (o->cfg.use_table)
          pv[p * C + c] += st(s) * o->table_lookup(mat, p, s, Tavg);
        else
          for (int i = 0; i <= o->cfg.p_order; ++i)
            pv[p * C + c] +=
                st(s) * o->cfg.poly[mat][p][s][i] * std::pow(Tavg, i);
      }
    if (ns > 1 && liquid_ratio > 0. && liquid_ratio < 1.)
      for (int s = 0; s < ns; ++s)
        pv[SPECIFIC_HEAT * C + c] +=
            st(s) * o->cfg.props[mat][LATENT] / (liquidus - solidus);
    double const T_inf = o->cfg.props[mat][RAD_TINF];
    if (T_inf != DBL_MAX)
    {
      double const e = pv[EMISSIVITY * C + c];
      pv[RAD_COEF * C + c] = e * kStefanBoltzmann * (Tavg + T_inf) *
                             (Tavg * Tavg + T_inf * T_inf);
    }
  }
}

void orc_mark_has_melted(orc_oracle *o, double threshold, double const *T,
                         uint8_t *out)
{
  for (int64_t c = 0; c < o->ncells; ++c)
  {
    if (o->active[c] && !o->has_melted[c])
      if (o->cell_average(c, T) > threshold)
        o->has_melted[c] = 1;
    if (out)
      out[c] = o->has_melted[c];
  }
}

// add_material_start/end (ThermalPhysics.templates.hh:595-825) on the fixed
// full-grid numbering: cell states are averaged, new cells become active,
// nodes that were not DoFs before get new_temperature, the inverse mass is
// recomputed and the cell state is broadcast back to the quadrature points.
void orc_activate_cells(orc_oracle *o, int64_t const *cells, int64_t n,
                        double new_temperature, double const *cos_new,
                        double const *sin_new, double *solution)
{
  o->set_state_to_material_properties();
  std::vector<uint8_t> old_nodes = o->node_active;
  for (int64_t k = 0; k < n; ++k)
  {
    int64_t const c = cells[k];
    if (o->active[c])
      continue;
    o->active[c] = 1;
    o->cosv[c] = cos_new ? cos_new[k] : 1.0;
    o->sinv[c] = sin_new ? sin_new[k] : 0.0;
    o->has_melted[c] = 1;
  }
  o->update_node_active();
  for (int64_t i = 0; i < o->nnodes; ++i)
    if (o->node_active[i] && !old_nodes[i])
      solution[i] = new_temperature;
  o->compute_inverse_mass();
  o->get_state_from_material_properties();
}

void orc_source_values(orc_oracle *o, int32_t beam, double const *points,
                       int64_t n_points, double *out)
{
  for (int64_t i = 0; i < n_points; ++i)
    out[i] = o->source_value(beam, points + 3 * i);
}

void orc_source_state(orc_oracle const *o, int32_t beam, double *out5)
{
  Beam const &b = o->beams[beam];
  out5[0] = b.center[0];
  out5[1] = b.center[1];
  out5[2] = b.center[2];
  out5[3] = b.alpha;
  out5[4] = b.on ? 1.0 : 0.0;
}

} // extern "C"
