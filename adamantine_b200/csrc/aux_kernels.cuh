// Small kernels around the tile kernel: stage preparation (heat-source state
// from the scan path on the device), lumped inverse mass, cell averages and
// material update, state averaging/broadcast, activation.
#pragma once

#include "beam_state.cuh"
#include "device_types.cuh"

#include <cuda_runtime.h>

namespace adm
{

// Set the stage clock of members [0, n): t and dt.
__global__ void set_clock_kernel(MemberData *members, int n, double t, double dt)
{
  int const m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n)
  {
    members[m].clock[0] = t;
    members[m].clock[1] = dt;
  }
}

// clock[0] += clock[1] (end of a captured time step).
__global__ void advance_clock_kernel(MemberData *members, int n)
{
  int const m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < n)
    members[m].clock[0] = members[m].clock[0] + members[m].clock[1];
}

// Heat-source state at t = clock[0] + c * clock[1] for every member and beam:
// ScanPath::value / get_power_modifier (source/ScanPath.cc:197-275) and
// GoldakHeatSource / ElectronBeamHeatSource / CubeHeatSource::update_time
// (source/GoldakHeatSource.cc:24-44, source/ElectronBeamHeatSource.cc:24-45,
// source/CubeHeatSource.cc:45-49). One block per member, one thread per beam.
// Zeroes n doubles (p 16-byte aligned, n even) with the evict-last L2
// policy: the atomic write-out that follows adds into lines still in L2.
// With members != nullptr, block m < n_members also prepares member m's beam
// states for stage coefficient c (stage_prepare_kernel's work, folded into
// the zeroing launch).
__global__ void zero_keep_kernel(double *p, size_t n, MemberData *members, int n_members, double c)
{
  if (members != nullptr && (int)blockIdx.x < n_members && (int)threadIdx.x < members[blockIdx.x].n_beams)
    prepare_beam(members[blockIdx.x], threadIdx.x, c);
  uint64_t const pol = l2_policy_evict_last();
  size_t const n2 = n / 2;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n2; i += (size_t)gridDim.x * blockDim.x)
    st_keep2(p + 2 * i, 0.0, 0.0, pol);
}

__global__ void stage_prepare_kernel(MemberData *members, int n_members, double c)
{
  int const m = blockIdx.x;
  int const b = threadIdx.x;
  if (m >= n_members || b >= members[m].n_beams)
    return;
  prepare_beam(members[m], b, c);
}

// Per-direction cells touching node i: (cell index, local node index).
__device__ __forceinline__ int node_cells(int i, int deg, int nc, int *cell, int *loc)
{
  int n = 0;
  if (deg == 2)
  {
    if (i & 1)
    {
      cell[n] = (i - 1) / 2;
      loc[n++] = 1;
    }
    else
    {
      if (i / 2 - 1 >= 0)
      {
        cell[n] = i / 2 - 1;
        loc[n++] = 2;
      }
      if (i / 2 < nc)
      {
        cell[n] = i / 2;
        loc[n++] = 0;
      }
    }
  }
  else
  {
    if (i - 1 >= 0)
    {
      cell[n] = i - 1;
      loc[n++] = 1;
    }
    if (i < nc)
    {
      cell[n] = i;
      loc[n++] = 0;
    }
  }
  return n;
}

struct GridArgs
{
  int nc[3], nn[3], pitch, deg;
  double vol;
  double glw[3]; // Gauss-Lobatto weights (lumped mass)
};

// compute_inverse_mass_matrix (source/ThermalOperator.templates.hh:118-164):
// Gauss-Lobatto lumped mass of the active cells, inverted on DoFs, 0 elsewhere.
// Inverse lumped mass of node (i, j, k) from the active cells around it.
__device__ __forceinline__ double node_inv_mass(GridArgs const &g, uint32_t const *cell_info, int i, int j, int k)
{
  int cx[2], ax[2], cy[2], ay[2], cz[2], az[2];
  int const nx = node_cells(i, g.deg, g.nc[0], cx, ax);
  int const ny = node_cells(j, g.deg, g.nc[1], cy, ay);
  int const nz = node_cells(k, g.deg, g.nc[2], cz, az);
  double m = 0.0;
  for (int c = 0; c < nz; ++c)
    for (int b = 0; b < ny; ++b)
      for (int a = 0; a < nx; ++a)
      {
        size_t const cell = cx[a] + (size_t)g.nc[0] * (cy[b] + (size_t)g.nc[1] * cz[c]);
        if (cell_info[cell] & CI_ACTIVE)
          m += g.vol * g.glw[ax[a]] * g.glw[ay[b]] * g.glw[az[c]];
      }
  return m > 0.0 ? 1.0 / m : 0.0;
}

__global__ void inverse_mass_kernel(GridArgs g, uint32_t const *cell_info,
                                    double *inv_mass, size_t n_total)
{
  size_t const idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= n_total)
    return;
  int const i = idx % g.pitch;
  size_t const r = idx / g.pitch;
  int const j = r % g.nn[1], k = r / g.nn[1];
  if (i >= g.nn[0])
  {
    inv_mass[idx] = 0.0;
    return;
  }
  inv_mass[idx] = node_inv_mass(g, cell_info, i, j, k);
}

// ------------------------------------------------------------ atomic schedule
// Stage update of the atomic schedule: the tile kernel added every node's
// residual into acc (zeroed before); this pass applies the inverse lumped mass
// and the explicit Runge-Kutta update exactly as the coloured schedule's last
// toucher does (blockIdx.y = member).
__global__ void stage_finalize_kernel(KernelArgs a, size_t n_nodes)
{
  size_t const g = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (g >= n_nodes)
    return;
  MemberData const &md = a.members[blockIdx.y];
  double *const y = a.y_override ? a.y_override : md.y;
  double const dt = md.clock[1];
  double const f = md.inv_mass[g] * md.acc[g];
  if (!isfinite(f))
    atomicCAS(md.error, 0, (int)DERR_NONFINITE);
  double const yv = y[g];
  if (a.n_stages == 1)
  {
    y[g] = yv + dt * f;
    return;
  }
  double const sv = a.stage > 0 ? md.s[g] : 0.0;
  if (!a.last)
  {
    double zn = yv;
    if (a.has_f0)
      zn = zn + (dt * a.a_next_f0) * md.f0[g];
    zn = zn + (dt * a.a_next) * f;
    (a.dst_sel == 1 ? md.za : md.zb)[g] = zn;
    double const sb = (dt * a.b_i) * f;
    md.s[g] = a.stage == 0 ? sb : sv + sb;
    if (a.store_f0)
      md.f0[g] = f;
  }
  else
  {
    y[g] = yv + (sv + (dt * a.b_i) * f);
  }
}

// ------------------------------------------------------------ deposition
// Boxes of material deposition against the cells of the structured mesh.
// Cell (i, j, k) spans [origin + i h, origin + (i + 1) h] per direction (the
// vertices of a subdivided hyper-rectangle); a cell and a box intersect when
// the closed intervals overlap in every direction (touching counts), as the
// bounding-box search of get_elements_to_activate
// (source/material_deposition.cc:374-438) decides.
struct BoxArgs
{
  int nc[3];
  double origin[3], h[3];
  double const *lo; // [n][3]
  double const *hi; // [n][3]
  int64_t b0;       // first box of the launch (block b handles box b0 + b)
};

__device__ __forceinline__ double vertex_coord(double origin, int i, double h)
{
  // no contraction into an FMA: the vertex is origin + (i * h) rounded twice
  return __dadd_rn(origin, __dmul_rn((double)i, h));
}

// Index range [i0, i1] of the cells whose closed extent meets [lo, hi].
__device__ __forceinline__ void box_range(double lo, double hi, double origin, double h, int n, int &i0,
                                          int &i1)
{
  double const fa = floor((lo - origin) / h) - 1.0, fb = floor((hi - origin) / h) + 1.0;
  int a = fa < 0.0 ? 0 : (fa > n - 1 ? n : (int)fa);
  int b = fb < 0.0 ? -1 : (fb > n - 1 ? n - 1 : (int)fb);
  while (a <= b && vertex_coord(origin, a + 1, h) < lo)
    ++a;
  while (b >= a && vertex_coord(origin, b, h) > hi)
    --b;
  i0 = a;
  i1 = b;
}

// Every inactive cell a box meets records the largest such box index (the
// last box of the window sets its deposition direction).
__global__ void box_mark_kernel(BoxArgs a, uint32_t const *cell_info, int32_t *last_box)
{
  int64_t const b = a.b0 + blockIdx.x;
  int r0[3], r1[3];
  for (int d = 0; d < 3; ++d)
    box_range(a.lo[3 * b + d], a.hi[3 * b + d], a.origin[d], a.h[d], a.nc[d], r0[d], r1[d]);
  int64_t const ex = r1[0] - r0[0] + 1, ey = r1[1] - r0[1] + 1, ez = r1[2] - r0[2] + 1;
  if (ex <= 0 || ey <= 0 || ez <= 0)
    return;
  int64_t const total = ex * ey * ez;
  for (int64_t e = threadIdx.x; e < total; e += blockDim.x)
  {
    int const x = r0[0] + (int)(e % ex), y = r0[1] + (int)((e / ex) % ey), z = r0[2] + (int)(e / (ex * ey));
    size_t const c = x + (size_t)a.nc[0] * (y + (size_t)a.nc[1] * z);
    if (!(cell_info[c] & CI_ACTIVE))
      atomicMax(&last_box[c], (int32_t)b);
  }
}

// Appends each marked cell once (by the box that marked it last) to the
// activation list.
__global__ void box_collect_kernel(BoxArgs a, int32_t const *last_box, int64_t *list, int32_t *list_box,
                                   unsigned long long *count, unsigned long long capacity)
{
  int64_t const b = a.b0 + blockIdx.x;
  int r0[3], r1[3];
  for (int d = 0; d < 3; ++d)
    box_range(a.lo[3 * b + d], a.hi[3 * b + d], a.origin[d], a.h[d], a.nc[d], r0[d], r1[d]);
  int64_t const ex = r1[0] - r0[0] + 1, ey = r1[1] - r0[1] + 1, ez = r1[2] - r0[2] + 1;
  if (ex <= 0 || ey <= 0 || ez <= 0)
    return;
  int64_t const total = ex * ey * ez;
  for (int64_t e = threadIdx.x; e < total; e += blockDim.x)
  {
    int const x = r0[0] + (int)(e % ex), y = r0[1] + (int)((e / ex) % ey), z = r0[2] + (int)(e / (ex * ey));
    size_t const c = x + (size_t)a.nc[0] * (y + (size_t)a.nc[1] * z);
    if (last_box[c] == (int32_t)b)
    {
      unsigned long long const slot = atomicAdd(count, 1ull);
      if (slot < capacity)
      {
        list[slot] = (int64_t)c;
        list_box[slot] = (int32_t)b;
      }
    }
  }
}

// New cells become active (material id from matid), take their box's
// deposition direction, count as melted before (the reference's transfer of
// the inactive cells' data), and leave the mark array clean.
__global__ void activate_list_kernel(int64_t const *list, int32_t const *list_box, int64_t n, uint8_t const *matid,
                                     double const *box_cos, double const *box_sin, uint32_t *cell_info,
                                     double *cosv, double *sinv, uint8_t *has_melted, int32_t *last_box)
{
  int64_t const w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= n)
    return;
  int64_t const c = list[w];
  int const b = list_box[w];
  cell_info[c] = CI_ACTIVE | ((uint32_t)(matid[c] & 15) << CI_MAT_SHIFT);
  if (cosv)
  {
    cosv[c] = box_cos[b];
    sinv[c] = box_sin[b];
  }
  has_melted[c] = 1;
  last_box[c] = -1;
}

// Face bits (active boundary / interface) of the listed cells and of their
// six neighbours, from the activity after the activation.
__global__ void face_bits_kernel(int64_t const *list, int64_t n, int nc0, int nc1, int nc2, uint32_t *cell_info)
{
  int64_t const w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (w >= n * 7)
    return;
  int64_t const c0 = list[w / 7];
  int const which = (int)(w % 7);
  int const nc[3] = {nc0, nc1, nc2};
  int cc[3] = {(int)(c0 % nc0), (int)((c0 / nc0) % nc1), (int)(c0 / ((int64_t)nc0 * nc1))};
  if (which > 0)
  {
    int const d = (which - 1) / 2;
    cc[d] += ((which - 1) % 2) ? 1 : -1;
    if (cc[d] < 0 || cc[d] >= nc[d])
      return;
  }
  size_t const c = cc[0] + (size_t)nc0 * (cc[1] + (size_t)nc1 * cc[2]);
  uint32_t const info = cell_info[c];
  if (!(info & CI_ACTIVE))
    return;
  uint32_t out = info & (CI_ACTIVE | (15u << CI_MAT_SHIFT));
  for (int f = 0; f < 6; ++f)
  {
    int const d = f / 2;
    int nb[3] = {cc[0], cc[1], cc[2]};
    nb[d] += (f % 2) ? 1 : -1;
    if (nb[d] < 0 || nb[d] >= nc[d])
      out |= 1u << (CI_FACE_SHIFT + f);
    else if (!(cell_info[nb[0] + (size_t)nc0 * (nb[1] + (size_t)nc1 * nb[2])] & CI_ACTIVE))
      out |= (1u << (CI_FACE_SHIFT + f)) | (1u << (CI_INTERFACE_SHIFT + f));
  }
  cell_info[c] = out;
}

// Inverse lumped mass of the nodes of the listed cells (after activation).
__global__ void inverse_mass_cells_kernel(GridArgs g, uint32_t const *cell_info, int64_t const *list, int64_t n,
                                          double *inv_mass)
{
  int64_t const w = blockIdx.x;
  if (w >= n)
    return;
  int const deg = g.deg, np = deg + 1;
  int64_t const c = list[w];
  int const ccx = c % g.nc[0], ccy = (c / g.nc[0]) % g.nc[1], ccz = c / ((int64_t)g.nc[0] * g.nc[1]);
  for (int l = threadIdx.x; l < np * np * np; l += blockDim.x)
  {
    int const i = deg * ccx + l % np, j = deg * ccy + (l / np) % np, k = deg * ccz + l / (np * np);
    inv_mass[i + (size_t)g.pitch * (j + (size_t)g.nn[1] * k)] = node_inv_mass(g, cell_info, i, j, k);
  }
}

// New DoFs of an activation get new_temperature: nodes of the cells in the
// list that no previously active cell touches (cell_info is the old one).
__global__ void activate_nodes_kernel(GridArgs g, uint32_t const *cell_info,
                                      int64_t const *cells, int64_t n_cells,
                                      double new_temperature, double *y)
{
  int64_t const w = blockIdx.x;
  if (w >= n_cells)
    return;
  int const deg = g.deg, np = deg + 1;
  int64_t const c = cells[w];
  int const ccx = c % g.nc[0];
  int const ccy = (c / g.nc[0]) % g.nc[1];
  int const ccz = c / ((int64_t)g.nc[0] * g.nc[1]);
  for (int l = threadIdx.x; l < np * np * np; l += blockDim.x)
  {
    int const i = deg * ccx + l % np, j = deg * ccy + (l / np) % np,
              k = deg * ccz + l / (np * np);
    int cx[2], ax[2], cy[2], ay[2], cz[2], az[2];
    int const nx = node_cells(i, deg, g.nc[0], cx, ax);
    int const ny = node_cells(j, deg, g.nc[1], cy, ay);
    int const nz = node_cells(k, deg, g.nc[2], cz, az);
    bool old = false;
    for (int c3 = 0; c3 < nz; ++c3)
      for (int b = 0; b < ny; ++b)
        for (int a = 0; a < nx; ++a)
        {
          size_t const cell = cx[a] + (size_t)g.nc[0] * (cy[b] + (size_t)g.nc[1] * cz[c3]);
          if (cell_info[cell] & CI_ACTIVE)
            old = true;
        }
    if (!old)
      y[i + (size_t)g.pitch * (j + (size_t)g.nn[1] * k)] = new_temperature;
  }
}

struct AvgArgs
{
  GridArgs g;
  int nq;        // points per direction
  double S[3][3]; // basis at the points
  double w[3];    // weights on [0,1]
};

// Cell-average temperature: sum_q sum_i phi_i(q) T_i JxW / sum_q sum_i phi_i(q) JxW
// (compute_average, source/MaterialProperty.templates.hh:33-73).
__device__ double cell_average(AvgArgs const &a, double const *T, int cx, int cy, int cz)
{
  int const deg = a.g.deg, np = deg + 1, nq = a.nq;
  double volume = 0.0, avg = 0.0;
  for (int q = 0; q < nq * nq * nq; ++q)
  {
    int const qa = q % nq, qb = (q / nq) % nq, qc = q / (nq * nq);
    double const JxW = a.g.vol * a.w[qa] * a.w[qb] * a.w[qc];
    for (int l = 0; l < np * np * np; ++l)
    {
      int const la = l % np, lb = (l / np) % np, lc = l / (np * np);
      double const phi = a.S[qa][la] * a.S[qb][lb] * a.S[qc][lc];
      size_t const node = (deg * cx + la) +
                          (size_t)a.g.pitch * ((deg * cy + lb) + (size_t)a.g.nn[1] * (deg * cz + lc));
      volume += phi * JxW;
      avg += phi * T[node] * JxW;
    }
  }
  return avg / volume;
}

// MaterialProperty::update (source/MaterialProperty.templates.hh:244-437).
__global__ void material_update_kernel(AvgArgs a, uint32_t const *cell_info,
                                       MaterialDesc const *gm, double const *T,
                                       double *state, double *pv, size_t C)
{
  size_t const c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= C)
    return;
  int const cx = c % a.g.nc[0], cy = (c / a.g.nc[0]) % a.g.nc[1],
            cz = c / ((size_t)a.g.nc[0] * a.g.nc[1]);
  uint32_t const info = cell_info[c];
  double const Tavg = (info & CI_ACTIVE) ? cell_average(a, T, cx, cy, cz) : 0.0;
  int const mat = (info >> CI_MAT_SHIFT) & 15;
  int const ns = gm->n_states;
  double const solidus = gm->props[mat][Q_SOLIDUS];
  double const liquidus = gm->props[mat][Q_LIQUIDUS];
  double solid_ratio = 1.0, liquid_ratio = 0.0;
  if (ns > 1)
  {
    if (Tavg < solidus)
      liquid_ratio = 0.0;
    else if (Tavg > liquidus)
      liquid_ratio = 1.0;
    else
      liquid_ratio = (Tavg - solidus) / (liquidus - solidus);
    if (ns == 2)
      solid_ratio = 1.0 - liquid_ratio;
    else
    {
      double const p_old = state[2 * C + c];
      double const oml = 1.0 - liquid_ratio;
      double const p = (p_old < oml) ? p_old : oml;
      solid_ratio = 1.0 - liquid_ratio - p;
      state[2 * C + c] = p;
    }
    state[C + c] = liquid_ratio;
  }
  state[c] = solid_ratio;
  for (int p = 0; p < kNStateProps; ++p)
  {
    double v = 0.0;
    for (int s = 0; s < ns; ++s)
    {
      double const ratio = state[s * C + c];
      if (gm->use_table)
      {
        double const(*t)[2] = gm->table[mat][p][s];
        double val;
        if (Tavg <= t[0][0])
          val = t[0][1];
        else
        {
          int i = 0;
          for (; i < kTableSize; ++i)
            if (Tavg < t[i][0])
              break;
          if (i >= kTableSize - 1)
            val = t[kTableSize - 1][1];
          else
            val = t[i - 1][1] + (Tavg - t[i - 1][0]) * (t[i][1] - t[i - 1][1]) /
                                    (t[i][0] - t[i - 1][0]);
        }
        v += ratio * val;
      }
      else
      {
        double tp = 1.0;
        for (int i = 0; i <= gm->p_order; ++i)
        {
          v += ratio * gm->poly[mat][p][s][i] * tp;
          tp *= Tavg;
        }
      }
    }
    pv[p * C + c] = v;
  }
  if (ns > 1 && liquid_ratio > 0.0 && liquid_ratio < 1.0)
    for (int s = 0; s < ns; ++s)
      pv[P_SPECIFIC_HEAT * C + c] += state[s * C + c] * gm->props[mat][Q_LATENT] / (liquidus - solidus);
  double const T_inf = gm->props[mat][Q_RAD_TINF];
  if (T_inf != 1.7976931348623157e308)
    pv[P_RAD_COEF * C + c] = pv[P_EMISSIVITY * C + c] * 5.670374419e-8 *
                             (Tavg + T_inf) * (Tavg * Tavg + T_inf * T_inf);
}

// ThermalPhysics::mark_has_melted (source/ThermalPhysics.templates.hh:537-593)
__global__ void has_melted_kernel(AvgArgs a, uint32_t const *cell_info,
                                  double const *T, double threshold,
                                  uint8_t *has_melted, size_t C)
{
  size_t const c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= C)
    return;
  if (!(cell_info[c] & CI_ACTIVE) || has_melted[c])
    return;
  int const cx = c % a.g.nc[0], cy = (c / a.g.nc[0]) % a.g.nc[1],
            cz = c / ((size_t)a.g.nc[0] * a.g.nc[1]);
  if (cell_average(a, T, cx, cy, cz) > threshold)
    has_melted[c] = 1;
}

// set_state_to_material_properties -> MaterialProperty::set_state
// (source/MaterialProperty.templates.hh:537-621): arithmetic means over the
// cell's quadrature points; inactive cells keep their state.
__global__ void set_state_kernel(uint32_t const *cell_info, int ns, int NN,
                                 double const *liquid_sum, uint8_t const *pmode,
                                 double const *pcell, double const *pq,
                                 double *state, size_t C)
{
  size_t const c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= C)
    return;
  if (ns == 1)
  {
    state[c] = 1.0;
    return;
  }
  if (!(cell_info[c] & CI_ACTIVE))
    return;
  double const l = liquid_sum[c] / NN;
  state[C + c] = l;
  if (ns == 2)
  {
    state[c] = 1.0 - l;
    return;
  }
  double ps = 0.0;
  int const mode = pmode[c];
  if (mode == 2)
    for (int q = 0; q < NN; ++q)
      ps += pq[c * NN + q];
  else if (mode == 1)
    for (int q = 0; q < NN; ++q)
      ps += pcell[c];
  double const p = ps / NN;
  state[2 * C + c] = p;
  state[c] = 1.0 - l - p;
}

// MaterialProperty::set_initial_state: state[s][c] = (s == init[c])
__global__ void init_state_kernel(uint8_t const *init, int ns, size_t C, double *state)
{
  size_t const c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= C)
    return;
  for (int s = 0; s < ns; ++s)
    state[(size_t)s * C + c] = init[c] == s ? 1.0 : 0.0;
}

// state[s][cells[k]] = values[k][s] (the other cells were cleared before)
__global__ void scatter_state_kernel(int32_t const *cells, double const *values, size_t n, int ns, size_t C,
                                     double *state)
{
  size_t const k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n)
    return;
  for (int s = 0; s < ns; ++s)
    state[(size_t)s * C + cells[k]] = values[k * ns + s];
}

// out[k][s] = state[s][cells[k]]
__global__ void gather_state_kernel(int32_t const *cells, size_t n, int ns, size_t C, double const *state,
                                    double *out)
{
  size_t const k = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (k >= n)
    return;
  for (int s = 0; s < ns; ++s)
    out[k * ns + s] = state[(size_t)s * C + cells[k]];
}

// get_state_from_material_properties (source/ThermalOperator.templates.hh:753-884):
// broadcast the cell state to the quadrature-point (and face) tables.
__global__ void get_state_kernel(uint32_t const *cell_info, int ns, int NN, int NF,
                                 double const *state, double *liquid_sum,
                                 uint8_t *pmode, double *pcell,
                                 int32_t const *face_slot, double *face_powder,
                                 size_t C)
{
  size_t const c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= C)
    return;
  if (!(cell_info[c] & CI_ACTIVE) || ns == 1)
    return;
  double const l = state[C + c];
  double ls = 0.0;
  for (int q = 0; q < NN; ++q)
    ls += l;
  liquid_sum[c] = ls;
  if (ns == 3)
  {
    double const p = state[2 * C + c];
    pmode[c] = p == 0.0 ? 0 : 1;
    pcell[c] = p;
    if (face_slot)
    {
      int const slot = face_slot[c];
      if (slot >= 0)
        for (int i = 0; i < 6 * NF; ++i)
          face_powder[(size_t)slot * 6 * NF + i] = p;
    }
  }
}

// Expand the powder representation to [C][NN] values (diagnostics).
__global__ void expand_powder_kernel(uint32_t const *cell_info, int NN,
                                     uint8_t const *pmode, double const *pcell,
                                     double const *pq, double *out, size_t C,
                                     uint8_t const *skip)
{
  size_t const idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= C * NN)
    return;
  size_t const c = idx / NN;
  // cells whose skip entry is 0 are left unwritten (no powder at the start
  // of an adjoint run: their readers never look)
  if (skip && skip[c] == 0)
    return;
  int const mode = pmode[c];
  out[idx] = mode == 2 ? pq[idx] : (mode == 1 ? pcell[c] : 0.0);
}

} // namespace adm
