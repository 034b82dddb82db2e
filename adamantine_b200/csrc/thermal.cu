// Host-side implementation of adm::Thermal: set-up, colour-scheduled launches
// of the fused tile kernel, time stepping (with CUDA-graph replay) and the
// state/material/activation entry points.
#include "aux_kernels.cuh"
#include "thermal.hpp"
#include "tile_kernel.cuh" // TileShape / TD only; kernels live in tile_d*_s*.cu

#include <cudaTypedefs.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

namespace adm
{

void check_cuda(cudaError_t e, char const *what, char const *file, int line)
{
  if (e != cudaSuccess)
  {
    (void)cudaGetLastError();
    throw Error(ADM_ERR_CUDA, std::string(what) + " failed at " + file + ":" +
                                  std::to_string(line) + ": " + cudaGetErrorString(e));
  }
}

// ------------------------------------------------------------ 1D rules
namespace
{
void lagrange(int n, long double const *nodes, long double x, long double *v,
              long double *dv)
{
  for (int i = 0; i < n; ++i)
  {
    long double val = 1.0L, der = 0.0L;
    for (int j = 0; j < n; ++j)
    {
      if (j == i)
        continue;
      long double const den = nodes[i] - nodes[j];
      der = der * (x - nodes[j]) / den + val / den;
      val *= (x - nodes[j]) / den;
    }
    v[i] = val;
    dv[i] = der;
  }
}

// The tile kernel's FE_Q(2) contractions skip the entries of the middle Gauss
// point's rows that are exactly 0 or +-1 (S[1] = (0, 1, 0), G[1] = (-1, 0, 1),
// D[1][1] = 0); this checks that the computed rule has them.
void check_q2_structure(Rule1D const &r)
{
  bool const ok = r.S[1][0] == 0.0 && r.S[1][1] == 1.0 && r.S[1][2] == 0.0 && r.G[1][0] == -1.0 &&
                  r.G[1][1] == 0.0 && r.G[1][2] == 1.0 && r.D[1][1] == 0.0;
  if (!ok)
    throw Error(ADM_ERR_UNSUPPORTED, "FE_Q(2) Gauss rule lacks the exact middle-point entries the kernels assume");
}

// The FE_Q(1) cell kernel takes the collocation derivative of the two
// points as one row repeated, D[q] = (-d, d), and equal weights; this checks
// that the computed rule has them exactly.
void check_q1_structure(Rule1D const &r)
{
  bool const ok = r.D[0][0] == r.D[1][0] && r.D[0][1] == r.D[1][1] && r.D[0][0] == -r.D[0][1] &&
                  r.w[0] == r.w[1];
  if (!ok)
    throw Error(ADM_ERR_UNSUPPORTED, "FE_Q(1) rule lacks the exact structure the kernels assume");
}

Rule1D make_rule(int deg, bool lobatto)
{
  Rule1D r;
  int const n = deg + 1;
  r.n = n;
  long double nodes[3], qx[3], qw[3];
  if (deg == 1)
  {
    nodes[0] = 0.0L;
    nodes[1] = 1.0L;
  }
  else
  {
    nodes[0] = 0.0L;
    nodes[1] = 0.5L;
    nodes[2] = 1.0L;
  }
  if (lobatto)
  {
    for (int i = 0; i < n; ++i)
      qx[i] = nodes[i];
    if (n == 2)
    {
      qw[0] = qw[1] = 0.5L;
    }
    else
    {
      qw[0] = qw[2] = 1.0L / 6.0L;
      qw[1] = 4.0L / 6.0L;
    }
  }
  else if (n == 2)
  {
    long double const d = 0.5L / std::sqrt(3.0L);
    qx[0] = 0.5L - d;
    qx[1] = 0.5L + d;
    qw[0] = qw[1] = 0.5L;
  }
  else
  {
    long double const d = 0.5L * std::sqrt(0.6L);
    qx[0] = 0.5L - d;
    qx[1] = 0.5L;
    qx[2] = 0.5L + d;
    qw[0] = qw[2] = 5.0L / 18.0L;
    qw[1] = 8.0L / 18.0L;
  }
  for (int q = 0; q < n; ++q)
  {
    r.x[q] = (double)qx[q];
    r.w[q] = (double)qw[q];
    long double v[3], dv[3];
    lagrange(n, nodes, qx[q], v, dv);
    for (int i = 0; i < n; ++i)
      r.S[q][i] = (double)v[i];
    // nodal-basis derivative at the point
    for (int i = 0; i < n; ++i)
      r.G[q][i] = (double)dv[i];
    // collocation derivative: Lagrange basis through the quadrature points
    lagrange(n, qx, qx[q], v, dv);
    for (int j = 0; j < n; ++j)
      r.D[q][j] = (double)dv[j];
  }
  if (deg == 2 && !lobatto)
    check_q2_structure(r);
  if (deg == 1)
    check_q1_structure(r);
  return r;
}
} // namespace

void check_config(adm_config const &cfg)
{
  if (cfg.dim != 3)
    throw Error(ADM_ERR_UNSUPPORTED, "the GPU path is three-dimensional (dim must be 3)");
  if (cfg.degree != 1 && cfg.degree != 2)
    throw Error(ADM_ERR_UNSUPPORTED, "FE degree must be 1 or 2");
  if (cfg.quadrature != 0 && cfg.quadrature != 1)
    throw Error(ADM_ERR_INVALID, "quadrature must be 0 (Gauss) or 1 (Gauss-Lobatto)");
  for (int d = 0; d < 3; ++d)
  {
    if (cfg.n_cells[d] < 1)
      throw Error(ADM_ERR_INVALID, "n_cells must be positive");
    if (!(cfg.extent[d] > 0.0))
      throw Error(ADM_ERR_INVALID, "extent must be positive");
  }
  if (cfg.n_materials < 1 || cfg.n_materials > kMaxMaterials)
    throw Error(ADM_ERR_INVALID, "n_materials must be in [1, 4]");
  if (cfg.n_states < 1 || cfg.n_states > 3)
    throw Error(ADM_ERR_INVALID, "n_states must be 1, 2 or 3");
  if (cfg.p_order < 0 || cfg.p_order > 4)
    throw Error(ADM_ERR_INVALID, "p_order must be in [0, 4]");
  if (cfg.n_boundary_types < 1 || cfg.n_boundary_types > 8)
    throw Error(ADM_ERR_INVALID, "n_boundary_types must be in [1, 8]");
  if (cfg.n_sources < 0 || cfg.n_sources > kMaxBeams)
    throw Error(ADM_ERR_INVALID, "n_sources must be in [0, 4]");
  if (cfg.time_method < 0 || cfg.time_method > 3)
    throw Error(ADM_ERR_INVALID, "time_method must be in [0, 3]");
  for (int b = 0; b < cfg.n_sources; ++b)
  {
    adm_source const &s = cfg.sources[b];
    if (s.type < 0 || s.type > 2)
      throw Error(ADM_ERR_INVALID, "unknown heat source type");
    if (s.type != 2)
    {
      if (s.n_segments < 0 || (s.n_segments > 0 && !s.segments))
        throw Error(ADM_ERR_INVALID, "scan path segments missing");
      for (int i = 1; i < s.n_segments; ++i)
        if (s.segments[i * 5] < s.segments[(i - 1) * 5])
          throw Error(ADM_ERR_INVALID, "scan path end times must be non-decreasing");
    }
  }
  long double const total = (long double)(cfg.degree * cfg.n_cells[0] + 4) *
                            (cfg.degree * cfg.n_cells[1] + 1) *
                            (cfg.degree * cfg.n_cells[2] + 1);
  if (total > 4.0e9L)
    throw Error(ADM_ERR_INVALID, "mesh too large");
}

void Mesh::init(adm_config const &cfg)
{
  deg = cfg.degree;
  if (deg == 1)
  {
    tx = TileShape<1>::TX;
    ty = TileShape<1>::TY;
    tz = TileShape<1>::TZ;
  }
  else
  {
    tx = TileShape<2>::TX;
    ty = TileShape<2>::TY;
    tz = TileShape<2>::TZ;
  }
  int const t[3] = {tx, ty, tz};
  for (int d = 0; d < 3; ++d)
  {
    nc[d] = cfg.n_cells[d];
    nn[d] = deg * nc[d] + 1;
    h[d] = cfg.extent[d] / nc[d];
    origin[d] = cfg.origin[d];
    nt[d] = (nc[d] + t[d] - 1) / t[d];
  }
  if (nt[0] > 2047 || nt[1] > 2047 || nt[2] > 1023)
    throw Error(ADM_ERR_INVALID, "mesh has too many cell tiles along one axis");
  pitch = (nn[0] + 3) / 4 * 4;
  n_nodes = (size_t)pitch * nn[1] * nn[2];
  n_cells = (size_t)nc[0] * nc[1] * nc[2];
  n_tiles = (size_t)nt[0] * nt[1] * nt[2];
  quad = make_rule(deg, cfg.quadrature == 1);
  gauss = make_rule(deg, false);
  Rule1D gl = make_rule(deg, true);
  for (int i = 0; i < 3; ++i)
    glw[i] = gl.w[i];
}

MaterialDesc make_material(adm_config const &cfg)
{
  MaterialDesc m;
  std::memset(&m, 0, sizeof(m));
  m.n_materials = cfg.n_materials;
  m.n_states = cfg.n_states;
  m.use_table = cfg.use_table;
  m.p_order = cfg.p_order;
  std::memcpy(m.poly, cfg.poly, sizeof(m.poly));
  std::memcpy(m.table, cfg.table, sizeof(m.table));
  std::memcpy(m.props, cfg.props, sizeof(m.props));
  // coefficients above p_order are never used by the reference
  for (int a = 0; a < kMaxMaterials; ++a)
    for (int p = 0; p < kNStateProps; ++p)
      for (int s = 0; s < kMaxStates; ++s)
        for (int i = cfg.p_order + 1; i < kMaxPoly; ++i)
          m.poly[a][p][s][i] = 0.0;
  for (int p = 0; p < kNStateProps; ++p)
  {
    int deg = 0;
    for (int a = 0; a < cfg.n_materials; ++a)
      for (int s = 0; s < cfg.n_states; ++s)
        for (int i = 0; i <= cfg.p_order; ++i)
          if (m.poly[a][p][s][i] != 0.0)
            deg = std::max(deg, i);
    m.prop_deg[p] = deg;
  }
  bool iso = true;
  for (int a = 0; a < cfg.n_materials && iso; ++a)
    for (int s = 0; s < cfg.n_states && iso; ++s)
    {
      if (cfg.use_table)
      {
        for (int i = 0; i < kTableSize; ++i)
          for (int k = 0; k < 2; ++k)
            if (m.table[a][P_KX][s][i][k] != m.table[a][P_KY][s][i][k] ||
                m.table[a][P_KX][s][i][k] != m.table[a][P_KZ][s][i][k])
              iso = false;
      }
      else
      {
        for (int i = 0; i < kMaxPoly; ++i)
          if (m.poly[a][P_KX][s][i] != m.poly[a][P_KY][s][i] ||
              m.poly[a][P_KX][s][i] != m.poly[a][P_KZ][s][i])
            iso = false;
      }
    }
  m.isotropic = iso ? 1 : 0;
  return m;
}

// Neighbour-activity masks of every tile: bit (ox + 1) + 3 (oy + 1) + 9 (oz + 1)
// is set when the tile at offset (ox, oy, oz) exists and is active (bit 13:
// the tile itself). Inactive tiles get their neighbours' bits too (the
// two-pass gather reads the mask of a node's owner tile, active or not).
void neighbour_masks(Mesh const &mesh, std::vector<uint8_t> const &ta, std::vector<uint32_t> &nbr, bool &all_active)
{
  nbr.assign(mesh.n_tiles, 0u);
  all_active = true;
  for (int tz = 0; tz < mesh.nt[2]; ++tz)
    for (int ty = 0; ty < mesh.nt[1]; ++ty)
      for (int tx = 0; tx < mesh.nt[0]; ++tx)
      {
        size_t const tile = tx + (size_t)mesh.nt[0] * (ty + (size_t)mesh.nt[1] * tz);
        if (!ta[tile])
          all_active = false;
        uint32_t mask = 0;
        for (int oz = -1; oz <= 1; ++oz)
          for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox)
            {
              int const ax = tx + ox, ay = ty + oy, az = tz + oz;
              if (ax < 0 || ay < 0 || az < 0 || ax >= mesh.nt[0] || ay >= mesh.nt[1] || az >= mesh.nt[2])
                continue;
              if (ta[ax + (size_t)mesh.nt[0] * (ay + (size_t)mesh.nt[1] * az)])
                mask |= 1u << ((ox + 1) + 3 * (oy + 1) + 9 * (oz + 1));
            }
        nbr[tile] = mask;
      }
}

CellTopology build_topology(Mesh const &mesh, std::vector<uint8_t> const &active,
                            std::vector<uint8_t> const &matid, bool need_slots,
                            std::vector<uint8_t> const *domain)
{
  std::vector<uint8_t> const &inside = domain ? *domain : active;
  CellTopology t;
  size_t const C = mesh.n_cells;
  t.cell_info.assign(C, 0u);
  int const nx = mesh.nc[0], ny = mesh.nc[1], nz = mesh.nc[2];
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x)
      {
        size_t const c = mesh.cell_index(x, y, z);
        if (!active[c])
          continue;
        uint32_t info = CI_ACTIVE | ((uint32_t)(matid[c] & 15) << CI_MAT_SHIFT);
        int const cc[3] = {x, y, z};
        for (int f = 0; f < 6; ++f)
        {
          int const d = f / 2;
          int nb[3] = {cc[0], cc[1], cc[2]};
          nb[d] += (f % 2) ? 1 : -1;
          if (nb[d] < 0 || nb[d] >= mesh.nc[d])
            info |= 1u << (CI_FACE_SHIFT + f);
          else if (!inside[mesh.cell_index(nb[0], nb[1], nb[2])])
            info |= (1u << (CI_FACE_SHIFT + f)) | (1u << (CI_INTERFACE_SHIFT + f));
        }
        t.cell_info[c] = info;
      }
  size_t const T = mesh.n_tiles;
  t.tile_active.assign(T, 0);
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x)
        if (active[mesh.cell_index(x, y, z)])
        {
          size_t const tile = (x / mesh.tx) + (size_t)mesh.nt[0] * ((y / mesh.ty) + (size_t)mesh.nt[1] * (z / mesh.tz));
          t.tile_active[tile] = 1;
        }
  neighbour_masks(mesh, t.tile_active, t.tile_nbr, t.all_tiles_active);
  if (need_slots)
  {
    t.face_slot.assign(C, -1);
    for (size_t c = 0; c < C; ++c)
      if ((t.cell_info[c] & CI_ACTIVE) && ((t.cell_info[c] >> CI_FACE_SHIFT) & 63u))
        t.face_slot[c] = t.n_slots++;
  }
  return t;
}

Thermal::Tableau Thermal::tableau(int method)
{
  // deal.II TimeStepping::ExplicitRungeKutta tableaux
  // (source/ThermalPhysics.templates.hh:449-471); RK2 is explicit midpoint.
  Tableau t;
  std::memset(&t, 0, sizeof(t));
  switch (method)
  {
  case 0:
    t.s = 1;
    t.b[0] = 1.0;
    break;
  case 1:
    t.s = 2;
    t.a[1][0] = 0.5;
    t.b[0] = 0.0;
    t.b[1] = 1.0;
    t.c[1] = 0.5;
    break;
  case 2:
    t.s = 3;
    t.a[1][0] = 0.5;
    t.a[2][0] = -1.0;
    t.a[2][1] = 2.0;
    t.b[0] = 1.0 / 6.0;
    t.b[1] = 2.0 / 3.0;
    t.b[2] = 1.0 / 6.0;
    t.c[1] = 0.5;
    t.c[2] = 1.0;
    break;
  default:
    t.s = 4;
    t.a[1][0] = 0.5;
    t.a[2][1] = 0.5;
    t.a[3][2] = 1.0;
    t.b[0] = 1.0 / 6.0;
    t.b[1] = 1.0 / 3.0;
    t.b[2] = 1.0 / 3.0;
    t.b[3] = 1.0 / 6.0;
    t.c[1] = 0.5;
    t.c[2] = 0.5;
    t.c[3] = 1.0;
    break;
  }
  return t;
}

// ------------------------------------------------------------ Thermal
Thermal::Thermal(adm_config const &cfg, int device, cudaStream_t stream, bool own_stage_vectors)
{
  check_config(cfg);
  cfg_ = cfg;
  device_ = device;
  ADM_CK(cudaSetDevice(device_));
  mesh_.init(cfg_);
  ns_ = cfg_.n_states;
  tab_ = tableau(cfg_.time_method);
  int n_adiabatic = 0;
  for (int i = 0; i < cfg_.n_boundary_types; ++i)
    if (cfg_.boundary_types[i] & B_ADIABATIC)
      ++n_adiabatic;
  adiabatic_only_ = n_adiabatic == cfg_.n_boundary_types;
  segments_.resize(kMaxBeams);
  for (int b = 0; b < cfg_.n_sources; ++b)
  {
    adm_source &s = cfg_.sources[b];
    if (s.n_segments > 0 && s.segments)
      segments_[b].assign(s.segments, s.segments + 5 * s.n_segments);
    s.segments = nullptr;
  }
  // NULL selects the CUDA default stream, so that work the caller enqueues
  // there (copies, other kernels) is ordered with this handle's kernels.
  stream_ = stream;

  size_t const N = mesh_.n_nodes, C = mesh_.n_cells;
  int const NN = (mesh_.deg + 1) * (mesh_.deg + 1) * (mesh_.deg + 1);
  inv_mass_.alloc(N);
  if (own_stage_vectors)
  {
    za_.alloc(N);
    zb_.alloc(N);
    acc_.alloc(N);
    if (tab_.s > 1)
      s_.alloc(N);
    if (cfg_.time_method == 2)
      f0_.alloc(N);
    za_p_ = za_.p;
    zb_p_ = zb_.p;
    acc_p_ = acc_.p;
    s_p_ = s_.p;
    f0_p_ = f0_.p;
    ADM_CK(cudaMemset(acc_.p, 0, N * sizeof(double)));
    ADM_CK(cudaMemset(za_.p, 0, N * sizeof(double)));
    ADM_CK(cudaMemset(zb_.p, 0, N * sizeof(double)));
  }
  if (ns_ > 1)
    liquid_sum_.alloc(C);
  if (ns_ == 3)
  {
    powder_mode_.alloc(C);
    powder_cell_.alloc(C);
    powder_q_.alloc(C * NN);
  }
  state_d_.alloc(C * ns_);
  cell_info_d_.alloc(C);
  has_melted_d_.alloc(C);
  tile_nbr_d_.alloc(mesh_.n_tiles);
  halo_d_.alloc(mesh_.n_tiles * two_pass_halo_size(mesh_.deg));
  clock_.alloc(2);
  error_d_.alloc(1);
  claim_d_.alloc(8);
  mat_d_.alloc(1);
  beam_state_d_.alloc(kMaxBeams);
  member_d_.alloc(1);
  size_t nseg = 0;
  for (auto const &v : segments_)
    nseg += v.size();
  if (nseg)
  {
    segs_.alloc(nseg);
    size_t off = 0;
    for (auto const &v : segments_)
    {
      if (!v.empty())
        ADM_CK(cudaMemcpy(segs_.p + off, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice));
      off += v.size();
    }
  }
  MaterialDesc const m = make_material(cfg_);
  ADM_CK(cudaMemcpy(mat_d_.p, &m, sizeof(m), cudaMemcpyHostToDevice));
  // degree of the common-path Horner: density, specific heat, conductivity
  int pmax = 0;
  for (int p : {(int)P_DENSITY, (int)P_SPECIFIC_HEAT, (int)P_KX, (int)P_KY, (int)P_KZ})
    pmax = std::max(pmax, m.prop_deg[p]);
  poly_p_ = pmax <= 2 ? 2 : 4;
  double const clk[2] = {0.0, 0.0};
  ADM_CK(cudaMemcpy(clock_.p, clk, sizeof(clk), cudaMemcpyHostToDevice));
  ADM_CK(cudaMemset(error_d_.p, 0, sizeof(int32_t)));
  // defaults: every cell active, material 0, solid, no rotation
  set_cells(nullptr, nullptr, nullptr, nullptr, nullptr);
}

Thermal::~Thermal()
{
  if (step_graph_)
    cudaGraphExecDestroy(step_graph_);
  cudaStreamSynchronize(stream_);
  if (copy_in_)
  {
    cudaStreamSynchronize(copy_in_);
    cudaStreamSynchronize(copy_out_);
    cudaStreamDestroy(copy_in_);
    cudaStreamDestroy(copy_out_);
    for (auto e : pipe_ev_)
      cudaEventDestroy(e);
  }
  if (graph_stream_)
  {
    cudaStreamSynchronize(graph_stream_);
    cudaStreamDestroy(graph_stream_);
    cudaEventDestroy(ev_a_);
    cudaEventDestroy(ev_b_);
  }
}

void Thermal::set_cells(uint8_t const *active, uint8_t const *material_id,
                        uint8_t const *initial_state, double const *cosv,
                        double const *sinv)
{
  size_t const C = mesh_.n_cells;
  active_.assign(C, 1);
  matid_.assign(C, 0);
  init_state_.assign(C, 0);
  cos_.assign(C, 1.0);
  sin_.assign(C, 0.0);
  has_melted_.assign(C, 0);
  for (size_t c = 0; c < C; ++c)
  {
    if (active)
      active_[c] = active[c] ? 1 : 0;
    if (material_id)
    {
      if (material_id[c] >= cfg_.n_materials)
        throw Error(ADM_ERR_INVALID, "material id out of range");
      matid_[c] = material_id[c];
    }
    if (initial_state)
    {
      if (initial_state[c] >= ns_)
        throw Error(ADM_ERR_INVALID, "initial state index out of range for the material states");
      init_state_[c] = initial_state[c];
    }
    if (cosv)
      cos_[c] = cosv[c];
    if (sinv)
      sin_[c] = sinv[c];
  }
  setup_done_ = false;
}

void Thermal::set_domain(uint8_t const *domain)
{
  domain_.clear();
  if (domain)
    domain_.assign(domain, domain + mesh_.n_cells);
  setup_done_ = false;
}

void Thermal::rebuild()
{
  size_t const C = mesh_.n_cells;
  has_rotation_ = false;
  for (size_t c = 0; c < C; ++c)
    if (cos_[c] != 1.0 || sin_[c] != 0.0)
    {
      has_rotation_ = true;
      break;
    }
  bool const need_slots = (ns_ == 3) && !adiabatic_only_;
  topo_ = build_topology(mesh_, active_, matid_, need_slots, domain_.empty() ? nullptr : &domain_);
  ADM_CK(cudaMemcpyAsync(cell_info_d_.p, topo_.cell_info.data(), C * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaMemcpyAsync(tile_nbr_d_.p, topo_.tile_nbr.data(), mesh_.n_tiles * sizeof(uint32_t), cudaMemcpyHostToDevice, stream_));
  // the two-pass gather reads the halo arrays of inactive tiles as zeros
  ADM_CK(cudaMemsetAsync(halo_d_.p, 0, halo_d_.n * sizeof(double), stream_));
  if (has_rotation_)
  {
    cos_d_.alloc(C);
    sin_d_.alloc(C);
    ADM_CK(cudaMemcpyAsync(cos_d_.p, cos_.data(), C * sizeof(double), cudaMemcpyHostToDevice, stream_));
    ADM_CK(cudaMemcpyAsync(sin_d_.p, sin_.data(), C * sizeof(double), cudaMemcpyHostToDevice, stream_));
  }
  if (need_slots)
  {
    int const NF = (mesh_.deg + 1) * (mesh_.deg + 1);
    face_slot_d_.alloc(C);
    ADM_CK(cudaMemcpyAsync(face_slot_d_.p, topo_.face_slot.data(), C * sizeof(int32_t), cudaMemcpyHostToDevice, stream_));
    face_powder_.alloc(std::max<size_t>(1, (size_t)topo_.n_slots * 6 * NF));
  }
  // colour work lists
  work_.clear();
  for (int col = 0; col < 8; ++col)
  {
    colour_off_[col] = (int)work_.size();
    // top layers first: the beam works the top surface, so the slow tiles
    // (melt pool, source) are claimed early and the others balance them
    int const tz_top = mesh_.nt[2] - 1 - (((mesh_.nt[2] - 1) ^ (col >> 2)) & 1);
    for (int tz = tz_top; tz >= 0; tz -= 2)
      for (int ty = (col >> 1) & 1; ty < mesh_.nt[1]; ty += 2)
        for (int tx = col & 1; tx < mesh_.nt[0]; tx += 2)
        {
          size_t const tile = tx + (size_t)mesh_.nt[0] * (ty + (size_t)mesh_.nt[1] * tz);
          if (topo_.tile_active[tile])
            work_.push_back(TileWork{0, (int32_t)tile, pack_tile(tx, ty, tz)});
        }
  }
  colour_off_[8] = (int)work_.size();
  build_atomic_list(topo_.tile_active);
  ++work_version_;
  work_d_.ensure(std::max<size_t>(1, work_.size()));
  if (!work_.empty())
    ADM_CK(cudaMemcpyAsync(work_d_.p, work_.data(), work_.size() * sizeof(TileWork), cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaMemcpyAsync(has_melted_d_.p, has_melted_.data(), C, cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  if (step_graph_)
  {
    cudaGraphExecDestroy(step_graph_);
    step_graph_ = nullptr;
  }
  upload_member();
}

void Thermal::upload_member()
{
  MemberData &md = md_;
  std::memset(&md, 0, sizeof(md));
  md.y = nullptr;
  md.za = za_p_;
  md.zb = zb_p_;
  md.s = s_p_;
  md.f0 = f0_p_;
  md.acc = acc_p_;
  md.inv_mass = inv_mass_.p;
  md.cell_info = cell_info_d_.p;
  md.powder_mode = powder_mode_.p;
  md.powder_cell = powder_cell_.p;
  md.powder_q = powder_q_.p;
  md.liquid_sum = liquid_sum_.p;
  md.face_slot = face_slot_d_.p;
  md.face_powder = face_powder_.p;
  md.cosv = cos_d_.p;
  md.sinv = sin_d_.p;
  md.tile_nbr = tile_nbr_d_.p;
  md.halo = halo_d_.p;
  md.mat = mat_d_.p;
  md.beam_state = beam_state_d_.p;
  md.clock = clock_.p;
  md.error = error_d_.p;
  md.n_beams = cfg_.n_sources;
  md.has_rotation = has_rotation_ ? 1 : 0;
  size_t off = 0;
  for (int b = 0; b < cfg_.n_sources; ++b)
  {
    adm_source const &s = cfg_.sources[b];
    BeamDesc &bd = md.beams[b];
    bd.type = s.type;
    bd.n_segments = (int)(segments_[b].size() / 5);
    bd.segments = segments_[b].empty() ? nullptr : segs_.p + off;
    off += segments_[b].size();
    bd.depth = s.depth;
    bd.absorption_efficiency = s.absorption_efficiency;
    bd.radius_squared = s.radius_squared;
    bd.max_power = s.max_power;
    bd.cube_start_time = s.cube_start_time;
    bd.cube_end_time = s.cube_end_time;
    bd.cube_value = s.cube_value;
    for (int d = 0; d < 3; ++d)
    {
      bd.cube_min[d] = s.cube_min[d];
      bd.cube_max[d] = s.cube_max[d];
    }
  }
  md.pi_over_3_to_1p5 = std::pow(3.14159265358979323846 / 3.0, 1.5);
  md.log_01 = std::log(0.1);
  ADM_CK(cudaMemcpyAsync(member_d_.p, &md, sizeof(md), cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
}

void Thermal::setup()
{
  ADM_CK(cudaSetDevice(device_));
  size_t const C = mesh_.n_cells;
  rebuild();
  // MaterialProperty::set_initial_state (on the device from the per-cell
  // state index)
  scratch_u8_.ensure(std::max<size_t>(1, C));
  ADM_CK(cudaMemcpyAsync(scratch_u8_.p, init_state_.data(), C, cudaMemcpyHostToDevice, stream_));
  init_state_kernel<<<(unsigned)((C + 255) / 256), 256, 0, stream_>>>(scratch_u8_.p, ns_, C, state_d_.p);
  ADM_CK(cudaGetLastError());
  if (ns_ == 3)
  {
    ADM_CK(cudaMemsetAsync(powder_mode_.p, 0, C, stream_));
    ADM_CK(cudaMemsetAsync(powder_cell_.p, 0, C * sizeof(double), stream_));
  }
  compute_inverse_mass_matrix();
  get_state_from_material_properties();
  set_clock(0.0, 0.0);
  ADM_CK(cudaStreamSynchronize(stream_));
  setup_done_ = true;
}

KernelArgs Thermal::base_args() const
{
  KernelArgs a;
  std::memset(&a, 0, sizeof(a));
  a.work = work_d_.p;
  a.members = member_d_.p;
  for (int d = 0; d < 3; ++d)
  {
    a.nc[d] = mesh_.nc[d];
    a.nn[d] = mesh_.nn[d];
    a.nt[d] = mesh_.nt[d];
    a.h[d] = mesh_.h[d];
    a.origin[d] = mesh_.origin[d];
  }
  a.pitch = mesh_.pitch;
  a.cells_per_thread = cells_per_thread_;
  a.faces = adiabatic_only_ ? 0 : 1;
  int const nb = cfg_.n_boundary_types;
  for (int f = 0; f < 6; ++f)
    a.boundary_type[f] = f < nb - 1 ? cfg_.boundary_types[f] : cfg_.boundary_types[nb - 1];
  a.interface_type = cfg_.boundary_types[nb - 1];
  double const vol = mesh_.h[0] * mesh_.h[1] * mesh_.h[2];
  a.vol = vol;
  for (int d = 0; d < 3; ++d)
  {
    a.vol_over_h2[d] = vol / (mesh_.h[d] * mesh_.h[d]);
    a.vol_over_h[d] = vol / mesh_.h[d];
    a.inv_h[d] = 1.0 / mesh_.h[d];
  }
  Rule1D const &r = mesh_.quad;
  std::memcpy(a.S, r.S, sizeof(a.S));
  std::memcpy(a.D, r.D, sizeof(a.D));
  std::memcpy(a.G, r.G, sizeof(a.G));
  std::memcpy(a.qw, r.w, sizeof(a.qw));
  std::memcpy(a.qx, r.x, sizeof(a.qx));
  int const n = r.n;
  for (int q = 0; q < n * n * n; ++q)
  {
    double const W = r.w[q % n] * r.w[(q / n) % n] * r.w[q / (n * n)];
    for (int d = 0; d < 3; ++d)
      a.cw[q][d] = W * a.vol_over_h2[d];
    a.cw[q][3] = W * vol;
  }
  return a;
}

void launch_tile_d1_s1_p2(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d1_s1_p4(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d1_s2_p2(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d1_s2_p4(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d1_s3_p2(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d1_s3_p4(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d2_s1_p2(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d2_s1_p4(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d2_s2_p2(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d2_s2_p4(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d2_s3_p2(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);
void launch_tile_d2_s3_p4(CUtensorMap const &, KernelArgs const &, int, cudaStream_t);

// P is the polynomial degree the common-path Horner evaluates (2 or 4).
void launch_tile(int deg, int ns, int p, CUtensorMap const &map, KernelArgs const &a, int n_items,
                 cudaStream_t stream)
{
  switch (deg * 100 + ns * 10 + p)
  {
  case 112:
    launch_tile_d1_s1_p2(map, a, n_items, stream);
    break;
  case 114:
    launch_tile_d1_s1_p4(map, a, n_items, stream);
    break;
  case 122:
    launch_tile_d1_s2_p2(map, a, n_items, stream);
    break;
  case 124:
    launch_tile_d1_s2_p4(map, a, n_items, stream);
    break;
  case 132:
    launch_tile_d1_s3_p2(map, a, n_items, stream);
    break;
  case 134:
    launch_tile_d1_s3_p4(map, a, n_items, stream);
    break;
  case 212:
    launch_tile_d2_s1_p2(map, a, n_items, stream);
    break;
  case 214:
    launch_tile_d2_s1_p4(map, a, n_items, stream);
    break;
  case 222:
    launch_tile_d2_s2_p2(map, a, n_items, stream);
    break;
  case 224:
    launch_tile_d2_s2_p4(map, a, n_items, stream);
    break;
  case 232:
    launch_tile_d2_s3_p2(map, a, n_items, stream);
    break;
  case 234:
    launch_tile_d2_s3_p4(map, a, n_items, stream);
    break;
  default:
    throw Error(ADM_ERR_INVALID, "no tile kernel for this degree / state count / polynomial order");
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no -lcuda).
static PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn)
  {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    ADM_CK(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess)
      throw Error(ADM_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor map of node vectors for the TMA brick loads: a 4D box of
// (BXP, BY, BZ, 1) nodes over the (nn0, nn1, nn2, members) array with row
// pitch `pitch` and member_stride doubles between members.
CUtensorMap brick_map(Mesh const &m, double const *base, int n_members, size_t member_stride, int tz_cells)
{
  CUtensorMap map;
  std::memset(&map, 0, sizeof(map));
  if ((reinterpret_cast<uintptr_t>(base) & 15u) != 0)
    throw Error(ADM_ERR_INVALID, "node vectors must be 16-byte aligned");
  if (n_members < 1 || (n_members > 1 && (member_stride * sizeof(double)) % 16 != 0) ||
      member_stride < m.n_nodes)
    throw Error(ADM_ERR_INVALID, "member stride must cover a node vector and be a multiple of 2 doubles");
  cuuint64_t const dims[4] = {(cuuint64_t)m.nn[0], (cuuint64_t)m.nn[1], (cuuint64_t)m.nn[2],
                              (cuuint64_t)n_members};
  cuuint64_t const strides[3] = {(cuuint64_t)m.pitch * sizeof(double),
                                 (cuuint64_t)m.pitch * m.nn[1] * sizeof(double),
                                 (cuuint64_t)member_stride * sizeof(double)};
  cuuint32_t box[4];
  box[3] = 1;
  if (m.deg == 1)
  {
    box[0] = TD<1>::BXP;
    box[1] = TD<1>::BY;
    box[2] = TD<1>::BZ;
  }
  else
  {
    box[0] = TD<2>::BXP;
    box[1] = TD<2>::BY;
    box[2] = tz_cells > 0 ? (cuuint32_t)(2 * tz_cells + 1) : (cuuint32_t)TD<2>::BZ;
  }
  cuuint32_t const elem[4] = {1, 1, 1, 1};
  CUresult const r = encode_fn()(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<double *>(base), dims,
                                 strides, box, elem, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                 CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS)
    throw Error(ADM_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return map;
}

void Thermal::launch_pass(KernelArgs a, double const *src)
{
  CUtensorMap const map = brick_map(mesh_, src, 1, mesh_.n_nodes);
  if (schedule_ == kScheduleTwoPass)
  {
    // one launch over every tile (no atomics): each node's owner writes it,
    // the partial sums of nodes on a tile's upper faces go to its halo
    // array, and the gather pass completes the shared nodes in a fixed
    // order; a stage then applies the update over all nodes
    int const count = colour_off_[8];
    a.two_pass = 1;
    if (count > 0)
    {
      a.work = awork_d_.p;
      launch_tile(mesh_.deg, ns_, poly_p_, map, a, count, stream_);
      ADM_CK(cudaGetLastError());
    }
    launch_two_pass_gather(mesh_.deg, a, 1, stream_);
    if (a.mode == 2)
      launch_stage_finalize(a, mesh_.n_nodes, 1, stream_);
    return;
  }
  if (schedule_ == kScheduleAtomic)
  {
    // one launch over every tile (the ascending list), items strided over
    // the CTAs (measured faster here than claiming them from a counter);
    // with 128-cell blocks over the z-pairs of tiles
    int count = colour_off_[8];
    size_t const N = mesh_.n_nodes;
    a.atomic = 1;
    CUtensorMap map_used = map;
    if (cells_per_block_ == 128)
    {
      build_pair_list();
      count = (int)pwork_.size();
      a.tile_pairs = 1;
      a.nt[2] = (mesh_.nt[2] + 1) / 2;
      a.work = pwork_d_.p;
      map_used = brick_map(mesh_, src, 1, mesh_.n_nodes, 2 * mesh_.tz);
    }
    if (a.mode == 2)
      launch_zero_keep(acc_p_, N, stream_, fold_prepare_c_ >= 0.0 ? member_d_.p : nullptr, 1, fold_prepare_c_);
    if (count > 0)
    {
      if (!a.tile_pairs)
        a.work = awork_d_.p;
      launch_tile(mesh_.deg, ns_, poly_p_, map_used, a, count, stream_);
      ADM_CK(cudaGetLastError());
    }
    if (a.mode == 2)
    {
      stage_finalize_kernel<<<dim3((unsigned)((N + 255) / 256), 1), 256, 0, stream_>>>(a, N);
      ADM_CK(cudaGetLastError());
    }
    return;
  }
  // colour launches claim their items from zeroed counters: a colour ends
  // with its slowest CTA, and a CTA held up by a tile under the beam takes
  // fewer of the others
  ADM_CK(cudaMemsetAsync(claim_d_.p, 0, 8 * sizeof(int32_t), stream_));
  for (int col = 0; col < 8; ++col)
  {
    int const count = colour_off_[col + 1] - colour_off_[col];
    if (count == 0)
      continue;
    a.work = work_d_.p + colour_off_[col];
    a.claim = claim_d_.p + col;
    launch_tile(mesh_.deg, ns_, poly_p_, map, a, count, stream_);
    ADM_CK(cudaGetLastError());
  }
}

void launch_set_clock(MemberData *members, int n, double t, double dt, cudaStream_t stream)
{
  set_clock_kernel<<<(n + 31) / 32, 32, 0, stream>>>(members, n, t, dt);
  ADM_CK(cudaGetLastError());
}

void launch_advance_clock(MemberData *members, int n, cudaStream_t stream)
{
  advance_clock_kernel<<<(n + 31) / 32, 32, 0, stream>>>(members, n);
  ADM_CK(cudaGetLastError());
}

void launch_stage_prepare(MemberData *members, int n, double c, cudaStream_t stream)
{
  stage_prepare_kernel<<<n, 32, 0, stream>>>(members, n, c);
  ADM_CK(cudaGetLastError());
}

void launch_zero_keep(double *p, size_t n, cudaStream_t stream, MemberData *members, int n_members, double c)
{
  if ((reinterpret_cast<uintptr_t>(p) & 15u) != 0 || (n & 1u) != 0)
  {
    ADM_CK(cudaMemsetAsync(p, 0, n * sizeof(double), stream));
    if (members != nullptr)
      launch_stage_prepare(members, n_members, c, stream);
    return;
  }
  size_t blocks = std::min<size_t>((n / 2 + 255) / 256, 148 * 16);
  blocks = std::max<size_t>(blocks, members != nullptr ? (size_t)n_members : 1);
  zero_keep_kernel<<<(unsigned)blocks, 256, 0, stream>>>(p, n, members, n_members, c);
  ADM_CK(cudaGetLastError());
}

void launch_stage_finalize(KernelArgs const &a, size_t n_nodes, int n_members, cudaStream_t stream)
{
  stage_finalize_kernel<<<dim3((unsigned)((n_nodes + 255) / 256), (unsigned)n_members), 256, 0, stream>>>(a, n_nodes);
  ADM_CK(cudaGetLastError());
}

void launch_expand_powder(uint32_t const *cell_info, int NN, uint8_t const *pmode, double const *pcell,
                          double const *pq, double *out, size_t C, cudaStream_t stream, uint8_t const *skip)
{
  expand_powder_kernel<<<(unsigned)((C * NN + 255) / 256), 256, 0, stream>>>(cell_info, NN, pmode, pcell, pq,
                                                                            out, C, skip);
  ADM_CK(cudaGetLastError());
}

void Thermal::set_clock(double t, double dt)
{
  set_clock_kernel<<<1, 32, 0, stream_>>>(member_d_.p, 1, t, dt);
  ADM_CK(cudaGetLastError());
}

void Thermal::prepare_stage(double c)
{
  if (cfg_.n_sources == 0)
    return;
  stage_prepare_kernel<<<1, 32, 0, stream_>>>(member_d_.p, 1, c);
  ADM_CK(cudaGetLastError());
}

void Thermal::set_time(double t)
{
  op_time_ = t;
  set_clock(t, 0.0);
}

void Thermal::vmult(double *dst, double const *src, bool add)
{
  NvtxRange const nvtx_range("adm::vmult");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  ADM_CK(cudaSetDevice(device_));
  // Nodes that only inactive tiles touch are not written by the tile kernel;
  // the atomic schedule adds into a zeroed vector.
  // (the two-pass gather writes every node itself)
  // (the beam preparation rides along with the zeroing launch when there is one)
  if (!add && schedule_ != kScheduleTwoPass && (!topo_.all_tiles_active || schedule_ == kScheduleAtomic))
    launch_zero_keep(dst, mesh_.n_nodes, stream_, cfg_.n_sources > 0 ? member_d_.p : nullptr, 1, 0.0);
  else
    prepare_stage(0.0);
  KernelArgs a = base_args();
  a.mode = add ? 1 : 0;
  a.vsrc = src;
  a.vdst = dst;
  launch_pass(a, src);
}

void Thermal::set_step_clock(double t, double dt)
{
  ADM_CK(cudaSetDevice(device_));
  op_time_ = t;
  set_clock(t, dt);
}

void Thermal::vmult_stage(double *dst, double const *src, double c)
{
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  if (schedule_ != kScheduleTwoPass && (!topo_.all_tiles_active || schedule_ == kScheduleAtomic))
    launch_zero_keep(dst, mesh_.n_nodes, stream_, cfg_.n_sources > 0 ? member_d_.p : nullptr, 1, c);
  else
    prepare_stage(c);
  KernelArgs a = base_args();
  a.mode = 0;
  a.vsrc = src;
  a.vdst = dst;
  launch_pass(a, src);
}

// Kernel arguments of RK stage i: stage input y (i == 0) or the stage vector
// the previous stage wrote; za/zb alternate as stage outputs.
KernelArgs Thermal::stage_args(int i) const
{
  KernelArgs a = base_args();
  a.mode = 2;
  a.stage = i;
  a.n_stages = tab_.s;
  a.last = i == tab_.s - 1;
  a.src_sel = i == 0 ? 0 : ((i & 1) ? 1 : 2);
  a.dst_sel = (i & 1) ? 2 : 1;
  a.c_stage = tab_.c[i];
  a.b_i = tab_.b[i];
  if (i + 1 < tab_.s)
  {
    a.a_next = tab_.a[i + 1][i];
    if (i >= 1 && tab_.a[i + 1][0] != 0.0)
    {
      a.has_f0 = 1;
      a.a_next_f0 = tab_.a[i + 1][0];
    }
  }
  if (i == 0)
    for (int k = 2; k < tab_.s; ++k)
      if (tab_.a[k][0] != 0.0)
        a.store_f0 = 1;
  return a;
}

void Thermal::launch_step(double *solution)
{
  for (int i = 0; i < tab_.s; ++i)
  {
    // the atomic schedule's zeroing launch prepares the beams itself
    if (schedule_ == kScheduleAtomic && cfg_.n_sources > 0)
      fold_prepare_c_ = tab_.c[i];
    else
      prepare_stage(tab_.c[i]);
    KernelArgs a = stage_args(i);
    a.y_override = solution;
    launch_pass(a, i == 0 ? solution : (a.src_sel == 1 ? za_p_ : zb_p_));
    fold_prepare_c_ = -1.0;
  }
}

double Thermal::evolve_one_time_step(double t, double dt, double *solution)
{
  NvtxRange const nvtx_range("adm::evolve_one_time_step");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  ADM_CK(cudaSetDevice(device_));
  set_clock(t, dt);
  launch_step(solution);
  op_time_ = t + tab_.c[tab_.s - 1] * dt;
  set_clock(op_time_, 0.0);
  return t + dt;
}

double Thermal::evolve_n_steps(double t, double dt, int n, double *solution)
{
  NvtxRange const nvtx_range("adm::evolve_n_steps");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  if (n <= 0)
    return t;
  ADM_CK(cudaSetDevice(device_));
  if (!graph_stream_)
  {
    ADM_CK(cudaStreamCreateWithFlags(&graph_stream_, cudaStreamNonBlocking));
    ADM_CK(cudaEventCreateWithFlags(&ev_a_, cudaEventDisableTiming));
    ADM_CK(cudaEventCreateWithFlags(&ev_b_, cudaEventDisableTiming));
  }
  if (!step_graph_ || graph_solution_ != solution)
  {
    if (step_graph_)
    {
      cudaGraphExecDestroy(step_graph_);
      step_graph_ = nullptr;
    }
    // the legacy default stream cannot be captured: capture on our own stream
    cudaStream_t const saved = stream_;
    stream_ = graph_stream_;
    cudaGraph_t graph;
    ADM_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try
    {
      launch_step(solution);
      advance_clock_kernel<<<1, 32, 0, stream_>>>(member_d_.p, 1);
    }
    catch (...)
    {
      cudaStreamEndCapture(stream_, &graph);
      stream_ = saved;
      throw;
    }
    cudaError_t const e = cudaStreamEndCapture(stream_, &graph);
    stream_ = saved;
    ADM_CK(e);
    ADM_CK(cudaGraphInstantiate(&step_graph_, graph, 0));
    cudaGraphDestroy(graph);
    graph_solution_ = solution;
  }
  set_clock(t, dt);
  ADM_CK(cudaEventRecord(ev_a_, stream_));
  ADM_CK(cudaStreamWaitEvent(graph_stream_, ev_a_, 0));
  double tt = t;
  for (int k = 0; k < n; ++k)
  {
    ADM_CK(cudaGraphLaunch(step_graph_, graph_stream_));
    tt = tt + dt;
  }
  ADM_CK(cudaEventRecord(ev_b_, graph_stream_));
  ADM_CK(cudaStreamWaitEvent(stream_, ev_b_, 0));
  op_time_ = (tt - dt) + tab_.c[tab_.s - 1] * dt;
  set_clock(op_time_, 0.0);
  return tt;
}

void Thermal::compute_inverse_mass_matrix()
{
  GridArgs g;
  for (int d = 0; d < 3; ++d)
  {
    g.nc[d] = mesh_.nc[d];
    g.nn[d] = mesh_.nn[d];
  }
  g.pitch = mesh_.pitch;
  g.deg = mesh_.deg;
  g.vol = mesh_.h[0] * mesh_.h[1] * mesh_.h[2];
  for (int i = 0; i < 3; ++i)
    g.glw[i] = mesh_.glw[i];
  size_t const N = mesh_.n_nodes;
  inverse_mass_kernel<<<(unsigned)((N + 255) / 256), 256, 0, stream_>>>(g, cell_info_d_.p, inv_mass_.p, N);
  ADM_CK(cudaGetLastError());
}

void Thermal::get_state_from_material_properties()
{
  size_t const C = mesh_.n_cells;
  int const np = mesh_.deg + 1;
  get_state_kernel<<<(unsigned)((C + 255) / 256), 256, 0, stream_>>>(
      cell_info_d_.p, ns_, np * np * np, np * np, state_d_.p, liquid_sum_.p,
      powder_mode_.p, powder_cell_.p, face_slot_d_.p, face_powder_.p, C);
  ADM_CK(cudaGetLastError());
}

void Thermal::set_state_to_material_properties()
{
  size_t const C = mesh_.n_cells;
  int const np = mesh_.deg + 1;
  set_state_kernel<<<(unsigned)((C + 255) / 256), 256, 0, stream_>>>(
      cell_info_d_.p, ns_, np * np * np, liquid_sum_.p, powder_mode_.p,
      powder_cell_.p, powder_q_.p, state_d_.p, C);
  ADM_CK(cudaGetLastError());
}

static AvgArgs avg_args(Mesh const &m, Rule1D const &r)
{
  AvgArgs a;
  std::memset(&a, 0, sizeof(a));
  for (int d = 0; d < 3; ++d)
  {
    a.g.nc[d] = m.nc[d];
    a.g.nn[d] = m.nn[d];
  }
  a.g.pitch = m.pitch;
  a.g.deg = m.deg;
  a.g.vol = m.h[0] * m.h[1] * m.h[2];
  a.nq = r.n;
  std::memcpy(a.S, r.S, sizeof(a.S));
  std::memcpy(a.w, r.w, sizeof(a.w));
  return a;
}

void Thermal::evaluate_material_properties(double const *temperature, double *pv)
{
  size_t const C = mesh_.n_cells;
  AvgArgs a = avg_args(mesh_, mesh_.gauss);
  material_update_kernel<<<(unsigned)((C + 127) / 128), 128, 0, stream_>>>(
      a, cell_info_d_.p, mat_d_.p, temperature, state_d_.p, pv, C);
  ADM_CK(cudaGetLastError());
}

void Thermal::get_cell_state(double *host)
{
  ADM_CK(cudaMemcpyAsync(host, state_d_.p, state_d_.n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
}

void Thermal::set_cell_state(double const *host)
{
  ADM_CK(cudaMemcpyAsync(state_d_.p, host, state_d_.n * sizeof(double), cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
}

void Thermal::get_cell_state_sparse(int32_t const *cells, size_t n, double *out)
{
  size_t const C = mesh_.n_cells;
  for (size_t k = 0; k < n; ++k)
    if (cells[k] < 0 || (size_t)cells[k] >= C)
      throw Error(ADM_ERR_INVALID, "cell index out of range");
  if (n == 0)
    return;
  scratch_i32_.ensure(n);
  scratch_f64_.ensure(n * ns_);
  ADM_CK(cudaMemcpyAsync(scratch_i32_.p, cells, n * sizeof(int32_t), cudaMemcpyHostToDevice, stream_));
  gather_state_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream_>>>(scratch_i32_.p, n, ns_, C, state_d_.p,
                                                                       scratch_f64_.p);
  ADM_CK(cudaGetLastError());
  ADM_CK(cudaMemcpyAsync(out, scratch_f64_.p, n * ns_ * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
}

void Thermal::set_cell_state_sparse(int32_t const *cells, double const *values, size_t n)
{
  size_t const C = mesh_.n_cells;
  for (size_t k = 0; k < n; ++k)
    if (cells[k] < 0 || (size_t)cells[k] >= C)
      throw Error(ADM_ERR_INVALID, "cell index out of range");
  ADM_CK(cudaMemsetAsync(state_d_.p, 0, state_d_.n * sizeof(double), stream_));
  if (n > 0)
  {
    scratch_i32_.ensure(n);
    scratch_f64_.ensure(n * ns_);
    ADM_CK(cudaMemcpyAsync(scratch_i32_.p, cells, n * sizeof(int32_t), cudaMemcpyHostToDevice, stream_));
    ADM_CK(cudaMemcpyAsync(scratch_f64_.p, values, n * ns_ * sizeof(double), cudaMemcpyHostToDevice, stream_));
    scatter_state_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream_>>>(scratch_i32_.p, scratch_f64_.p, n, ns_,
                                                                          C, state_d_.p);
    ADM_CK(cudaGetLastError());
  }
  ADM_CK(cudaStreamSynchronize(stream_)); // the host arrays may go once this returns
}

void Thermal::get_qp_powder(double *host)
{
  size_t const C = mesh_.n_cells;
  int const np = mesh_.deg + 1, NN = np * np * np;
  if (ns_ != 3)
  {
    std::fill(host, host + C * NN, 0.0);
    return;
  }
  DevBuf<double> tmp;
  tmp.alloc(C * NN);
  expand_powder_kernel<<<(unsigned)((C * NN + 255) / 256), 256, 0, stream_>>>(
      cell_info_d_.p, NN, powder_mode_.p, powder_cell_.p, powder_q_.p, tmp.p, C, nullptr);
  ADM_CK(cudaGetLastError());
  ADM_CK(cudaMemcpyAsync(host, tmp.p, C * NN * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
}

void Thermal::mark_has_melted(double threshold, double const *temperature, uint8_t *host)
{
  size_t const C = mesh_.n_cells;
  AvgArgs a = avg_args(mesh_, mesh_.quad);
  has_melted_kernel<<<(unsigned)((C + 127) / 128), 128, 0, stream_>>>(
      a, cell_info_d_.p, temperature, threshold, has_melted_d_.p, C);
  ADM_CK(cudaGetLastError());
  ADM_CK(cudaMemcpyAsync(has_melted_.data(), has_melted_d_.p, C, cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  if (host)
    std::memcpy(host, has_melted_.data(), C);
}

void Thermal::set_has_melted(uint8_t const *host)
{
  size_t const C = mesh_.n_cells;
  for (size_t c = 0; c < C; ++c)
    has_melted_[c] = host[c] ? 1 : 0;
  ADM_CK(cudaMemcpyAsync(has_melted_d_.p, has_melted_.data(), C, cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
}

void Thermal::activate_cells(int64_t const *cells, int64_t n, double new_temperature,
                             double const *cos_new, double const *sin_new, double *solution)
{
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  size_t const C = mesh_.n_cells;
  for (int64_t k = 0; k < n; ++k)
    if (cells[k] < 0 || (size_t)cells[k] >= C)
      throw Error(ADM_ERR_INVALID, "cell index out of range");
  ADM_CK(cudaSetDevice(device_));
  set_state_to_material_properties();
  if (n > 0)
  {
    cells_d_.alloc((size_t)n);
    ADM_CK(cudaMemcpyAsync(cells_d_.p, cells, n * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
    GridArgs g;
    for (int d = 0; d < 3; ++d)
    {
      g.nc[d] = mesh_.nc[d];
      g.nn[d] = mesh_.nn[d];
    }
    g.pitch = mesh_.pitch;
    g.deg = mesh_.deg;
    activate_nodes_kernel<<<(unsigned)n, 32, 0, stream_>>>(g, cell_info_d_.p, cells_d_.p, n,
                                                           new_temperature, solution);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaStreamSynchronize(stream_));
  }
  for (int64_t k = 0; k < n; ++k)
  {
    size_t const c = (size_t)cells[k];
    if (active_[c])
      continue;
    active_[c] = 1;
    cos_[c] = cos_new ? cos_new[k] : 1.0;
    sin_[c] = sin_new ? sin_new[k] : 0.0;
    has_melted_[c] = 1;
  }
  rebuild();
  compute_inverse_mass_matrix();
  get_state_from_material_properties();
}

int64_t Thermal::activate_in_boxes(DeviceBoxes const &boxes, int64_t b0, int64_t b1, double new_temperature,
                                   double *solution)
{
  NvtxRange const nvtx_range("adm::activate_in_boxes");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  if (b0 < 0 || b1 > boxes.n || b0 > b1)
    throw Error(ADM_ERR_INVALID, "box range out of bounds");
  if (b0 == b1)
    return 0;
  ADM_CK(cudaSetDevice(device_));
  size_t const C = mesh_.n_cells;
  if (last_box_d_.n != C)
  {
    last_box_d_.alloc(C);
    ADM_CK(cudaMemsetAsync(last_box_d_.p, 0xff, C * sizeof(int32_t), stream_)); // -1
    list_d_.alloc(C);
    list_box_d_.alloc(C);
    count_d_.alloc(1);
    matid_d_.alloc(C);
  }
  ADM_CK(cudaMemcpyAsync(matid_d_.p, matid_.data(), C, cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaMemsetAsync(count_d_.p, 0, sizeof(unsigned long long), stream_));
  BoxArgs ba;
  for (int d = 0; d < 3; ++d)
  {
    ba.nc[d] = mesh_.nc[d];
    ba.origin[d] = mesh_.origin[d];
    ba.h[d] = mesh_.h[d];
  }
  ba.lo = boxes.lo;
  ba.hi = boxes.hi;
  ba.b0 = b0;
  unsigned const nb = (unsigned)(b1 - b0);
  box_mark_kernel<<<nb, 256, 0, stream_>>>(ba, cell_info_d_.p, last_box_d_.p);
  ADM_CK(cudaGetLastError());
  box_collect_kernel<<<nb, 256, 0, stream_>>>(ba, last_box_d_.p, list_d_.p, list_box_d_.p, count_d_.p,
                                              (unsigned long long)C);
  ADM_CK(cudaGetLastError());
  unsigned long long cnt = 0;
  ADM_CK(cudaMemcpyAsync(&cnt, count_d_.p, sizeof(cnt), cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  int64_t const n = (int64_t)cnt;
  if (n == 0)
    return 0;
  std::vector<int64_t> list(n);
  std::vector<int32_t> lbox(n);
  ADM_CK(cudaMemcpyAsync(list.data(), list_d_.p, n * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaMemcpyAsync(lbox.data(), list_box_d_.p, n * sizeof(int32_t), cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  std::vector<double> cn(n), sn(n);
  bool rotation = false;
  for (int64_t k = 0; k < n; ++k)
  {
    cn[k] = boxes.cos_host[lbox[k]];
    sn[k] = boxes.sin_host[lbox[k]];
    rotation = rotation || cn[k] != 1.0 || sn[k] != 0.0;
  }
  bool const need_slots = (ns_ == 3) && !adiabatic_only_;
  if (need_slots)
  {
    // the per-face powder slots are laid out on the host: full rebuild
    ADM_CK(cudaMemsetAsync(last_box_d_.p, 0xff, C * sizeof(int32_t), stream_));
    activate_cells(list.data(), n, new_temperature, cn.data(), sn.data(), solution);
    return n;
  }
  // add_material_start: the phase state goes to the cells
  set_state_to_material_properties();
  GridArgs g;
  for (int d = 0; d < 3; ++d)
  {
    g.nc[d] = mesh_.nc[d];
    g.nn[d] = mesh_.nn[d];
  }
  g.pitch = mesh_.pitch;
  g.deg = mesh_.deg;
  g.vol = mesh_.h[0] * mesh_.h[1] * mesh_.h[2];
  for (int i = 0; i < 3; ++i)
    g.glw[i] = mesh_.glw[i];
  // new DoFs get the new-material temperature (old cell info)
  activate_nodes_kernel<<<(unsigned)n, 32, 0, stream_>>>(g, cell_info_d_.p, list_d_.p, n, new_temperature,
                                                         solution);
  ADM_CK(cudaGetLastError());
  // host bookkeeping of the activity and directions
  for (int64_t k = 0; k < n; ++k)
  {
    size_t const c = (size_t)list[k];
    active_[c] = 1;
    cos_[c] = cn[k];
    sin_[c] = sn[k];
    has_melted_[c] = 1;
  }
  bool const rotation_added = rotation && !has_rotation_;
  if (rotation_added)
  {
    cos_d_.alloc(C);
    sin_d_.alloc(C);
    ADM_CK(cudaMemcpyAsync(cos_d_.p, cos_.data(), C * sizeof(double), cudaMemcpyHostToDevice, stream_));
    ADM_CK(cudaMemcpyAsync(sin_d_.p, sin_.data(), C * sizeof(double), cudaMemcpyHostToDevice, stream_));
    has_rotation_ = true;
  }
  unsigned const blk = (unsigned)((n + 255) / 256);
  activate_list_kernel<<<blk, 256, 0, stream_>>>(list_d_.p, list_box_d_.p, n, matid_d_.p, boxes.cosv, boxes.sinv,
                                                 cell_info_d_.p, has_rotation_ ? cos_d_.p : nullptr,
                                                 has_rotation_ ? sin_d_.p : nullptr, has_melted_d_.p,
                                                 last_box_d_.p);
  ADM_CK(cudaGetLastError());
  face_bits_kernel<<<(unsigned)((7 * n + 255) / 256), 256, 0, stream_>>>(list_d_.p, n, mesh_.nc[0], mesh_.nc[1],
                                                                         mesh_.nc[2], cell_info_d_.p);
  ADM_CK(cudaGetLastError());
  inverse_mass_cells_kernel<<<(unsigned)n, 32, 0, stream_>>>(g, cell_info_d_.p, list_d_.p, n, inv_mass_.p);
  ADM_CK(cudaGetLastError());
  // tiles: activity, neighbour masks and colour work lists (host, per tile)
  std::vector<uint8_t> &ta = topo_.tile_active;
  for (int64_t k = 0; k < n; ++k)
  {
    size_t const c = (size_t)list[k];
    int const x = c % mesh_.nc[0], y = (c / mesh_.nc[0]) % mesh_.nc[1], z = c / ((size_t)mesh_.nc[0] * mesh_.nc[1]);
    ta[(x / mesh_.tx) + (size_t)mesh_.nt[0] * ((y / mesh_.ty) + (size_t)mesh_.nt[1] * (z / mesh_.tz))] = 1;
  }
  neighbour_masks(mesh_, ta, topo_.tile_nbr, topo_.all_tiles_active);
  work_.clear();
  for (int col = 0; col < 8; ++col)
  {
    colour_off_[col] = (int)work_.size();
    // top layers first: the beam works the top surface, so the slow tiles
    // (melt pool, source) are claimed early and the others balance them
    int const tz_top = mesh_.nt[2] - 1 - (((mesh_.nt[2] - 1) ^ (col >> 2)) & 1);
    for (int tz = tz_top; tz >= 0; tz -= 2)
      for (int ty = (col >> 1) & 1; ty < mesh_.nt[1]; ty += 2)
        for (int tx = col & 1; tx < mesh_.nt[0]; tx += 2)
        {
          size_t const tile = tx + (size_t)mesh_.nt[0] * (ty + (size_t)mesh_.nt[1] * tz);
          if (ta[tile])
            work_.push_back(TileWork{0, (int32_t)tile, pack_tile(tx, ty, tz)});
        }
  }
  colour_off_[8] = (int)work_.size();
  build_atomic_list(ta);
  ++work_version_;
  work_d_.ensure(std::max<size_t>(1, work_.size()));
  ADM_CK(cudaMemcpyAsync(work_d_.p, work_.data(), work_.size() * sizeof(TileWork), cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaMemcpyAsync(tile_nbr_d_.p, topo_.tile_nbr.data(), mesh_.n_tiles * sizeof(uint32_t),
                         cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaMemsetAsync(halo_d_.p, 0, halo_d_.n * sizeof(double), stream_));
  // add_material_end: the cell state goes back to the quadrature points
  get_state_from_material_properties();
  ADM_CK(cudaStreamSynchronize(stream_));
  if (step_graph_)
  {
    cudaGraphExecDestroy(step_graph_);
    step_graph_ = nullptr;
  }
  if (rotation_added)
    upload_member();
  return n;
}

void Thermal::update_beam(int i, adm_source const &beam)
{
  if (i < 0 || i >= cfg_.n_sources)
    throw Error(ADM_ERR_INVALID, "source index out of range");
  adm_source &s = cfg_.sources[i];
  s.depth = beam.depth;
  s.absorption_efficiency = beam.absorption_efficiency;
  s.radius_squared = beam.radius_squared;
  s.max_power = beam.max_power;
  upload_member();
}

void Thermal::update_material(adm_config const &cfg)
{
  if (cfg.n_materials != cfg_.n_materials || cfg.n_states != cfg_.n_states ||
      cfg.use_table != cfg_.use_table)
    throw Error(ADM_ERR_INVALID, "update_material: the number of materials and states and the "
                                 "table/polynomial choice must not change");
  if (cfg.p_order < 0 || cfg.p_order > 4)
    throw Error(ADM_ERR_INVALID, "p_order must be in [0, 4]");
  ADM_CK(cudaSetDevice(device_));
  cfg_.p_order = cfg.p_order;
  std::memcpy(cfg_.poly, cfg.poly, sizeof(cfg_.poly));
  std::memcpy(cfg_.table, cfg.table, sizeof(cfg_.table));
  std::memcpy(cfg_.props, cfg.props, sizeof(cfg_.props));
  MaterialDesc const m = make_material(cfg_);
  ADM_CK(cudaMemcpyAsync(mat_d_.p, &m, sizeof(m), cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  int pmax = 0;
  for (int p : {(int)P_DENSITY, (int)P_SPECIFIC_HEAT, (int)P_KX, (int)P_KY, (int)P_KZ})
    pmax = std::max(pmax, m.prop_deg[p]);
  int const p_new = pmax <= 2 ? 2 : 4;
  if (p_new != poly_p_ && step_graph_)
  {
    cudaGraphExecDestroy(step_graph_);
    step_graph_ = nullptr;
  }
  poly_p_ = p_new;
}

int32_t Thermal::device_error()
{
  int32_t e = 0;
  ADM_CK(cudaMemcpyAsync(&e, error_d_.p, sizeof(e), cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  return e;
}

void Thermal::synchronize() { ADM_CK(cudaStreamSynchronize(stream_)); }

// The atomic schedule's list: every active tile, colour by colour, bottom
// layers first (measured faster for the one strided launch than the top-down
// order of the colour lists, which suits the claimed colour launches).
void Thermal::build_atomic_list(std::vector<uint8_t> const &tile_active)
{
  awork_.clear();
  for (int col = 0; col < 8; ++col)
    for (int tz = (col >> 2) & 1; tz < mesh_.nt[2]; tz += 2)
      for (int ty = (col >> 1) & 1; ty < mesh_.nt[1]; ty += 2)
        for (int tx = col & 1; tx < mesh_.nt[0]; tx += 2)
        {
          size_t const tile = tx + (size_t)mesh_.nt[0] * (ty + (size_t)mesh_.nt[1] * tz);
          if (tile_active[tile])
            awork_.push_back(TileWork{0, (int32_t)tile, pack_tile(tx, ty, tz)});
        }
  awork_d_.ensure(std::max<size_t>(1, awork_.size()));
  if (!awork_.empty())
    ADM_CK(cudaMemcpyAsync(awork_d_.p, awork_.data(), awork_.size() * sizeof(TileWork), cudaMemcpyHostToDevice,
                           stream_));
}

void Thermal::set_cells_per_block(int n)
{
  int const tile = mesh_.tx * mesh_.ty * mesh_.tz;
  if (n != tile && !(mesh_.deg == 2 && n == 2 * tile))
    throw Error(ADM_ERR_INVALID, "cells per block: the tile's (64 for FE_Q(2), 128 for FE_Q(1)) or, for FE_Q(2), "
                                 "128 (z-pairs of tiles)");
  int const v = n == tile ? 0 : n;
  if (v != cells_per_block_ && step_graph_)
  {
    cudaGraphExecDestroy(step_graph_);
    step_graph_ = nullptr;
  }
  cells_per_block_ = v;
}

// The z-pairs (tiles at layers 2p and 2p + 1) that hold an active tile, for
// the 128-cell blocks of the atomic schedule: x fastest, bottom pairs first
// (the order of the atomic schedule's tile list).
void Thermal::build_pair_list()
{
  if (pwork_version_ == work_version_ && !pwork_.empty())
    return;
  pwork_.clear();
  int const nt0 = mesh_.nt[0], nt1 = mesh_.nt[1], nt2 = mesh_.nt[2];
  std::vector<uint8_t> const &ta = topo_.tile_active;
  for (int p = 0; 2 * p < nt2; ++p)
    for (int ty = 0; ty < nt1; ++ty)
      for (int tx = 0; tx < nt0; ++tx)
      {
        size_t const t0 = tx + (size_t)nt0 * (ty + (size_t)nt1 * (2 * p));
        size_t const t1 = t0 + (size_t)nt0 * nt1;
        if (!ta[t0] && !(2 * p + 1 < nt2 && ta[t1]))
          continue;
        TileWork w;
        w.member = 0;
        w.tile = (int32_t)t0;
        w.xyz = pack_tile(tx, ty, p);
        pwork_.push_back(w);
      }
  pwork_d_.ensure(std::max<size_t>(1, pwork_.size()));
  if (!pwork_.empty())
    ADM_CK(cudaMemcpyAsync(pwork_d_.p, pwork_.data(), pwork_.size() * sizeof(TileWork), cudaMemcpyHostToDevice,
                           stream_));
  pwork_version_ = work_version_;
}

void Thermal::set_cells_per_thread(int n)
{
  if (n != 1 && n != 2 && n != 4)
    throw Error(ADM_ERR_INVALID, "cells per thread must be 1, 2 or 4");
  if (n != 1 && mesh_.deg != 1)
    throw Error(ADM_ERR_UNSUPPORTED, "two or four cells per thread are variants of the FE_Q(1) kernel");
  if (n != cells_per_thread_ && step_graph_)
  {
    cudaGraphExecDestroy(step_graph_);
    step_graph_ = nullptr;
  }
  cells_per_thread_ = n;
}

void Thermal::set_schedule(int schedule)
{
  if (schedule != kScheduleColoured && schedule != kScheduleAtomic && schedule != kScheduleTwoPass)
    throw Error(ADM_ERR_INVALID, "unknown schedule");
  if (schedule != schedule_ && step_graph_)
  {
    cudaGraphExecDestroy(step_graph_);
    step_graph_ = nullptr;
  }
  schedule_ = schedule;
}

Thermal::PhaseSnapshot Thermal::save_phase() const
{
  PhaseSnapshot p;
  size_t const C = mesh_.n_cells;
  int const NN = (mesh_.deg + 1) * (mesh_.deg + 1) * (mesh_.deg + 1);
  if (ns_ == 3)
  {
    p.mode.alloc(C);
    p.cell.alloc(C);
    p.q.alloc(C * NN);
    ADM_CK(cudaMemcpyAsync(p.mode.p, powder_mode_.p, C, cudaMemcpyDeviceToDevice, stream_));
    ADM_CK(cudaMemcpyAsync(p.cell.p, powder_cell_.p, C * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    ADM_CK(cudaMemcpyAsync(p.q.p, powder_q_.p, C * NN * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    if (face_powder_.p)
    {
      p.face.alloc(face_powder_.n);
      ADM_CK(cudaMemcpyAsync(p.face.p, face_powder_.p, face_powder_.n * sizeof(double), cudaMemcpyDeviceToDevice,
                             stream_));
    }
  }
  if (ns_ > 1)
  {
    p.liquid.alloc(C);
    ADM_CK(cudaMemcpyAsync(p.liquid.p, liquid_sum_.p, C * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
  }
  p.clock.alloc(2);
  ADM_CK(cudaMemcpyAsync(p.clock.p, clock_.p, 2 * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
  return p;
}

void Thermal::restore_phase(PhaseSnapshot const &p)
{
  if (p.mode.p)
  {
    ADM_CK(cudaMemcpyAsync(powder_mode_.p, p.mode.p, p.mode.n, cudaMemcpyDeviceToDevice, stream_));
    ADM_CK(cudaMemcpyAsync(powder_cell_.p, p.cell.p, p.cell.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    ADM_CK(cudaMemcpyAsync(powder_q_.p, p.q.p, p.q.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
  }
  if (p.face.p)
    ADM_CK(cudaMemcpyAsync(face_powder_.p, p.face.p, p.face.n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
  if (p.liquid.p)
    ADM_CK(cudaMemcpyAsync(liquid_sum_.p, p.liquid.p, p.liquid.n * sizeof(double), cudaMemcpyDeviceToDevice,
                           stream_));
  ADM_CK(cudaMemcpyAsync(clock_.p, p.clock.p, 2 * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
}

// Times the schedules on the handle's problem (vmults of `field`, the phase
// history saved before and restored after) and keeps the fastest.
int Thermal::autotune(double const *field, double *ms_out)
{
  NvtxRange const nvtx_range("adm::autotune");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  ADM_CK(cudaSetDevice(device_));
  PhaseSnapshot const snap = save_phase();
  DevBuf<double> dst;
  dst.alloc(mesh_.n_nodes);
  cudaEvent_t e0, e1;
  ADM_CK(cudaEventCreate(&e0));
  ADM_CK(cudaEventCreate(&e1));
  int const saved = schedule_, saved_cz = cells_per_thread_, saved_cpb = cells_per_block_;
  double best = 0.0;
  int choice = saved, choice_cz = saved_cz, choice_cpb = saved_cpb;
  // launch schedules x kernel variants (FE_Q(1): cells per thread; FE_Q(2),
  // atomic schedule: 64- or 128-cell blocks); ms_out[schedule] is the
  // schedule's best time. An untimed round over every variant first: the
  // first launches of each kernel and the clock ramp of an idle GPU would
  // otherwise fall on the first variant timed.
  struct Variant
  {
    int sch, cz, cpb;
  };
  std::vector<Variant> variants;
  for (int sch : {kScheduleColoured, kScheduleAtomic, kScheduleTwoPass})
  {
    if (mesh_.deg == 1)
      for (int cz : {1, 2, 4})
        variants.push_back({sch, cz, 0});
    else
    {
      variants.push_back({sch, 1, 0});
      if (sch == kScheduleAtomic)
        variants.push_back({sch, 1, 128});
    }
  }
  auto select = [&](Variant const &v) {
    schedule_ = v.sch;
    cells_per_thread_ = v.cz;
    cells_per_block_ = v.cpb;
  };
  for (Variant const &v : variants)
  {
    select(v);
    for (int r = 0; r < 2; ++r)
      vmult(dst.p, field, false);
  }
  bool first_of[3] = {true, true, true}; // per schedule
  for (Variant const &v : variants)
  {
    select(v);
    for (int r = 0; r < 2; ++r)
      vmult(dst.p, field, false);
    ADM_CK(cudaEventRecord(e0, stream_));
    int const reps = 5;
    for (int r = 0; r < reps; ++r)
      vmult(dst.p, field, false);
    ADM_CK(cudaEventRecord(e1, stream_));
    ADM_CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    ADM_CK(cudaEventElapsedTime(&ms, e0, e1));
    double const per = ms / reps;
    if (ms_out && (first_of[v.sch] || per < ms_out[v.sch]))
      ms_out[v.sch] = per;
    first_of[v.sch] = false;
    if (best == 0.0 || per < best)
    {
      best = per;
      choice = v.sch;
      choice_cz = v.cz;
      choice_cpb = v.cpb;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  schedule_ = saved;
  cells_per_thread_ = saved_cz;
  cells_per_block_ = saved_cpb;
  restore_phase(snap);
  ADM_CK(cudaStreamSynchronize(stream_));
  set_schedule(choice);
  set_cells_per_thread(choice_cz);
  set_cells_per_block(choice_cpb == 0 ? mesh_.tx * mesh_.ty * mesh_.tz : choice_cpb);
  return choice;
}

void Thermal::bind_stage_vectors(double *za, double *zb, double *s, double *f0, double *acc)
{
  za_p_ = za;
  zb_p_ = zb;
  s_p_ = s;
  f0_p_ = f0;
  acc_p_ = acc;
  if (step_graph_)
  {
    cudaGraphExecDestroy(step_graph_);
    step_graph_ = nullptr;
  }
  upload_member();
}

namespace
{
bool is_pinned(void const *p)
{
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess)
  {
    (void)cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}
} // namespace

void Thermal::vmult_host(double *dst_host, double const *src_host)
{
  NvtxRange const nvtx_range("adm::vmult_host");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  ADM_CK(cudaSetDevice(device_));
  size_t const n = mesh_.n_nodes;
  stage_in_.alloc(n);
  stage_out_.alloc(n);
  int const nt2 = mesh_.nt[2];
  if (nt2 < 2 || colour_off_[8] == 0 || !is_pinned(src_host) || !is_pinned(dst_host))
  {
    ADM_CK(cudaMemcpyAsync(stage_in_.p, src_host, n * sizeof(double), cudaMemcpyHostToDevice, stream_));
    vmult(stage_out_.p, stage_in_.p, false);
    ADM_CK(cudaMemcpyAsync(dst_host, stage_out_.p, n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    ADM_CK(cudaStreamSynchronize(stream_));
    return;
  }
  // Pinned host buffers: the vector moves in z-slabs on two copy streams and
  // the tiles of each slab run (atomic schedule) as soon as their nodes have
  // arrived, so the host-to-device copy, the kernel and the device-to-host
  // copy of earlier slabs overlap.
  if (zwork_version_ != work_version_ || zwork_.empty())
  {
    zwork_.assign(work_.begin(), work_.end());
    int const per_layer = mesh_.nt[0] * mesh_.nt[1];
    std::stable_sort(zwork_.begin(), zwork_.end(),
                     [&](TileWork const &a, TileWork const &b) { return a.tile / per_layer < b.tile / per_layer; });
    zwork_d_.alloc(zwork_.size());
    ADM_CK(cudaMemcpyAsync(zwork_d_.p, zwork_.data(), zwork_.size() * sizeof(TileWork), cudaMemcpyHostToDevice,
                           stream_));
    zwork_version_ = work_version_;
  }
  if (!copy_in_)
  {
    ADM_CK(cudaStreamCreateWithFlags(&copy_in_, cudaStreamNonBlocking));
    ADM_CK(cudaStreamCreateWithFlags(&copy_out_, cudaStreamNonBlocking));
    for (auto &e : pipe_ev_)
      ADM_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  }
  int const chunks = std::min(kPipeChunks, nt2);
  int const per_layer = mesh_.nt[0] * mesh_.nt[1];
  size_t const row = (size_t)mesh_.pitch * mesh_.nn[1]; // doubles per node z-row
  int const rows_per_layer = mesh_.deg * mesh_.tz;
  int const nrows = mesh_.nn[2];
  cudaEvent_t const start = pipe_ev_[2 * kPipeChunks], done = pipe_ev_[2 * kPipeChunks + 1];
  ADM_CK(cudaEventRecord(start, stream_));
  ADM_CK(cudaStreamWaitEvent(copy_in_, start, 0));
  ADM_CK(cudaStreamWaitEvent(copy_out_, start, 0));
  ADM_CK(cudaMemsetAsync(stage_out_.p, 0, n * sizeof(double), stream_));
  prepare_stage(0.0);
  KernelArgs a = base_args();
  a.mode = 0;
  a.atomic = 1;
  a.vsrc = stage_in_.p;
  a.vdst = stage_out_.p;
  CUtensorMap const map = brick_map(mesh_, stage_in_.p, 1, n);
  int rows_in = 0, rows_out = 0;
  size_t item = 0;
  for (int c = 0; c < chunks; ++c)
  {
    int const tz1 = (int)((int64_t)(c + 1) * nt2 / chunks);
    // node rows the tiles of layers < tz1 read, and the rows that are final
    int const need = std::min(nrows, rows_per_layer * tz1 + 1);
    int const final_rows = c == chunks - 1 ? nrows : rows_per_layer * tz1;
    cudaEvent_t const e_in = pipe_ev_[2 * c], e_k = pipe_ev_[2 * c + 1];
    if (need > rows_in)
      ADM_CK(cudaMemcpyAsync(stage_in_.p + rows_in * row, src_host + rows_in * row, (need - rows_in) * row * sizeof(double),
                             cudaMemcpyHostToDevice, copy_in_));
    rows_in = std::max(rows_in, need);
    ADM_CK(cudaEventRecord(e_in, copy_in_));
    ADM_CK(cudaStreamWaitEvent(stream_, e_in, 0));
    size_t end = item;
    while (end < zwork_.size() && zwork_[end].tile / per_layer < tz1)
      ++end;
    if (end > item)
    {
      a.work = zwork_d_.p + item;
      launch_tile(mesh_.deg, ns_, poly_p_, map, a, (int)(end - item), stream_);
      ADM_CK(cudaGetLastError());
    }
    item = end;
    ADM_CK(cudaEventRecord(e_k, stream_));
    ADM_CK(cudaStreamWaitEvent(copy_out_, e_k, 0));
    if (final_rows > rows_out)
      ADM_CK(cudaMemcpyAsync(dst_host + rows_out * row, stage_out_.p + rows_out * row,
                             (final_rows - rows_out) * row * sizeof(double), cudaMemcpyDeviceToHost, copy_out_));
    rows_out = std::max(rows_out, final_rows);
  }
  ADM_CK(cudaEventRecord(done, copy_out_));
  ADM_CK(cudaStreamWaitEvent(stream_, done, 0));
  ADM_CK(cudaStreamSynchronize(stream_));
}

double Thermal::evolve_one_time_step_host(double t, double dt, double *solution_host)
{
  size_t const n = mesh_.n_nodes;
  stage_in_.alloc(n);
  ADM_CK(cudaMemcpyAsync(stage_in_.p, solution_host, n * sizeof(double), cudaMemcpyHostToDevice, stream_));
  double const tn = evolve_one_time_step(t, dt, stage_in_.p);
  ADM_CK(cudaMemcpyAsync(solution_host, stage_in_.p, n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  return tn;
}

} // namespace adm
