// Microstructure data of the temperature field (Microstructure::
// set_old_temperature and compute_G_and_R, source/Microstructure.hh:41-207,
// Microstructure.cc:57-63).
//
// A node scan lists the nodes that crossed some material's liquidus
// downward during the step; then one thread per (listed node, cell around
// it) checks the cell (active, its material's liquidus) and evaluates the
// gradient of the cell's interpolant of the new field at that node with the
// nodal derivative
// matrix of the 1D Lagrange basis (the Gauss-Lobatto points of
// QGaussLobatto(p + 1) are the support points), G = |grad T|, the cooling
// rate as the reference computes it (old - new / delta_t, the division
// binding to the new value only) and R = rate / G, and appends the record
// with its (cell, point) key to a device list. The host sorts the few
// records by key, which is the reference's output order (cells in
// triangulation order, points lexicographic). A node shared by several
// cells gives one record per cell with that cell's one-sided gradient, as in
// the reference. Sums are evaluated left to right with each product rounded
// (no fused multiply-add), so the records equal the oracle's bit for bit.
#include "capi_common.hpp"
#include "../../include/adamantine_b200_microstructure.h"

#include <algorithm>
#include <numeric>
#include <vector>

namespace adm
{
namespace
{
struct GrGeom
{
  int deg;
  int nc[3];
  int nn1, pitch;
  double h[3], origin[3];
  double pt[3];      // support points of the 1D basis on [0, 1]
  double D[3][3];    // D[a][i] = phi_i'(pt[a])
};

// Pass 1, one thread per node (coalesced): the nodes whose old value is
// above and new value at or below the liquidus of some material go to a
// compact list (the few nodes the step solidified).
__global__ void gr_scan_kernel(GrGeom g, int nn0, size_t n_nodes, int n_mat, MaterialDesc const *mat,
                               double const *t_old, double const *t_new, int64_t *list, unsigned long long *count,
                               unsigned long long cap)
{
  size_t const i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= n_nodes || (int)(i % g.pitch) >= nn0)
    return;
  double const to = t_old[i], tn = t_new[i];
  bool hit = false;
  for (int m = 0; m < n_mat; ++m)
  {
    double const liq = mat->props[m][Q_LIQUIDUS];
    hit |= to > liq && tn <= liq;
  }
  if (!hit)
    return;
  unsigned long long const slot = atomicAdd(count, 1ull);
  if (slot < cap)
    list[slot] = (int64_t)i;
}

// Pass 2, one thread per (listed node, cell that may hold it): the up to
// eight cells around the node (one per axis where the node is inside a
// cell), each with its own material's liquidus; the crossing records of the
// reference with the key (cell, point).
__global__ void gr_kernel(GrGeom g, uint32_t const *cell_info, MaterialDesc const *mat, double const *t_old,
                          double const *t_new, double dt, int64_t const *list, size_t n_list, double *rec,
                          int64_t *key, unsigned long long *count, unsigned long long cap)
{
  int const n = g.deg + 1, nq = n * n * n;
  size_t const idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (idx >= n_list * 8)
    return;
  size_t const node = (size_t)list[idx / 8];
  int const combo = (int)(idx % 8);
  int const nidx[3] = {(int)(node % g.pitch), (int)((node / g.pitch) % g.nn1),
                       (int)(node / ((size_t)g.pitch * g.nn1))};
  int cell[3], loc[3];
  for (int d = 0; d < 3; ++d)
  {
    int const lower = (combo >> d) & 1; // 1: the cell below the node along d
    int cd = nidx[d] / g.deg;
    if (lower)
    {
      if (nidx[d] % g.deg != 0)
        return; // inside a cell along d: only one cell holds the node
      cd -= 1;
    }
    if (cd < 0 || cd >= g.nc[d])
      return;
    cell[d] = cd;
    loc[d] = nidx[d] - g.deg * cd;
  }
  size_t const c = cell[0] + (size_t)g.nc[0] * (cell[1] + (size_t)g.nc[1] * cell[2]);
  uint32_t const info = cell_info[c];
  if (!(info & CI_ACTIVE))
    return;
  double const liq = mat->props[(info >> CI_MAT_SHIFT) & 15][Q_LIQUIDUS];
  double const to = t_old[node], tn = t_new[node];
  if (!(to > liq && tn <= liq))
    return;
  int const q = loc[0] + n * (loc[1] + n * loc[2]);
  size_t const stride[3] = {1, (size_t)g.pitch, (size_t)g.pitch * g.nn1};
  double G2 = 0.0;
  for (int d = 0; d < 3; ++d)
  {
    size_t const first = node - (size_t)loc[d] * stride[d];
    double s = 0.0;
    for (int i = 0; i < n; ++i)
      s = __dadd_rn(s, __dmul_rn(g.D[loc[d]][i], t_new[first + i * stride[d]]));
    double const gd = s / g.h[d];
    G2 = __dadd_rn(G2, __dmul_rn(gd, gd));
  }
  double const G = sqrt(G2);
  double const rate = to - tn / dt;
  unsigned long long const slot = atomicAdd(count, 1ull);
  if (slot >= cap)
    return;
  double *r = rec + 6 * slot;
  for (int d = 0; d < 3; ++d)
    r[d] = __dadd_rn(__dadd_rn(g.origin[d], __dmul_rn((double)cell[d], g.h[d])), __dmul_rn(g.pt[loc[d]], g.h[d]));
  r[3] = G;
  r[4] = rate;
  r[5] = rate / G;
  key[slot] = (int64_t)(c * nq + q);
}
} // namespace

class Microstructure
{
public:
  explicit Microstructure(Thermal &t) : th_(t) {}

  void set_old_temperature(double const *old_t)
  {
    if (!th_.setup_done_)
      throw Error(ADM_ERR_INVALID, "setup() has not been called");
    ADM_CK(cudaSetDevice(th_.device_));
    size_t const n = th_.mesh_.n_nodes;
    old_.alloc(n);
    ADM_CK(cudaMemcpyAsync(old_.p, old_t, n * sizeof(double), cudaMemcpyDeviceToDevice, th_.stream_));
    has_old_ = true;
  }

  int64_t compute(double const *t_new, double dt, int64_t capacity, double *out)
  {
    NvtxRange const nvtx_range("adm::microstructure_G_R");
    if (!has_old_)
      throw Error(ADM_ERR_INVALID, "set_old_temperature() has not been called");
    Thermal &t = th_;
    Mesh const &m = t.mesh_;
    ADM_CK(cudaSetDevice(t.device_));
    cudaStream_t const st = t.stream_;
    GrGeom g{};
    g.deg = m.deg;
    for (int d = 0; d < 3; ++d)
    {
      g.nc[d] = m.nc[d];
      g.h[d] = m.h[d];
      g.origin[d] = m.origin[d];
    }
    g.nn1 = m.nn[1];
    g.pitch = m.pitch;
    // Lagrange basis on {0, 1} or {0, 1/2, 1}: exact derivative values
    if (m.deg == 1)
    {
      double const pt[2] = {0.0, 1.0};
      double const D[2][2] = {{-1.0, 1.0}, {-1.0, 1.0}};
      for (int a = 0; a < 2; ++a)
      {
        g.pt[a] = pt[a];
        for (int i = 0; i < 2; ++i)
          g.D[a][i] = D[a][i];
      }
    }
    else
    {
      double const pt[3] = {0.0, 0.5, 1.0};
      double const D[3][3] = {{-3.0, 4.0, -1.0}, {-1.0, 0.0, 1.0}, {1.0, -4.0, 3.0}};
      for (int a = 0; a < 3; ++a)
      {
        g.pt[a] = pt[a];
        for (int i = 0; i < 3; ++i)
          g.D[a][i] = D[a][i];
      }
    }
    count_.alloc(1);
    // pass 1: the crossing nodes (the list grows and the scan reruns when
    // it overflows)
    unsigned long long n_nodes_hit = 0;
    int const n_mat = t.cfg_.n_materials;
    for (int pass = 0; pass < 2; ++pass)
    {
      ADM_CK(cudaMemsetAsync(count_.p, 0, sizeof(unsigned long long), st));
      gr_scan_kernel<<<(unsigned)((m.n_nodes + 255) / 256), 256, 0, st>>>(g, m.nn[0], m.n_nodes, n_mat, t.mat_d_.p,
                                                                          old_.p, t_new, list_.p, count_.p,
                                                                          list_cap_);
      ADM_CK(cudaGetLastError());
      ADM_CK(cudaMemcpyAsync(&n_nodes_hit, count_.p, sizeof(n_nodes_hit), cudaMemcpyDeviceToHost, st));
      ADM_CK(cudaStreamSynchronize(st));
      if (n_nodes_hit <= list_cap_)
        break;
      list_cap_ = std::max<unsigned long long>(n_nodes_hit, 2 * list_cap_);
      list_.alloc(list_cap_);
    }
    // pass 2: the records of the cells around those nodes
    unsigned long long n_rec = 0;
    for (int pass = 0; pass < 2 && n_nodes_hit > 0; ++pass)
    {
      ADM_CK(cudaMemsetAsync(count_.p, 0, sizeof(unsigned long long), st));
      size_t const threads = 8 * (size_t)n_nodes_hit;
      gr_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, st>>>(g, t.cell_info_d_.p, t.mat_d_.p, old_.p, t_new,
                                                                   dt, list_.p, n_nodes_hit, rec_.p, key_.p,
                                                                   count_.p, cap_);
      ADM_CK(cudaGetLastError());
      ADM_CK(cudaMemcpyAsync(&n_rec, count_.p, sizeof(n_rec), cudaMemcpyDeviceToHost, st));
      ADM_CK(cudaStreamSynchronize(st));
      if (n_rec <= cap_)
        break;
      // more records than the list holds: grow it and run again
      cap_ = std::max<unsigned long long>(n_rec, 2 * cap_);
      rec_.alloc(6 * cap_);
      key_.alloc(cap_);
    }
    if (out && capacity >= (int64_t)n_rec && n_rec > 0)
    {
      std::vector<double> rec(6 * n_rec);
      std::vector<int64_t> key(n_rec);
      ADM_CK(cudaMemcpyAsync(rec.data(), rec_.p, rec.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
      ADM_CK(cudaMemcpyAsync(key.data(), key_.p, key.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st));
      ADM_CK(cudaStreamSynchronize(st));
      std::vector<size_t> order(n_rec);
      std::iota(order.begin(), order.end(), 0);
      std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return key[a] < key[b]; });
      for (size_t r = 0; r < n_rec; ++r)
        std::copy(rec.begin() + 6 * order[r], rec.begin() + 6 * order[r] + 6, out + 6 * r);
    }
    return (int64_t)n_rec;
  }

private:
  Thermal &th_;
  DevBuf<double> old_, rec_;
  DevBuf<int64_t> key_, list_;
  DevBuf<unsigned long long> count_;
  unsigned long long cap_ = 0, list_cap_ = 0;
  bool has_old_ = false;
};

} // namespace adm

extern "C" {

int adm_microstructure_create(adm_thermal *h, adm_microstructure **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && out, "null argument");
    *out = reinterpret_cast<adm_microstructure *>(new adm::Microstructure(*reinterpret_cast<adm::Thermal *>(h)));
  });
}

int adm_microstructure_destroy(adm_microstructure *m)
{
  return adm::guard([&] { delete reinterpret_cast<adm::Microstructure *>(m); });
}

int adm_microstructure_set_old_temperature(adm_microstructure *m, double const *old_temperature)
{
  return adm::guard([&] {
    ADM_REQUIRE(m && old_temperature, "null argument");
    reinterpret_cast<adm::Microstructure *>(m)->set_old_temperature(old_temperature);
  });
}

int adm_microstructure_compute_G_and_R(adm_microstructure *m, double const *temperature, double delta_t,
                                       int64_t capacity, double *records, int64_t *n_records)
{
  return adm::guard([&] {
    ADM_REQUIRE(m && temperature && n_records, "null argument");
    ADM_REQUIRE(capacity >= 0, "negative capacity");
    *n_records = reinterpret_cast<adm::Microstructure *>(m)->compute(temperature, delta_t, capacity, records);
  });
}

} // extern "C"
