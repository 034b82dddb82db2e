/* Refined meshes for the thermal path: a forest of octrees over the coarse
 * box mesh, refined along the beams' paths and balanced 2:1 across faces and
 * edges, with hanging-node constraints.
 *
 * Reference behaviour followed:
 *  - compute_cells_to_refine (application/adamantine.hh:540-606): the active
 *    cells whose bounding box meets a beam's box (scaled by 2) at any of
 *    n_time_steps sample times in [time, next_refinement_time);
 *    HeatSource::get_bounding_box (GoldakHeatSource.cc:152-190,
 *    ElectronBeamHeatSource.cc:162-200, CubeHeatSource.cc:111-123);
 *  - refine_mesh (application/adamantine.hh:608-681): n_refinements rounds of
 *    {coarsen flags on every cell above level 0 when coarsen_after_beam,
 *    cleared on the cells to refine; refine flags on the cells to refine
 *    below level n_refinements; execute};
 *  - make_hanging_node_constraints (application/adamantine.hh:514-523): the
 *    value at a node of a fine cell lying inside a face or edge of a coarser
 *    active neighbour, and not one of its nodes, is the coarse cell's
 *    interpolant there;
 *  - ThermalOperator::vmult_add with constraints (ThermalOperator.templates.hh
 *    :205-224: read through the constraints, distribute the result back) and
 *    compute_inverse_mass_matrix (:140-160);
 *  - refine_and_transfer (application/adamantine.hh:312-539): the solution is
 *    interpolated onto the new mesh (SolutionTransfer: the old finite-element
 *    field evaluated at the new nodes) and the cell data carried over
 *    (CellDataTransfer: children copy their parent; a coarsened parent takes
 *    its first child's data).
 *
 * B200 layout: one structured level grid per refinement level (the coarse box
 * refined 2^l times), with the tile kernel of the uniform path run on the
 * tiles that hold leaves of that level (its active cells); faces towards
 * cells of the material region are interior on every level. The composite
 * vector holds the non-hanging nodes; one gather kernel prolongs it to the
 * level grids (constraints resolved, C y) and one gather kernel restricts the
 * level results back (C^T), both from host-built CSR tables, deterministic
 * (no atomics).
 *
 * Lattice: every node of a level-l cell lies on the vertex lattice of level
 * max_level + 1 (degree 1 and 2 nodes are vertices and midpoints), so a node
 * is keyed by its integer lattice coordinates and coincident nodes of
 * different levels share a key.
 */
#include "capi_common.hpp"
#include "thermal.hpp"
#include "../../include/adamantine_b200_amr.h"

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <unordered_map>
#include <vector>

namespace adm
{
constexpr int kRemeshPhases = ADM_AMR_REMESH_PHASES;
namespace
{

// face (6) and edge (12) neighbour offsets
struct Offsets
{
  int o[18][3];
  int n = 0;
  Offsets()
  {
    for (int z = -1; z <= 1; ++z)
      for (int y = -1; y <= 1; ++y)
        for (int x = -1; x <= 1; ++x)
        {
          int const nz = (x != 0) + (y != 0) + (z != 0);
          if (nz == 1 || nz == 2)
          {
            o[n][0] = x;
            o[n][1] = y;
            o[n][2] = z;
            ++n;
          }
        }
  }
};
Offsets const kFaceEdge;

// 1-D Lagrange basis of degree p on the equidistant (= Gauss-Lobatto for
// p <= 2) nodes a / p, at u in [0, 1].
double lagrange(int p, int a, double u)
{
  double v = 1.0;
  for (int b = 0; b <= p; ++b)
    if (b != a)
      v *= (u * p - b) / (double)(a - b);
  return v;
}

} // namespace

// ---------------------------------------------------------------- forest
struct Forest
{
  int nc[3] = {0, 0, 0};
  int max_level = 0;
  std::vector<std::vector<uint8_t>> leaf, exists;

  int64_t n(int l, int d) const { return (int64_t)nc[d] << l; }
  int64_t cells(int l) const { return n(l, 0) * n(l, 1) * n(l, 2); }
  int64_t index(int l, int64_t i, int64_t j, int64_t k) const { return i + n(l, 0) * (j + n(l, 1) * k); }
  bool inside(int l, int64_t i, int64_t j, int64_t k) const
  {
    return i >= 0 && j >= 0 && k >= 0 && i < n(l, 0) && j < n(l, 1) && k < n(l, 2);
  }

  void init(int const c[3], int L)
  {
    std::copy(c, c + 3, nc);
    max_level = L;
    leaf.assign(L + 1, {});
    exists.assign(L + 1, {});
    for (int l = 0; l <= L; ++l)
    {
      leaf[l].assign(cells(l), 0);
      exists[l].assign(cells(l), 0);
    }
    std::fill(leaf[0].begin(), leaf[0].end(), 1);
    std::fill(exists[0].begin(), exists[0].end(), 1);
  }

  // m <= l: the region of cell (l, i, j, k) lies in the leaf of level m;
  // l + 1: that cell exists and is refined.
  int status(int l, int64_t i, int64_t j, int64_t k) const
  {
    for (int m = l; m >= 0; --m)
    {
      int const s = l - m;
      int64_t const c = index(m, i >> s, j >> s, k >> s);
      if (exists[m][c])
        return leaf[m][c] ? m : m + 1;
    }
    return 0;
  }

  void refine(int l, int64_t i, int64_t j, int64_t k)
  {
    int64_t const c = index(l, i, j, k);
    leaf[l][c] = 0;
    for (int q = 0; q < 8; ++q)
    {
      int64_t const cc = index(l + 1, 2 * i + (q & 1), 2 * j + ((q >> 1) & 1), 2 * k + (q >> 2));
      exists[l + 1][cc] = 1;
      leaf[l + 1][cc] = 1;
    }
  }

  void coarsen(int l, int64_t i, int64_t j, int64_t k)
  {
    for (int q = 0; q < 8; ++q)
    {
      int64_t const cc = index(l + 1, 2 * i + (q & 1), 2 * j + ((q >> 1) & 1), 2 * k + (q >> 2));
      exists[l + 1][cc] = 0;
      leaf[l + 1][cc] = 0;
    }
    leaf[l][index(l, i, j, k)] = 1;
  }

  // Leaves no more than one level apart across every face and edge: a leaf
  // of level l whose face/edge neighbour region lies in a leaf of level
  // m < l - 1 refines that leaf (repeated until nothing changes).
  void balance()
  {
    bool changed = true;
    while (changed)
    {
      changed = false;
      for (int l = max_level; l >= 2; --l)
        for (int64_t k = 0; k < n(l, 2); ++k)
          for (int64_t j = 0; j < n(l, 1); ++j)
          {
            uint8_t const *lf = &leaf[l][index(l, 0, j, k)];
            for (int64_t i = 0; i < n(l, 0); ++i)
            {
              if (!lf[i])
                continue;
              for (int o = 0; o < kFaceEdge.n; ++o)
              {
                int64_t const a = i + kFaceEdge.o[o][0], b = j + kFaceEdge.o[o][1], c = k + kFaceEdge.o[o][2];
                if (!inside(l, a, b, c))
                  continue;
                int const m = status(l, a, b, c);
                if (m < l - 1)
                {
                  int const s = l - m;
                  refine(m, a >> s, b >> s, c >> s);
                  changed = true;
                }
              }
            }
          }
    }
  }

  // Coarsening the family of parent (l, i, j, k) keeps the balance: no
  // face/edge neighbour of its children is refined below level l + 1.
  bool coarsening_keeps_balance(int l, int64_t i, int64_t j, int64_t k) const
  {
    for (int q = 0; q < 8; ++q)
    {
      int64_t const ci = 2 * i + (q & 1), cj = 2 * j + ((q >> 1) & 1), ck = 2 * k + (q >> 2);
      for (int o = 0; o < kFaceEdge.n; ++o)
      {
        int64_t const a = ci + kFaceEdge.o[o][0], b = cj + kFaceEdge.o[o][1], c = ck + kFaceEdge.o[o][2];
        if (!inside(l + 1, a, b, c) || ((a >> 1) == i && (b >> 1) == j && (c >> 1) == k))
          continue;
        if (status(l + 1, a, b, c) > l + 1)
          return false;
      }
    }
    return true;
  }
};

// ------------------------------------------------------------------ mesh
// DoFs, hanging-node constraints and the level-grid maps of a forest.
struct AmrMesh
{
  adm_config cfg{};
  std::vector<std::vector<double>> segments; // per source, 5 doubles per segment
  int p = 1;
  Forest forest;
  std::vector<uint8_t> coarse_active, coarse_mat, coarse_init;
  // lattice (vertex lattice of level max_level + 1)
  int64_t NX[3] = {0, 0, 0};
  // composite DoFs (sorted lattice keys) and hanging constraints
  std::vector<int64_t> dof_key;
  std::vector<uint8_t> node_map; // lattice byte map of the last build (1 node, 2 hanging)
  std::unordered_map<int64_t, std::vector<std::pair<int32_t, double>>> hanging;
  int64_t n_nodes_all = 0; // distinct node positions of the active leaves

  int64_t key(int64_t X, int64_t Y, int64_t Z) const { return X + (NX[0] + 1) * (Y + (NX[1] + 1) * Z); }
  void unkey(int64_t k, int64_t x[3]) const
  {
    x[0] = k % (NX[0] + 1);
    k /= NX[0] + 1;
    x[1] = k % (NX[1] + 1);
    x[2] = k / (NX[1] + 1);
  }
  // lattice coordinate of local node a of cell i of level l
  int64_t lat(int l, int64_t i, int a) const { return (p * i + a) * ((int64_t)2 << (forest.max_level - l)) / p; }
  int64_t cell_size(int l) const { return (int64_t)2 << (forest.max_level - l); }

  bool in_domain(int l, int64_t i, int64_t j, int64_t k) const
  {
    return coarse_active[forest.index(0, i >> l, j >> l, k >> l)] != 0;
  }
  bool active_leaf(int l, int64_t i, int64_t j, int64_t k) const
  {
    return forest.leaf[l][forest.index(l, i, j, k)] && in_domain(l, i, j, k);
  }

  void init(adm_config const &c, int max_level)
  {
    cfg = c;
    if (cfg.degree != 1 && cfg.degree != 2)
      throw Error(ADM_ERR_UNSUPPORTED, "refined meshes take FE degree 1 or 2");
    if (max_level < 0 || max_level > 6)
      throw Error(ADM_ERR_UNSUPPORTED, "refinement levels: 0 to 6");
    for (int d = 0; d < 3; ++d)
      if (cfg.n_cells[d] < 1)
        throw Error(ADM_ERR_INVALID, "n_cells must be positive");
    p = cfg.degree;
    segments.assign(cfg.n_sources, {});
    for (int b = 0; b < cfg.n_sources; ++b)
    {
      adm_source const &s = cfg.sources[b];
      if (s.type != 2 && s.n_segments > 0)
      {
        if (!s.segments)
          throw Error(ADM_ERR_INVALID, "scan path segments missing");
        segments[b].assign(s.segments, s.segments + 5 * s.n_segments);
      }
      cfg.sources[b].segments = nullptr;
    }
    forest.init(cfg.n_cells, max_level);
    for (int d = 0; d < 3; ++d)
      NX[d] = (int64_t)cfg.n_cells[d] << (max_level + 1);
    size_t const C = forest.cells(0);
    coarse_active.assign(C, 1);
    coarse_mat.assign(C, 0);
    coarse_init.assign(C, 0);
  }

  void set_cells(uint8_t const *active, uint8_t const *mat, uint8_t const *init)
  {
    size_t const C = forest.cells(0);
    for (size_t c = 0; c < C; ++c)
    {
      coarse_active[c] = active ? (active[c] ? 1 : 0) : 1;
      if (mat && mat[c] >= cfg.n_materials)
        throw Error(ADM_ERR_INVALID, "material id out of range");
      coarse_mat[c] = mat ? mat[c] : 0;
      if (init && init[c] >= cfg.n_states)
        throw Error(ADM_ERR_INVALID, "initial state index out of range for the material states");
      coarse_init[c] = init ? init[c] : 0;
    }
  }

  // ScanPath::value (source/ScanPath.cc:228-257): the beam centre at t;
  // after the last segment a point far outside the domain.
  void beam_center(int b, double t, double out[3]) const
  {
    std::vector<double> const &sg = segments[b];
    int const n = (int)(sg.size() / 5);
    if (n == 0 || t > sg[(n - 1) * 5])
    {
      out[0] = out[1] = out[2] = std::numeric_limits<double>::lowest();
      return;
    }
    int lo = 0, hi = n - 1;
    while (lo < hi)
    {
      int const mid = (lo + hi) / 2;
      if (t > sg[mid * 5])
        lo = mid + 1;
      else
        hi = mid;
    }
    double st_t = 0.0, sp[3];
    for (int d = 0; d < 3; ++d)
      sp[d] = lo > 0 ? sg[(lo - 1) * 5 + 2 + d] : sg[lo * 5 + 2 + d];
    if (lo > 0)
      st_t = sg[(lo - 1) * 5];
    double const et = sg[lo * 5];
    for (int d = 0; d < 3; ++d)
      out[d] = sp[d] + (sg[lo * 5 + 2 + d] - sp[d]) / (et - st_t) * (t - st_t);
  }

  // compute_cells_to_refine: every leaf (material or not) whose bounding box
  // meets a beam box at one of the sample times (closed boxes).
  std::vector<uint8_t> cells_to_refine(int l, double time, double next_time, int n_steps) const
  {
    std::vector<std::array<double, 6>> boxes;
    double const scaling = 2.0;
    for (int s = 0; s < n_steps; ++s)
    {
      double const t = time + (double)s / (double)n_steps * (next_time - time);
      for (int b = 0; b < cfg.n_sources; ++b)
      {
        adm_source const &src = cfg.sources[b];
        if (src.type == 2)
        {
          boxes.push_back({src.cube_min[0], src.cube_min[1], src.cube_min[2], src.cube_max[0], src.cube_max[1],
                           src.cube_max[2]});
          continue;
        }
        double c[3];
        beam_center(b, t, c);
        double const r = std::sqrt(src.radius_squared);
        boxes.push_back({c[0] - scaling * r, c[1] - scaling * r, c[2] - scaling * src.depth, c[0] + scaling * r,
                         c[1] + scaling * r, c[2]});
      }
    }
    std::vector<uint8_t> flag(forest.cells(l), 0);
    double h[3];
    for (int d = 0; d < 3; ++d)
      h[d] = cfg.extent[d] / (double)forest.n(l, d);
    // only the cells that meet the boxes' union can meet a box
    double ulo[3] = {std::numeric_limits<double>::max(), std::numeric_limits<double>::max(),
                     std::numeric_limits<double>::max()};
    double uhi[3] = {std::numeric_limits<double>::lowest(), std::numeric_limits<double>::lowest(),
                     std::numeric_limits<double>::lowest()};
    for (auto const &bx : boxes)
      for (int d = 0; d < 3; ++d)
      {
        ulo[d] = std::min(ulo[d], bx[d]);
        uhi[d] = std::max(uhi[d], bx[3 + d]);
      }
    int64_t lo_i[3], hi_i[3];
    for (int d = 0; d < 3; ++d)
    {
      // cells i with origin + i h <= uhi and origin + (i + 1) h >= ulo, one
      // cell of margin against rounding (the exact test follows)
      double const a = std::floor((ulo[d] - cfg.origin[d]) / h[d]) - 2.0;
      double const b = std::floor((uhi[d] - cfg.origin[d]) / h[d]) + 2.0;
      lo_i[d] = boxes.empty() ? 1 : (int64_t)std::max(0.0, std::min(a, (double)forest.n(l, d)));
      hi_i[d] = boxes.empty() ? 0 : (int64_t)std::max(-1.0, std::min(b, (double)forest.n(l, d) - 1.0));
    }
    for (int64_t k = lo_i[2]; k <= hi_i[2]; ++k)
      for (int64_t j = lo_i[1]; j <= hi_i[1]; ++j)
        for (int64_t i = lo_i[0]; i <= hi_i[0]; ++i)
        {
          int64_t const c = forest.index(l, i, j, k);
          if (!forest.leaf[l][c])
            continue;
          double const lo[3] = {cfg.origin[0] + i * h[0], cfg.origin[1] + j * h[1], cfg.origin[2] + k * h[2]};
          double const hi[3] = {cfg.origin[0] + (i + 1) * h[0], cfg.origin[1] + (j + 1) * h[1],
                                cfg.origin[2] + (k + 1) * h[2]};
          for (auto const &bx : boxes)
            if (lo[0] <= bx[3] && bx[0] <= hi[0] && lo[1] <= bx[4] && bx[1] <= hi[1] && lo[2] <= bx[5] &&
                bx[2] <= hi[2])
            {
              flag[c] = 1;
              break;
            }
        }
    return flag;
  }

  // Execute per-leaf refine / coarsen flags (level-indexed arrays of the
  // current leaves): refine, coarsen the families whose 8 children are all
  // flagged leaves (unless that breaks the balance), then balance.
  void execute(std::vector<std::vector<uint8_t>> const &refine, std::vector<std::vector<uint8_t>> const &coarsen)
  {
    Forest const old = forest;
    int const L = forest.max_level;
    for (int l = 0; l < L; ++l)
      for (int64_t k = 0; k < forest.n(l, 2); ++k)
        for (int64_t j = 0; j < forest.n(l, 1); ++j)
          for (int64_t i = 0; i < forest.n(l, 0); ++i)
          {
            int64_t const c = forest.index(l, i, j, k);
            if (old.leaf[l][c] && !refine[l].empty() && refine[l][c])
              forest.refine(l, i, j, k);
          }
    for (int l = L - 1; l >= 0; --l)
    {
      if (coarsen[l + 1].empty())
        continue;
      for (int64_t k = 0; k < forest.n(l, 2); ++k)
        for (int64_t j = 0; j < forest.n(l, 1); ++j)
          for (int64_t i = 0; i < forest.n(l, 0); ++i)
          {
            int64_t const c = forest.index(l, i, j, k);
            if (!forest.exists[l][c] || forest.leaf[l][c])
              continue;
            bool all = true;
            for (int q = 0; q < 8 && all; ++q)
            {
              int64_t const cc = forest.index(l + 1, 2 * i + (q & 1), 2 * j + ((q >> 1) & 1), 2 * k + (q >> 2));
              all = forest.leaf[l + 1][cc] && old.leaf[l + 1][cc] && coarsen[l + 1][cc];
            }
            if (all && forest.coarsening_keeps_balance(l, i, j, k))
              forest.coarsen(l, i, j, k);
          }
    }
    forest.balance();
  }

  // refine_mesh: n_refinements rounds of beam-box flags.
  void refine_mesh(double time, double next_time, int n_steps, int n_refinements, bool coarsen_after_beam)
  {
    int const L = forest.max_level;
    if (n_refinements > L)
      throw Error(ADM_ERR_INVALID, "n_refinements exceeds the mesh's maximum level");
    if (n_steps < 1)
      throw Error(ADM_ERR_INVALID, "n_time_steps must be positive");
    for (int r = 0; r < n_refinements; ++r)
    {
      std::vector<std::vector<uint8_t>> ref(L + 1), crs(L + 1);
      for (int l = 0; l <= L; ++l)
      {
        std::vector<uint8_t> const hit = cells_to_refine(l, time, next_time, n_steps);
        int64_t const nc = forest.cells(l);
        ref[l].resize(nc);
        crs[l].resize(nc);
        uint8_t const *lf = forest.leaf[l].data(), *h = hit.data();
        uint8_t *rf = ref[l].data(), *cr = crs[l].data();
        uint8_t const do_crs = (coarsen_after_beam && l > 0) ? 1 : 0, do_ref = l < n_refinements ? 1 : 0;
        // leaves: coarsen the ones the beam misses (above level 0), refine
        // the ones it meets (below the refinement count)
        for (int64_t c = 0; c < nc; ++c)
        {
          uint8_t const leaf = lf[c] != 0, hitc = h[c] != 0;
          cr[c] = leaf & (hitc ^ 1) & do_crs;
          rf[c] = leaf & hitc & do_ref;
        }
      }
      execute(ref, crs);
    }
  }

  // DoFs and constraints of the current forest.
  void build()
  {
    int const L = forest.max_level;
    // node positions of the active leaves on a dense byte map of the
    // lattice (1: node, 2: hanging node); its scan in key order gives the
    // sorted DoF keys
    size_t const n_lat = (size_t)(NX[0] + 1) * (NX[1] + 1) * (NX[2] + 1);
    node_map.assign(n_lat, 0);
    int64_t n_all = 0;
    int64_t const sx = 1, sy = NX[0] + 1, sz = (NX[0] + 1) * (NX[1] + 1); // key strides
    for (int l = 0; l <= L; ++l)
    {
      int64_t const fac = cell_size(l) / p; // lattice spacing of the level's nodes
      for (int64_t k = 0; k < forest.n(l, 2); ++k)
        for (int64_t j = 0; j < forest.n(l, 1); ++j)
        {
          uint8_t const *lf = &forest.leaf[l][forest.index(l, 0, j, k)];
          for (int64_t i = 0; i < forest.n(l, 0); ++i)
          {
            if (!lf[i] || !in_domain(l, i, j, k))
              continue;
            int64_t const k0 = key(lat(l, i, 0), lat(l, j, 0), lat(l, k, 0));
            for (int c = 0; c <= p; ++c)
              for (int b = 0; b <= p; ++b)
                for (int a = 0; a <= p; ++a)
                {
                  uint8_t &v = node_map[k0 + fac * (a * sx + b * sy + c * sz)];
                  n_all += v == 0;
                  v = 1;
                }
          }
        }
    }
    n_nodes_all = n_all;
    // hanging nodes: fine nodes on a face / edge of an active leaf whose
    // neighbour region across it is refined material, off the leaf's nodes
    std::unordered_map<int64_t, std::vector<std::pair<int64_t, double>>> hk;
    for (int l = 0; l < L; ++l)
      for (int64_t k = 0; k < forest.n(l, 2); ++k)
        for (int64_t j = 0; j < forest.n(l, 1); ++j)
        {
          uint8_t const *lf = &forest.leaf[l][forest.index(l, 0, j, k)];
          for (int64_t i = 0; i < forest.n(l, 0); ++i)
          {
            if (!lf[i] || !in_domain(l, i, j, k))
              continue;
            int64_t const cc[3] = {i, j, k};
            for (int o = 0; o < kFaceEdge.n; ++o)
            {
              int64_t nb[3];
              for (int d = 0; d < 3; ++d)
                nb[d] = cc[d] + kFaceEdge.o[o][d];
              if (!forest.inside(l, nb[0], nb[1], nb[2]) || !in_domain(l, nb[0], nb[1], nb[2]))
                continue;
              // the neighbour region is refined (Forest::status == l + 1)
              // exactly when its level-l cell exists and is not a leaf
              int64_t const nbc = forest.index(l, nb[0], nb[1], nb[2]);
              if (!forest.exists[l][nbc] || forest.leaf[l][nbc])
                continue;
              // the shared entity: fixed coordinate (0 or p) along the
              // offset's nonzero directions, free along the others
              int fixed[3];
              for (int d = 0; d < 3; ++d)
                fixed[d] = kFaceEdge.o[o][d] == 0 ? -1 : (kFaceEdge.o[o][d] > 0 ? 2 * p : 0);
              int const lim[3] = {fixed[0] < 0 ? 2 * p : 0, fixed[1] < 0 ? 2 * p : 0, fixed[2] < 0 ? 2 * p : 0};
              for (int sz = 0; sz <= lim[2]; ++sz)
                for (int sy = 0; sy <= lim[1]; ++sy)
                  for (int sx = 0; sx <= lim[0]; ++sx)
                  {
                    int s[3] = {sx, sy, sz};
                    for (int d = 0; d < 3; ++d)
                      if (fixed[d] >= 0)
                        s[d] = fixed[d];
                    // s: level-(l+1) node offsets within the leaf (0..2p)
                    if (s[0] % 2 == 0 && s[1] % 2 == 0 && s[2] % 2 == 0)
                      continue; // a node of the leaf itself
                    int64_t X[3];
                    for (int d = 0; d < 3; ++d)
                      X[d] = lat(l, cc[d], 0) + (int64_t)s[d] * cell_size(l) / (2 * p);
                    int64_t const hkey = key(X[0], X[1], X[2]);
                    if (hk.count(hkey))
                      continue;
                    std::vector<std::pair<int64_t, double>> ent;
                    double wsum = 0.0;
                    for (int c = 0; c <= p; ++c)
                      for (int b = 0; b <= p; ++b)
                        for (int a = 0; a <= p; ++a)
                        {
                          int const abc[3] = {a, b, c};
                          double w = 1.0;
                          for (int d = 0; d < 3; ++d)
                            w *= lagrange(p, abc[d], s[d] / (2.0 * p));
                          if (w == 0.0)
                            continue;
                          ent.push_back({key(lat(l, i, a), lat(l, j, b), lat(l, k, c)), w});
                          wsum += w;
                        }
                    (void)wsum;
                    hk[hkey] = std::move(ent);
                  }
            }
          }
        }
    // masters: the keys of the non-hanging nodes, in key order (the map is
    // scanned eight entries at a time, skipping empty words)
    for (auto const &kv : hk)
      node_map[kv.first] = 2;
    dof_key.clear();
    dof_key.reserve(n_all);
    {
      size_t const nw = n_lat / 8;
      uint64_t const *w = reinterpret_cast<uint64_t const *>(node_map.data());
      for (size_t q = 0; q < nw; ++q)
      {
        uint64_t x = 0;
        std::memcpy(&x, w + q, 8);
        if (!x)
          continue;
        for (int b = 0; b < 8; ++b)
          if (node_map[8 * q + b] == 1)
            dof_key.push_back((int64_t)(8 * q + b));
      }
      for (size_t q = 8 * nw; q < n_lat; ++q)
        if (node_map[q] == 1)
          dof_key.push_back((int64_t)q);
    }
    // resolve chains (a master that is itself hanging)
    hanging.clear();
    for (auto const &kv : hk)
    {
      std::vector<std::pair<int64_t, double>> cur = kv.second;
      for (int depth = 0; depth < 8; ++depth)
      {
        bool again = false;
        std::vector<std::pair<int64_t, double>> nxt;
        for (auto const &e : cur)
        {
          auto it = hk.find(e.first);
          if (it == hk.end())
            nxt.push_back(e);
          else
          {
            again = true;
            for (auto const &f : it->second)
              nxt.push_back({f.first, e.second * f.second});
          }
        }
        cur.swap(nxt);
        if (!again)
          break;
        if (depth == 7)
          throw Error(ADM_ERR_INVALID, "internal: hanging-node constraints do not resolve");
      }
      std::vector<std::pair<int32_t, double>> res;
      for (auto const &e : cur)
      {
        int32_t const dof = find_dof(e.first);
        if (dof < 0)
          throw Error(ADM_ERR_INVALID, "internal: constraint master is not a node of the mesh");
        bool merged = false;
        for (auto &r : res)
          if (r.first == dof)
          {
            r.second += e.second;
            merged = true;
          }
        if (!merged)
          res.push_back({dof, e.second});
      }
      std::sort(res.begin(), res.end());
      hanging[kv.first] = std::move(res);
    }
  }

  // the DoF of a node key, or -1 (binary search of the sorted keys)
  int32_t find_dof(int64_t k) const
  {
    auto const it = std::lower_bound(dof_key.begin(), dof_key.end(), k);
    return (it != dof_key.end() && *it == k) ? (int32_t)(it - dof_key.begin()) : -1;
  }

  // entries (dof, weight) of the value at a node key
  void entries(int64_t k, std::vector<std::pair<int32_t, double>> &out) const
  {
    out.clear();
    int32_t const dof = find_dof(k);
    if (dof >= 0)
    {
      out.push_back({dof, 1.0});
      return;
    }
    auto h = hanging.find(k);
    if (h == hanging.end())
      throw Error(ADM_ERR_INVALID, "internal: node without DoF or constraint");
    out = h->second;
  }

  int64_t n_active_leaves(int l) const
  {
    int64_t n = 0;
    for (int64_t k = 0; k < forest.n(l, 2); ++k)
      for (int64_t j = 0; j < forest.n(l, 1); ++j)
        for (int64_t i = 0; i < forest.n(l, 0); ++i)
          n += active_leaf(l, i, j, k) ? 1 : 0;
    return n;
  }
};

// ------------------------------------------------------------ GPU kernels
namespace
{
// y_lev[row_pos[r]] = sum_e w[e] y[dof[e]] over the row's entries
// A composite vector given as y + dt sum_j a_j k_j (nk <= 3 terms; nk 0:
// y itself): an RK stage input formed where it is read.
struct StageSum
{
  double const *y;
  double dt;
  int nk;
  double a[3];
  double const *k[3];
};

__device__ __forceinline__ double stage_value(StageSum const &v, int64_t d)
{
  double x = v.y[d];
  double s = 0.0;
  for (int j = 0; j < v.nk; ++j)
    s = fma(v.a[j], v.k[j][d], s);
  return v.nk ? fma(v.dt, s, x) : x;
}

// lev[row_pos[r]] = sum_e w[e] v[dof[e]], v the composite vector
__global__ void prolong_kernel(int64_t n_rows, int64_t const *row_pos, int64_t const *row_ptr, int32_t const *dof,
                               double const *w, StageSum v, double *lev)
{
  int64_t const r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n_rows)
    return;
  double s = 0.0;
  for (int64_t e = row_ptr[r]; e < row_ptr[r + 1]; ++e)
    s += w[e] * stage_value(v, dof[e]);
  lev[row_pos[r]] = s;
}

// out[d] = sum_e w[e] lev[pos[e]] (add: out[d] += ...; scale: times
// scale[d], the inverse mass of an RK stage derivative)
__global__ void restrict_kernel(int64_t n_dofs, int64_t const *ptr, int64_t const *pos, double const *w,
                                double const *lev, double *out, int add, double const *scale)
{
  int64_t const d = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (d >= n_dofs)
    return;
  double s = 0.0;
  for (int64_t e = ptr[d]; e < ptr[d + 1]; ++e)
    s += w[e] * lev[pos[e]];
  if (scale)
    s *= scale[d];
  out[d] = add ? out[d] + s : s;
}

// out[r] = lev[pos[r]]
__global__ void gather_kernel(int64_t n, int64_t const *pos, double const *lev, double *out)
{
  int64_t const r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r < n)
    out[r] = lev[pos[r]];
}

__global__ void invert_kernel(int64_t n, double *m)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n)
    m[i] = m[i] > 0.0 ? 1.0 / m[i] : 0.0;
}

// mass_lev = 1 / inv_mass_lev on the rows' nodes
__global__ void mass_from_inverse_kernel(int64_t n_rows, int64_t const *row_pos, int64_t off,
                                         double const *inv_mass, double *lev)
{
  int64_t const r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= n_rows)
    return;
  int64_t const p = row_pos[r];
  double const v = inv_mass[p - off];
  lev[p] = v > 0.0 ? 1.0 / v : 0.0;
}

// z = y + dt sum_j a_j k_j (up to 3 stage vectors)
__global__ void stage_input_kernel(int64_t n, double const *y, double dt, int nk, double a0, double const *k0,
                                   double a1, double const *k1, double a2, double const *k2, double *z)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n)
    return;
  double s = 0.0;
  if (nk > 0)
    s += a0 * k0[i];
  if (nk > 1)
    s += a1 * k1[i];
  if (nk > 2)
    s += a2 * k2[i];
  z[i] = y[i] + dt * s;
}

__global__ void fill_kernel(int64_t n, double v, double *y)
{
  int64_t const i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n)
    y[i] = v;
}

unsigned blocks(int64_t n) { return (unsigned)std::max<int64_t>(1, (n + 255) / 256); }
} // namespace

// -------------------------------------------------------------- GPU driver
class Amr
{
public:
  // All work runs on the handle's own stream, ordered after the caller's
  // stream at every entry and before it at every exit (events), so a time
  // step can be captured in a graph whatever stream the caller uses.
  Amr(adm_config const &cfg, int max_level, int device, cudaStream_t stream) : device_(device), user_(stream)
  {
    mesh_.init(cfg, max_level);
    if (cfg.dim != 3)
      throw Error(ADM_ERR_UNSUPPORTED, "refined meshes are 3-D");
    ADM_CK(cudaSetDevice(device_));
    ADM_CK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    ADM_CK(cudaEventCreateWithFlags(&ev_in_, cudaEventDisableTiming));
    ADM_CK(cudaEventCreateWithFlags(&ev_out_, cudaEventDisableTiming));
    ADM_CK(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
    // one stream per level grid: the levels' operators run concurrently,
    // forked from the handle's stream and joined back (events)
    lstream_.assign(max_level + 1, nullptr);
    ev_lev_.assign(max_level + 1, nullptr);
    for (int l = 0; l <= max_level; ++l)
    {
      ADM_CK(cudaStreamCreateWithFlags(&lstream_[l], cudaStreamNonBlocking));
      ADM_CK(cudaEventCreateWithFlags(&ev_lev_[l], cudaEventDisableTiming));
    }
  }

  ~Amr()
  {
    cudaSetDevice(device_);
    if (stream_)
      cudaStreamSynchronize(stream_);
    drop_graph();
    for (cudaStream_t ls : lstream_)
      if (ls)
        cudaStreamSynchronize(ls);
    levels_.clear();
    for (cudaStream_t ls : lstream_)
      if (ls)
        cudaStreamDestroy(ls);
    for (cudaEvent_t e : ev_lev_)
      if (e)
        cudaEventDestroy(e);
    if (ev_fork_)
      cudaEventDestroy(ev_fork_);
    if (ev_in_)
      cudaEventDestroy(ev_in_);
    if (ev_out_)
      cudaEventDestroy(ev_out_);
    if (stream_)
      cudaStreamDestroy(stream_);
  }

  Amr(Amr const &) = delete;
  Amr &operator=(Amr const &) = delete;

  struct Ordered
  {
    Amr &a;
    explicit Ordered(Amr &x) : a(x)
    {
      ADM_CK(cudaSetDevice(a.device_));
      ADM_CK(cudaEventRecord(a.ev_in_, a.user_));
      ADM_CK(cudaStreamWaitEvent(a.stream_, a.ev_in_, 0));
    }
    ~Ordered()
    {
      cudaEventRecord(a.ev_out_, a.stream_);
      cudaStreamWaitEvent(a.user_, a.ev_out_, 0);
    }
  };

  AmrMesh &mesh() { return mesh_; }
  AmrMesh const &mesh() const { return mesh_; }
  int64_t n_dofs() const { return (int64_t)mesh_.dof_key.size(); }
  double *solution() { return y_.p; }

  void setup(double initial_temperature)
  {
    Ordered ord(*this);
    mesh_.build();
    build_levels(nullptr);
    y_.alloc(n_dofs());
    fill_kernel<<<blocks(n_dofs()), 256, 0, stream_>>>(n_dofs(), initial_temperature, y_.p);
    ADM_CK(cudaGetLastError());
    compute_inverse_mass();
    ready_ = true;
  }

  void require_ready() const
  {
    if (!ready_)
      throw Error(ADM_ERR_INVALID, "setup() has not been called");
  }

  // phase time since the last lap
  void remesh_lap(int phase)
  {
    auto const now = std::chrono::steady_clock::now();
    remesh_ms_[phase] = std::chrono::duration<double, std::milli>(now - remesh_clock_).count();
    remesh_clock_ = now;
  }

  // refine_and_transfer around an AmrMesh change (done by `change`)
  template <class F> void remesh(F &&change)
  {
    require_ready();
    Ordered ord(*this);
    remesh_clock_ = std::chrono::steady_clock::now();
    auto lap = [&](int phase) { remesh_lap(phase); };
    // the old field at the level nodes of the old leaves (constraints
    // resolved; only those nodes come back to the host) and the old cell
    // states (ThermalPhysics::set_state_to_material_properties)
    prolong(y_.p);
    Snapshot old;
    old.forest = mesh_.forest;
    old.off = lev_off_;
    // the old composite values with their (sorted) lattice keys: a new DoF
    // on an old DoF's position takes its value as it is
    old.dof_key = mesh_.dof_key;
    old.dof_val.resize(n_dofs());
    ADM_CK(cudaMemcpyAsync(old.dof_val.data(), y_.p, n_dofs() * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    ADM_CK(cudaStreamSynchronize(stream_));
    if (n_rows_ > 0)
    {
      snap_rows_.ensure(n_rows_);
      gather_kernel<<<blocks(n_rows_), 256, 0, stream_>>>(n_rows_, row_pos_.p, src_lev_.p, snap_rows_.p);
      ADM_CK(cudaGetLastError());
      old.row_val.resize(n_rows_);
      ADM_CK(cudaMemcpyAsync(old.row_val.data(), snap_rows_.p, n_rows_ * sizeof(double), cudaMemcpyDeviceToHost,
                             stream_));
      ADM_CK(cudaStreamSynchronize(stream_));
      old.row_pos = row_pos_h_; // ascending: levels in order, nodes sorted
    }
    int const ns = mesh_.cfg.n_states;
    fork();
    old.states.resize(levels_.size());
    old.melted.resize(levels_.size());
    old.pitch.assign(levels_.size(), 0);
    old.nn1.assign(levels_.size(), 0);
    old.state_cells.resize(levels_.size());
    for (size_t l = 0; l < levels_.size(); ++l)
    {
      if (!alive(l))
        continue;
      levels_[l]->set_state_to_material_properties();
      // the states of the level's active leaves (ascending cell index)
      std::vector<int32_t> &cells = old.state_cells[l];
      for (int64_t k = 0; k < mesh_.forest.n((int)l, 2); ++k)
        for (int64_t j = 0; j < mesh_.forest.n((int)l, 1); ++j)
          for (int64_t i = 0; i < mesh_.forest.n((int)l, 0); ++i)
            if (mesh_.active_leaf((int)l, i, j, k))
              cells.push_back((int32_t)mesh_.forest.index((int)l, i, j, k));
      old.states[l].resize(cells.size() * ns);
      levels_[l]->get_cell_state_sparse(cells.data(), cells.size(), old.states[l].data());
      old.melted[l] = levels_[l]->has_melted_cells();
      old.pitch[l] = levels_[l]->mesh().pitch;
      old.nn1[l] = levels_[l]->mesh().nn[1];
    }
    lap(0);
    change();
    lap(1);
    mesh_.build();
    lap(2);
    build_levels(&old); // phases 3-5
    // SolutionTransfer: the old field at the new nodes
    // both key lists ascend: one walk through the old keys
    std::vector<double> y(n_dofs());
    size_t at = 0;
    for (int64_t d = 0; d < n_dofs(); ++d)
    {
      int64_t const key = mesh_.dof_key[d];
      while (at < old.dof_key.size() && old.dof_key[at] < key)
        ++at;
      y[d] = (at < old.dof_key.size() && old.dof_key[at] == key) ? old.dof_val[at] : old.evaluate(mesh_, key);
    }
    y_.ensure(n_dofs());
    ADM_CK(cudaMemcpyAsync(y_.p, y.data(), y.size() * sizeof(double), cudaMemcpyHostToDevice, stream_));
    ADM_CK(cudaStreamSynchronize(stream_));
    lap(6);
    compute_inverse_mass();
    ADM_CK(cudaStreamSynchronize(stream_));
    lap(7);
  }

  // host wall time of the last remesh's phases: snapshot of the old field
  // and states, flagging and execution, nodes and constraints, level-grid
  // set-up, cell-state transfer, prolongation tables, solution transfer,
  // inverse mass
  double remesh_ms_[kRemeshPhases] = {0, 0, 0, 0, 0, 0, 0, 0};
  std::chrono::steady_clock::time_point remesh_clock_;

  // Level-grid schedule (coloured: 8 launches per level and application,
  // deterministic; atomic: 1 launch, additions in any order; two-pass: a
  // tile launch and a gather, deterministic).
  void set_schedule(int schedule)
  {
    if (schedule != Thermal::kScheduleColoured && schedule != Thermal::kScheduleAtomic &&
        schedule != Thermal::kScheduleTwoPass)
      throw Error(ADM_ERR_INVALID, "unknown schedule");
    schedule_ = schedule;
    drop_graph();
    for (auto &th : levels_)
      if (th)
        th->set_schedule(schedule);
  }

  void set_time(double t)
  {
    require_ready();
    Ordered ord(*this);
    fork();
    for (size_t l = 0; l < levels_.size(); ++l)
      if (alive(l))
        levels_[l]->set_time(t);
    join();
  }

  // dst = C^T (sum_l A_l) C src (composite vectors on the device)
  void vmult(double *dst, double const *src)
  {
    require_ready();
    Ordered ord(*this);
    prolong(src);
    fork();
    for (size_t l = 0; l < levels_.size(); ++l)
      if (alive(l))
        levels_[l]->vmult(dst_lev_.p + lev_off_[l], src_lev_.p + lev_off_[l], false);
    join();
    restrict_to(dst, 0);
  }

  double const *inverse_mass() const { return inv_m_.p; }

  void copy_inverse_mass(double *dst)
  {
    require_ready();
    Ordered ord(*this);
    ADM_CK(cudaMemcpyAsync(dst, inv_m_.p, n_dofs() * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    ADM_CK(cudaStreamSynchronize(stream_));
  }

  // device copies of the solution, ordered on the handle's stream
  void copy_solution(double *other, bool out)
  {
    require_ready();
    Ordered ord(*this);
    size_t const bytes = n_dofs() * sizeof(double);
    if (out)
      ADM_CK(cudaMemcpyAsync(other, y_.p, bytes, cudaMemcpyDeviceToDevice, stream_));
    else
      ADM_CK(cudaMemcpyAsync(y_.p, other, bytes, cudaMemcpyDeviceToDevice, stream_));
    ADM_CK(cudaStreamSynchronize(stream_));
  }

  // One explicit Runge-Kutta step of the solution: the level clocks are set
  // to (t, dt), then the step's launches (stage inputs, prolongation, the
  // levels' operators with the sources at t + c_i dt, restriction, inverse
  // mass, update) replay as one graph, captured on the first step after a
  // mesh change or with a new dt.
  double evolve_one_time_step(double t, double dt)
  {
    require_ready();
    Ordered ord(*this);
    Thermal::Tableau const tab = Thermal::tableau(mesh_.cfg.time_method);
    int64_t const n = n_dofs();
    double *before[4];
    for (int i = 0; i < 4; ++i)
      before[i] = k_[i].p;
    for (int i = 0; i < tab.s; ++i)
      k_[i].ensure(n);
    for (int i = 0; i < 4; ++i)
      if (k_[i].p != before[i])
        drop_graph(); // the graph holds the stage vectors' addresses
    // the level clocks, after the last replay and before this one
    fork();
    for (size_t l = 0; l < levels_.size(); ++l)
      if (alive(l))
        levels_[l]->set_step_clock(t, dt);
    join();
    if (!step_exec_ || step_dt_ != dt)
    {
      drop_graph();
      cudaGraph_t g = nullptr;
      ADM_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
      try
      {
        step_body(dt, tab);
      }
      catch (...)
      {
        cudaStreamEndCapture(stream_, &g);
        if (g)
          cudaGraphDestroy(g);
        throw;
      }
      ADM_CK(cudaStreamEndCapture(stream_, &g));
      cudaError_t const e = cudaGraphInstantiate(&step_exec_, g, 0);
      cudaGraphDestroy(g);
      ADM_CK(e);
      step_dt_ = dt;
    }
    ADM_CK(cudaGraphLaunch(step_exec_, stream_));
    return t + dt;
  }

  // the composite field on the level grid of level l (constraints resolved)
  void level_values(int l, double *host)
  {
    require_ready();
    Ordered ord(*this);
    if (l < 0 || l >= (int)levels_.size() || !alive(l))
      throw Error(ADM_ERR_INVALID, "no leaves on this level");
    prolong(y_.p);
    ADM_CK(cudaMemcpyAsync(host, src_lev_.p + lev_off_[l], levels_[l]->m() * sizeof(double),
                           cudaMemcpyDeviceToHost, stream_));
    ADM_CK(cudaStreamSynchronize(stream_));
  }

  Thermal *level(int l) { return (l >= 0 && l < (int)levels_.size() && alive(l)) ? levels_[l].get() : nullptr; }
  bool alive(size_t l) const { return l < alive_.size() && alive_[l] && levels_[l]; }

  void synchronize() { ADM_CK(cudaStreamSynchronize(stream_)); }

  // the level streams wait for the handle's stream / the handle's stream
  // waits for the level streams
  void fork()
  {
    ADM_CK(cudaEventRecord(ev_fork_, stream_));
    for (size_t l = 0; l < lstream_.size(); ++l)
      if (levels_.size() > l && levels_[l])
        ADM_CK(cudaStreamWaitEvent(lstream_[l], ev_fork_, 0));
  }

  void join()
  {
    for (size_t l = 0; l < lstream_.size(); ++l)
      if (levels_.size() > l && levels_[l])
      {
        ADM_CK(cudaEventRecord(ev_lev_[l], lstream_[l]));
        ADM_CK(cudaStreamWaitEvent(stream_, ev_lev_[l], 0));
      }
  }

  // ThermalPhysics::mark_has_melted on the refined mesh: the leaves whose
  // cell average of the field exceeds threshold (flags stay set)
  void mark_has_melted(double threshold)
  {
    require_ready();
    Ordered ord(*this);
    prolong(y_.p);
    fork();
    for (size_t l = 0; l < levels_.size(); ++l)
      if (alive(l))
        levels_[l]->mark_has_melted(threshold, src_lev_.p + lev_off_[l], nullptr);
    join();
  }

  // the has_melted flags of a level grid's cells (host, cells of the grid)
  void level_has_melted(int l, uint8_t *host)
  {
    require_ready();
    Thermal *th = level(l);
    if (!th)
      throw Error(ADM_ERR_INVALID, "no leaves on this level");
    std::copy(th->has_melted_cells().begin(), th->has_melted_cells().end(), host);
  }

  // the cell states of a level grid (host, n_states x cells of the grid)
  void level_cell_state(int l, double *host)
  {
    require_ready();
    Ordered ord(*this);
    Thermal *th = level(l);
    if (!th)
      throw Error(ADM_ERR_INVALID, "no leaves on this level");
    fork();
    th->set_state_to_material_properties();
    th->get_cell_state(host);
  }

private:
  void drop_graph()
  {
    if (step_exec_)
    {
      cudaGraphExecDestroy(step_exec_);
      step_exec_ = nullptr;
    }
  }

  // k = C^T (sum_l A_l) C src with the sources at stage c of the clocked step
  // dst = (scale .) C^T sum_l A_l C v at the stage time t + c dt, v the
  // composite vector (a stage input formed in the prolongation)
  void vmult_stage(double *dst, StageSum const &v, double c, double const *scale = nullptr)
  {
    prolong(v);
    fork();
    for (size_t l = 0; l < levels_.size(); ++l)
      if (alive(l))
        levels_[l]->vmult_stage(dst_lev_.p + lev_off_[l], src_lev_.p + lev_off_[l], c);
    join();
    restrict_to(dst, 0, scale);
  }

  void vmult_stage(double *dst, double const *src, double c)
  {
    StageSum v{};
    v.y = src;
    vmult_stage(dst, v, c);
  }

  void step_body(double dt, Thermal::Tableau const &tab)
  {
    int64_t const n = n_dofs();
    for (int i = 0; i < tab.s; ++i)
    {
      // the stage input y + dt sum_{j<i} a_ij k_j is formed by the
      // prolongation, and k_i = M^-1 (...) by the restriction
      StageSum v{};
      v.y = y_.p;
      v.dt = dt;
      for (int j = 0; j < i; ++j)
        if (tab.a[i][j] != 0.0)
        {
          if (v.nk == 3)
            throw Error(ADM_ERR_INVALID, "internal: more than three stage terms");
          v.a[v.nk] = tab.a[i][j];
          v.k[v.nk] = k_[j].p;
          ++v.nk;
        }
      vmult_stage(k_[i].p, v, tab.c[i], inv_m_.p);
    }
    // y += dt sum_i b_i k_i
    double a[3] = {0, 0, 0};
    double const *kk[3] = {k_[0].p, k_[0].p, k_[0].p};
    int nk = 0;
    for (int i = 0; i < tab.s; ++i)
      if (tab.b[i] != 0.0)
      {
        if (nk == 3)
        {
          stage_input_kernel<<<blocks(n), 256, 0, stream_>>>(n, y_.p, dt, nk, a[0], kk[0], a[1], kk[1], a[2],
                                                              kk[2], y_.p);
          nk = 0;
        }
        a[nk] = tab.b[i];
        kk[nk] = k_[i].p;
        ++nk;
      }
    stage_input_kernel<<<blocks(n), 256, 0, stream_>>>(n, y_.p, dt, nk, a[0], kk[0], a[1], kk[1], a[2], kk[2],
                                                        y_.p);
    ADM_CK(cudaGetLastError());
  }

  struct Snapshot
  {
    Forest forest;
    std::vector<int64_t> off;
    // the old field at the old leaves' level nodes (ascending level-buffer
    // positions) and the old composite DoFs (ascending lattice keys)
    std::vector<int64_t> row_pos, dof_key;
    std::vector<double> row_val, dof_val;

    std::vector<std::vector<int32_t>> state_cells; // per level: the active leaves, ascending
    std::vector<std::vector<double>> states;       // per level: their states [leaf][n_states]
    std::vector<std::vector<uint8_t>> melted;
    std::vector<int> pitch, nn1;

    // the old field at lattice node k: an old active leaf containing it
    double evaluate(AmrMesh const &m, int64_t k) const
    {
      int64_t X[3];
      m.unkey(k, X);
      int const p = m.p;
      for (int l = 0; l <= forest.max_level; ++l)
      {
        int64_t const S = m.cell_size(l);
        int64_t lo[3], hi[3];
        for (int d = 0; d < 3; ++d)
        {
          hi[d] = X[d] / S;
          lo[d] = (X[d] % S == 0) ? hi[d] - 1 : hi[d];
        }
        for (int64_t c = lo[2]; c <= hi[2]; ++c)
          for (int64_t b = lo[1]; b <= hi[1]; ++b)
            for (int64_t a = lo[0]; a <= hi[0]; ++a)
            {
              if (!forest.inside(l, a, b, c) || !forest.leaf[l][forest.index(l, a, b, c)] ||
                  !m.in_domain(l, a, b, c))
                continue;
              int64_t const cell[3] = {a, b, c};
              double u[3];
              for (int d = 0; d < 3; ++d)
                u[d] = (double)(X[d] - cell[d] * S) / (double)S;
              double v = 0.0;
              for (int q2 = 0; q2 <= p; ++q2)
                for (int q1 = 0; q1 <= p; ++q1)
                  for (int q0 = 0; q0 <= p; ++q0)
                  {
                    double const w = lagrange(p, q0, u[0]) * lagrange(p, q1, u[1]) * lagrange(p, q2, u[2]);
                    if (w == 0.0)
                      continue;
                    int64_t const nidx = (p * a + q0) + (int64_t)pitch[l] * ((p * b + q1) + (int64_t)nn1[l] * (p * c + q2));
                    auto it = std::lower_bound(row_pos.begin(), row_pos.end(), off[l] + nidx);
                    if (it == row_pos.end() || *it != off[l] + nidx)
                      throw Error(ADM_ERR_INVALID, "internal: old leaf node without a value");
                    v += w * row_val[it - row_pos.begin()];
                  }
              return v;
            }
      }
      throw Error(ADM_ERR_INVALID, "internal: a new node lies in no old active leaf");
    }

    // CellDataTransfer: the state and has_melted flag of the new leaf
    // (l, i, j, k)
    void state_of(int l, int64_t i, int64_t j, int64_t k, int ns, double *out, uint8_t *melt = nullptr) const
    {
      int m = forest.status(l, i, j, k);
      int64_t a = i, b = j, c = k;
      if (m <= l)
      {
        int const s = l - m;
        a >>= s;
        b >>= s;
        c >>= s;
      }
      else
      {
        // coarsened: the first child, down to a leaf
        m = l;
        while (!forest.leaf[m][forest.index(m, a, b, c)])
        {
          a *= 2;
          b *= 2;
          c *= 2;
          ++m;
        }
      }
      int64_t const cell = forest.index(m, a, b, c);
      std::vector<int32_t> const &lc = state_cells[m];
      auto const it = std::lower_bound(lc.begin(), lc.end(), (int32_t)cell);
      bool const found = it != lc.end() && *it == (int32_t)cell;
      for (int q = 0; q < ns; ++q)
        out[q] = found ? states[m][(size_t)(it - lc.begin()) * ns + q] : 0.0;
      if (melt)
        *melt = melted[m].empty() ? 0 : melted[m][cell];
    }
  };

  void build_levels(Snapshot const *old)
  {
    auto lap_ms = [&] {
      auto const now = std::chrono::steady_clock::now();
      double const ms = std::chrono::duration<double, std::milli>(now - remesh_clock_).count();
      remesh_clock_ = now;
      return ms;
    };
    double t_setup = 0.0, t_states = 0.0;
    lap_ms();
    drop_graph();
    fork();
    int const L = mesh_.forest.max_level;
    int const ns = mesh_.cfg.n_states;
    // level Thermals persist across remeshing (set up again on the new
    // leaves); a level without leaves keeps its grid and is skipped
    levels_.resize(L + 1);
    alive_.assign(L + 1, 0);
    for (int l = 0; l <= L; ++l)
    {
      if (mesh_.n_active_leaves(l) == 0)
        continue;
      alive_[l] = 1;
      if (!levels_[l])
      {
        adm_config c = mesh_.cfg;
        for (int d = 0; d < 3; ++d)
          c.n_cells[d] = (int32_t)mesh_.forest.n(l, d);
        for (int b = 0; b < c.n_sources; ++b)
          c.sources[b].segments = mesh_.segments[b].empty() ? nullptr : mesh_.segments[b].data();
        levels_[l] = std::make_unique<Thermal>(c, device_, lstream_[l]);
        levels_[l]->set_schedule(schedule_);
      }
      Thermal *th = levels_[l].get();
      int64_t const C = mesh_.forest.cells(l);
      std::vector<uint8_t> act(C), dom(C), mat(C), init(C);
      for (int64_t k = 0; k < mesh_.forest.n(l, 2); ++k)
        for (int64_t j = 0; j < mesh_.forest.n(l, 1); ++j)
          for (int64_t i = 0; i < mesh_.forest.n(l, 0); ++i)
          {
            int64_t const cell = mesh_.forest.index(l, i, j, k);
            int64_t const coarse = mesh_.forest.index(0, i >> l, j >> l, k >> l);
            dom[cell] = mesh_.coarse_active[coarse];
            act[cell] = mesh_.active_leaf(l, i, j, k) ? 1 : 0;
            mat[cell] = mesh_.coarse_mat[coarse];
            init[cell] = mesh_.coarse_init[coarse];
          }
      th->set_cells(act.data(), mat.data(), init.data(), nullptr, nullptr);
      th->set_domain(dom.data());
      th->setup();
      t_setup += lap_ms();
      if (old)
      {
        // the states of the active leaves only (CellDataTransfer)
        std::vector<int32_t> cells;
        std::vector<double> st;
        std::vector<uint8_t> melt(C, 0);
        for (int64_t k = 0; k < mesh_.forest.n(l, 2); ++k)
          for (int64_t j = 0; j < mesh_.forest.n(l, 1); ++j)
            for (int64_t i = 0; i < mesh_.forest.n(l, 0); ++i)
            {
              int64_t const cell = mesh_.forest.index(l, i, j, k);
              if (!act[cell])
                continue;
              double v[3] = {0, 0, 0};
              old->state_of(l, i, j, k, ns, v, &melt[cell]);
              cells.push_back((int32_t)cell);
              st.insert(st.end(), v, v + ns);
            }
        th->set_cell_state_sparse(cells.data(), st.data(), cells.size());
        th->get_state_from_material_properties();
        th->set_has_melted(melt.data());
        t_states += lap_ms();
      }
    }
    remesh_ms_[3] = t_setup;
    remesh_ms_[4] = t_states;
    lev_off_.assign(L + 1, 0);
    int64_t off = 0;
    for (int l = 0; l <= L; ++l)
      if (levels_[l])
      {
        lev_off_[l] = off;
        off += (int64_t)((levels_[l]->m() + 31) / 32 * 32);
      }
    lev_n_ = off;
    src_lev_.ensure(std::max<int64_t>(1, lev_n_));
    dst_lev_.ensure(std::max<int64_t>(1, lev_n_));
    ADM_CK(cudaMemsetAsync(src_lev_.p, 0, lev_n_ * sizeof(double), stream_));
    // prolongation rows (level nodes of active leaves) and their transpose
    std::vector<int64_t> row_pos, row_ptr{0};
    std::vector<int32_t> ent_dof;
    std::vector<double> ent_w;
    row_lev_.assign(L + 2, 0);
    std::vector<std::pair<int32_t, double>> ent;
    for (int l = 0; l <= L; ++l)
    {
      row_lev_[l] = (int64_t)row_pos.size();
      if (!alive(l))
        continue;
      Mesh const &lm = levels_[l]->mesh();
      // the level nodes of the active leaves, in ascending order: marked on
      // a byte map of the level grid, then collected by a scan that skips
      // empty 8-byte words
      size_t const n_lev = lm.n_nodes;
      node_mark_.assign(n_lev, 0);
      int const p = mesh_.p;
      for (int64_t k = 0; k < mesh_.forest.n(l, 2); ++k)
        for (int64_t j = 0; j < mesh_.forest.n(l, 1); ++j)
        {
          uint8_t const *lf = &mesh_.forest.leaf[l][mesh_.forest.index(l, 0, j, k)];
          for (int64_t i = 0; i < mesh_.forest.n(l, 0); ++i)
          {
            if (!lf[i] || !mesh_.in_domain(l, i, j, k))
              continue;
            for (int c = 0; c <= p; ++c)
              for (int b = 0; b <= p; ++b)
                for (int a = 0; a <= p; ++a)
                  node_mark_[(p * i + a) + (int64_t)lm.pitch * ((p * j + b) + (int64_t)lm.nn[1] * (p * k + c))] = 1;
          }
        }
      std::vector<int64_t> nodes;
      for (size_t q = 0; q < n_lev / 8; ++q)
      {
        uint64_t x = 0;
        std::memcpy(&x, node_mark_.data() + 8 * q, 8);
        if (!x)
          continue;
        for (int b = 0; b < 8; ++b)
          if (node_mark_[8 * q + b])
            nodes.push_back((int64_t)(8 * q + b));
      }
      for (size_t q = n_lev / 8 * 8; q < n_lev; ++q)
        if (node_mark_[q])
          nodes.push_back((int64_t)q);
      // the nodes' lattice keys ascend with their level positions (both
      // order by z, y, x), so the DoF keys are walked once alongside
      size_t at = 0;
      for (int64_t nidx : nodes)
      {
        int64_t const x = nidx % lm.pitch, y = (nidx / lm.pitch) % lm.nn[1], z = nidx / ((int64_t)lm.pitch * lm.nn[1]);
        int const s = mesh_.forest.max_level - l;
        int64_t const f = ((int64_t)2 << s) / mesh_.p;
        int64_t const key = mesh_.key(x * f, y * f, z * f);
        while (at < mesh_.dof_key.size() && mesh_.dof_key[at] < key)
          ++at;
        if (at < mesh_.dof_key.size() && mesh_.dof_key[at] == key)
        {
          ent.clear();
          ent.push_back({(int32_t)at, 1.0});
        }
        else
          mesh_.entries(key, ent);
        row_pos.push_back(lev_off_[l] + nidx);
        for (auto const &e : ent)
        {
          ent_dof.push_back(e.first);
          ent_w.push_back(e.second);
        }
        row_ptr.push_back((int64_t)ent_dof.size());
      }
    }
    row_lev_[L + 1] = (int64_t)row_pos.size();
    n_rows_ = (int64_t)row_pos.size();
    // transpose
    int64_t const nd = n_dofs();
    std::vector<int64_t> tptr(nd + 1, 0);
    for (int32_t d : ent_dof)
      ++tptr[d + 1];
    for (int64_t d = 0; d < nd; ++d)
      tptr[d + 1] += tptr[d];
    std::vector<int64_t> tpos(ent_dof.size()), fill(tptr.begin(), tptr.end() - 1);
    std::vector<double> tw(ent_dof.size());
    for (int64_t r = 0; r < n_rows_; ++r)
      for (int64_t e = row_ptr[r]; e < row_ptr[r + 1]; ++e)
      {
        int64_t const at = fill[ent_dof[e]]++;
        tpos[at] = row_pos[r];
        tw[at] = ent_w[e];
      }
    upload(row_pos_, row_pos);
    row_pos_h_ = row_pos;
    upload(row_ptr_, row_ptr);
    upload(ent_dof_, ent_dof);
    upload(ent_w_, ent_w);
    upload(tptr_, tptr);
    upload(tpos_, tpos);
    upload(tw_, tw);
    ADM_CK(cudaStreamSynchronize(stream_));
    remesh_lap(5);
  }

  template <class T> void upload(DevBuf<T> &buf, std::vector<T> const &v)
  {
    buf.ensure(std::max<size_t>(1, v.size()));
    if (!v.empty())
      ADM_CK(cudaMemcpyAsync(buf.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream_));
    // the host vectors die with the caller: finish the copies first
    ADM_CK(cudaStreamSynchronize(stream_));
  }

  void prolong(StageSum const &v)
  {
    if (n_rows_ == 0)
      return;
    prolong_kernel<<<blocks(n_rows_), 256, 0, stream_>>>(n_rows_, row_pos_.p, row_ptr_.p, ent_dof_.p, ent_w_.p, v,
                                                          src_lev_.p);
    ADM_CK(cudaGetLastError());
  }

  void prolong(double const *y)
  {
    StageSum v{};
    v.y = y;
    prolong(v);
  }

  void restrict_to(double *dst, int add, double const *scale = nullptr)
  {
    restrict_kernel<<<blocks(n_dofs()), 256, 0, stream_>>>(n_dofs(), tptr_.p, tpos_.p, tw_.p, dst_lev_.p, dst, add,
                                                            scale);
    ADM_CK(cudaGetLastError());
  }

  // compute_inverse_mass_matrix: 1 / (C^T sum_l M_l) with the lumped level
  // masses of the leaves (the composite vector has no constrained entries)
  void compute_inverse_mass()
  {
    inv_m_.ensure(std::max<int64_t>(1, n_dofs()));
    fork();
    for (size_t l = 0; l < levels_.size(); ++l)
      if (alive(l))
        levels_[l]->compute_inverse_mass_matrix();
    join();
    for (size_t l = 0; l < levels_.size(); ++l)
    {
      if (!alive(l))
        continue;
      int64_t const r0 = row_lev_[l], r1 = row_lev_[l + 1];
      if (r1 > r0)
        mass_from_inverse_kernel<<<blocks(r1 - r0), 256, 0, stream_>>>(r1 - r0, row_pos_.p + r0, lev_off_[l],
                                                                       levels_[l]->inverse_mass_matrix(),
                                                                       dst_lev_.p);
      ADM_CK(cudaGetLastError());
    }
    restrict_to(inv_m_.p, 0);
    invert_kernel<<<blocks(n_dofs()), 256, 0, stream_>>>(n_dofs(), inv_m_.p);
    ADM_CK(cudaGetLastError());
    ADM_CK(cudaStreamSynchronize(stream_));
  }

  int device_ = 0;
  cudaStream_t user_ = nullptr, stream_ = nullptr;
  cudaEvent_t ev_in_ = nullptr, ev_out_ = nullptr;
  cudaGraphExec_t step_exec_ = nullptr;
  cudaEvent_t ev_fork_ = nullptr;
  std::vector<cudaStream_t> lstream_;
  std::vector<cudaEvent_t> ev_lev_;
  double step_dt_ = 0.0;
  bool ready_ = false;
  AmrMesh mesh_;
  std::vector<std::unique_ptr<Thermal>> levels_;
  std::vector<uint8_t> alive_;
  std::vector<int64_t> row_pos_h_;
  std::vector<uint8_t> node_mark_; // level-grid byte map (prolongation rows)
  DevBuf<double> snap_rows_;       // the old field at the old rows (remesh snapshot)
  int schedule_ = Thermal::kScheduleAtomic;
  std::vector<int64_t> lev_off_, row_lev_;
  int64_t lev_n_ = 0, n_rows_ = 0;
  DevBuf<double> src_lev_, dst_lev_;
  DevBuf<int64_t> row_pos_, row_ptr_, tptr_, tpos_;
  DevBuf<int32_t> ent_dof_;
  DevBuf<double> ent_w_, tw_;
  DevBuf<double> y_, inv_m_, k_[4];
};

} // namespace adm

struct adm_amr_mesh
{
  adm::AmrMesh m;
};
struct adm_amr
{
  std::unique_ptr<adm::Amr> a;
};

namespace
{
std::vector<std::vector<uint8_t>> level_flags(adm::AmrMesh const &m, uint8_t const *flags)
{
  // flags: one byte per active leaf ... of every leaf, in leaf order
  std::vector<std::vector<uint8_t>> out(m.forest.max_level + 1);
  int64_t q = 0;
  for (int l = 0; l <= m.forest.max_level; ++l)
  {
    out[l].assign(m.forest.cells(l), 0);
    for (int64_t c = 0; c < m.forest.cells(l); ++c)
      if (m.forest.leaf[l][c])
        out[l][c] = flags ? flags[q++] : 0;
  }
  return out;
}

int64_t n_leaves(adm::AmrMesh const &m)
{
  int64_t n = 0;
  for (int l = 0; l <= m.forest.max_level; ++l)
    for (int64_t c = 0; c < m.forest.cells(l); ++c)
      n += m.forest.leaf[l][c];
  return n;
}

void leaves(adm::AmrMesh const &m, int32_t *out)
{
  int64_t q = 0;
  for (int l = 0; l <= m.forest.max_level; ++l)
    for (int64_t k = 0; k < m.forest.n(l, 2); ++k)
      for (int64_t j = 0; j < m.forest.n(l, 1); ++j)
        for (int64_t i = 0; i < m.forest.n(l, 0); ++i)
          if (m.forest.leaf[l][m.forest.index(l, i, j, k)])
          {
            out[4 * q + 0] = l;
            out[4 * q + 1] = (int32_t)i;
            out[4 * q + 2] = (int32_t)j;
            out[4 * q + 3] = (int32_t)k;
            ++q;
          }
}

void dof_lattice(adm::AmrMesh const &m, int64_t *xyz)
{
  for (size_t d = 0; d < m.dof_key.size(); ++d)
    m.unkey(m.dof_key[d], xyz + 3 * d);
}

void constraints(adm::AmrMesh const &m, int64_t *n_hanging, int64_t *n_entries, int64_t *xyz, int64_t *ptr,
                 int32_t *dof, double *w)
{
  std::vector<int64_t> keys;
  for (auto const &kv : m.hanging)
    keys.push_back(kv.first);
  std::sort(keys.begin(), keys.end());
  int64_t ne = 0;
  for (int64_t k : keys)
    ne += (int64_t)m.hanging.at(k).size();
  if (n_hanging)
    *n_hanging = (int64_t)keys.size();
  if (n_entries)
    *n_entries = ne;
  if (!xyz || !ptr || !dof || !w)
    return;
  int64_t e = 0;
  ptr[0] = 0;
  for (size_t h = 0; h < keys.size(); ++h)
  {
    m.unkey(keys[h], xyz + 3 * h);
    for (auto const &pe : m.hanging.at(keys[h]))
    {
      dof[e] = pe.first;
      w[e] = pe.second;
      ++e;
    }
    ptr[h + 1] = e;
  }
}
} // namespace

extern "C" {

// ------------------------------------------------------ host mesh entries
int adm_amr_mesh_create(adm_config const *cfg, int max_level, adm_amr_mesh **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(cfg && out, "null argument");
    auto h = std::make_unique<adm_amr_mesh>();
    h->m.init(*cfg, max_level);
    *out = h.release();
  });
}

int adm_amr_mesh_destroy(adm_amr_mesh *h)
{
  delete h;
  return ADM_OK;
}

int adm_amr_mesh_set_cells(adm_amr_mesh *h, uint8_t const *active, uint8_t const *material_id,
                           uint8_t const *initial_state)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->m.set_cells(active, material_id, initial_state);
  });
}

int adm_amr_mesh_refine_mesh(adm_amr_mesh *h, double time, double next_refinement_time, int n_time_steps,
                             int n_refinements, int coarsen_after_beam)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->m.refine_mesh(time, next_refinement_time, n_time_steps, n_refinements, coarsen_after_beam != 0);
    h->m.build();
  });
}

int adm_amr_mesh_execute(adm_amr_mesh *h, uint8_t const *refine, uint8_t const *coarsen)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->m.execute(level_flags(h->m, refine), level_flags(h->m, coarsen));
    h->m.build();
  });
}

int adm_amr_mesh_build(adm_amr_mesh *h)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->m.build();
  });
}

int adm_amr_mesh_n_leaves(adm_amr_mesh const *h, int64_t *n)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && n, "null argument");
    *n = n_leaves(h->m);
  });
}

int adm_amr_mesh_leaves(adm_amr_mesh const *h, int32_t *lijk)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && lijk, "null argument");
    leaves(h->m, lijk);
  });
}

int adm_amr_mesh_n_dofs(adm_amr_mesh const *h, int64_t *n_dofs, int64_t *n_nodes)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    if (n_dofs)
      *n_dofs = (int64_t)h->m.dof_key.size();
    if (n_nodes)
      *n_nodes = h->m.n_nodes_all;
  });
}

int adm_amr_mesh_dof_lattice(adm_amr_mesh const *h, int64_t *xyz)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && xyz, "null argument");
    dof_lattice(h->m, xyz);
  });
}

int adm_amr_mesh_constraints(adm_amr_mesh const *h, int64_t *n_hanging, int64_t *n_entries, int64_t *xyz,
                             int64_t *ptr, int32_t *dof, double *w)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    constraints(h->m, n_hanging, n_entries, xyz, ptr, dof, w);
  });
}

// ------------------------------------------------------------ GPU entries
int adm_amr_create(adm_config const *cfg, int max_level, int device, void *stream, adm_amr **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(cfg && out, "null argument");
    auto h = std::make_unique<adm_amr>();
    h->a = std::make_unique<adm::Amr>(*cfg, max_level, device, (cudaStream_t)stream);
    *out = h.release();
  });
}

int adm_amr_destroy(adm_amr *h)
{
  delete h;
  return ADM_OK;
}

int adm_amr_set_cells(adm_amr *h, uint8_t const *active, uint8_t const *material_id, uint8_t const *initial_state)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->a->mesh().set_cells(active, material_id, initial_state);
  });
}

int adm_amr_setup(adm_amr *h, double initial_temperature)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->a->setup(initial_temperature);
  });
}

int adm_amr_refine_mesh(adm_amr *h, double time, double next_refinement_time, int n_time_steps, int n_refinements,
                        int coarsen_after_beam)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->a->remesh([&] {
      h->a->mesh().refine_mesh(time, next_refinement_time, n_time_steps, n_refinements, coarsen_after_beam != 0);
    });
  });
}

int adm_amr_execute(adm_amr *h, uint8_t const *refine, uint8_t const *coarsen)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    auto r = level_flags(h->a->mesh(), refine);
    auto c = level_flags(h->a->mesh(), coarsen);
    h->a->remesh([&] { h->a->mesh().execute(r, c); });
  });
}

int adm_amr_remesh_profile(adm_amr const *h, double *ms)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && ms, "null argument");
    for (int i = 0; i < adm::kRemeshPhases; ++i)
      ms[i] = h->a->remesh_ms_[i];
  });
}

int adm_amr_n_dofs(adm_amr const *h, int64_t *n_dofs, int64_t *n_nodes)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    if (n_dofs)
      *n_dofs = (int64_t)h->a->mesh().dof_key.size();
    if (n_nodes)
      *n_nodes = h->a->mesh().n_nodes_all;
  });
}

int adm_amr_n_leaves(adm_amr const *h, int64_t *n)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && n, "null argument");
    *n = n_leaves(h->a->mesh());
  });
}

int adm_amr_leaves(adm_amr const *h, int32_t *lijk)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && lijk, "null argument");
    leaves(h->a->mesh(), lijk);
  });
}

int adm_amr_dof_lattice(adm_amr const *h, int64_t *xyz)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && xyz, "null argument");
    dof_lattice(h->a->mesh(), xyz);
  });
}

int adm_amr_solution(adm_amr *h, double **y)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && y, "null argument");
    h->a->require_ready();
    *y = h->a->solution();
  });
}

int adm_amr_get_solution(adm_amr *h, double *dst)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst, "null argument");
    h->a->copy_solution(dst, true);
  });
}

int adm_amr_set_solution(adm_amr *h, double const *src)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && src, "null argument");
    h->a->copy_solution(const_cast<double *>(src), false);
  });
}

int adm_amr_set_time(adm_amr *h, double t)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->a->require_ready();
    h->a->set_time(t);
  });
}

int adm_amr_vmult(adm_amr *h, double *dst, double const *src)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst && src, "null argument");
    h->a->vmult(dst, src);
  });
}

int adm_amr_inverse_mass(adm_amr *h, double *dst)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst, "null argument");
    h->a->require_ready();
    h->a->copy_inverse_mass(dst);
  });
}

int adm_amr_evolve_one_time_step(adm_amr *h, double t, double dt, double *t_out)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    double const tn = h->a->evolve_one_time_step(t, dt);
    if (t_out)
      *t_out = tn;
  });
}

int adm_amr_level_values(adm_amr *h, int level, double *host)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && host, "null argument");
    h->a->level_values(level, host);
  });
}

int adm_amr_level_cell_state(adm_amr *h, int level, double *host)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && host, "null argument");
    h->a->level_cell_state(level, host);
  });
}

int adm_amr_mark_has_melted(adm_amr *h, double threshold)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->a->mark_has_melted(threshold);
  });
}

int adm_amr_level_has_melted(adm_amr *h, int level, uint8_t *host)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && host, "null argument");
    h->a->level_has_melted(level, host);
  });
}

int adm_amr_level_layout(adm_amr *h, int level, int64_t nodes[3], int64_t *pitch)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && nodes && pitch, "null argument");
    adm::Thermal *th = h->a->level(level);
    ADM_REQUIRE(th, "no leaves on this level");
    for (int d = 0; d < 3; ++d)
      nodes[d] = th->mesh().nn[d];
    *pitch = th->mesh().pitch;
  });
}

int adm_amr_set_schedule(adm_amr *h, int schedule)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->a->set_schedule(schedule);
  });
}

int adm_amr_synchronize(adm_amr *h)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    h->a->synchronize();
  });
}

} // extern "C"
