// Compiled test of the C++ adapter (include/adamantine_b200.hpp): the
// reference's ThermalOperatorBase / ThermalPhysicsInterface method names,
// driven from C++ over the C ABI, against the CPU oracle (oracle/) on the
// same problem -- a Q2 solid/liquid box with a Goldak beam and a convective
// + radiative top, 10 x 8 x 6 cells. Test infrastructure: prints OK and
// returns 0 when every check passes.
#include "adamantine_b200.hpp"
#include "thermal_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <random>
#include <vector>

namespace
{
int failures = 0;

void expect(bool ok, char const *what, double value)
{
  std::printf("%-48s %.3e %s\n", what, value, ok ? "ok" : "FAILED");
  if (!ok)
    ++failures;
}

double rel_max(std::vector<double> const &a, std::vector<double> const &b)
{
  double num = 0.0, den = 1e-300;
  for (std::size_t i = 0; i < a.size(); ++i)
  {
    num = std::max(num, std::fabs(a[i] - b[i]));
    den = std::max(den, std::fabs(b[i]));
  }
  return num / den;
}

adm_config problem(std::vector<double> &segments)
{
  adm_config c{};
  c.dim = 3;
  c.degree = 2;
  c.quadrature = 0;
  c.n_cells[0] = 10;
  c.n_cells[1] = 8;
  c.n_cells[2] = 6;
  c.extent[0] = 2.0e-3;
  c.extent[1] = 1.6e-3;
  c.extent[2] = 1.2e-3;
  c.n_materials = 1;
  c.n_states = 2;
  c.use_table = 0;
  c.p_order = 1;
  // [material][state property][state][coefficient]: density, specific heat,
  // k_x, k_y, k_z, emissivity, radiation coefficient (unused), convection
  // coefficient; states solid, liquid
  for (int s = 0; s < 2; ++s)
  {
    c.poly[0][0][s][0] = 7800.0;
    c.poly[0][0][s][1] = -0.1;
    c.poly[0][1][s][0] = 450.0;
    c.poly[0][1][s][1] = 0.2;
    for (int k = 2; k <= 4; ++k)
    {
      c.poly[0][k][s][0] = s == 0 ? 20.0 : 30.0;
      c.poly[0][k][s][1] = s == 0 ? 0.01 : 0.0;
    }
    c.poly[0][5][s][0] = 0.4;
    c.poly[0][5][s][1] = 1e-4;
    c.poly[0][7][s][0] = 10.0;
    c.poly[0][7][s][1] = 0.01;
  }
  c.props[0][0] = 1650.0; // liquidus
  c.props[0][1] = 1600.0; // solidus
  c.props[0][2] = 2.5e5;  // latent heat
  c.props[0][3] = 295.0;  // radiation temperature infinity
  c.props[0][4] = 300.0;  // convection temperature infinity
  c.n_boundary_types = 6;
  for (int f = 0; f < 6; ++f)
    c.boundary_types[f] = 1; // adiabatic
  c.boundary_types[5] = 2 | 4; // z+: radiative and convective
  c.n_sources = 1;
  adm_source &b = c.sources[0];
  b.type = 0; // Goldak
  b.depth = 2e-4;
  b.absorption_efficiency = 0.35;
  b.radius_squared = 2e-4 * 2e-4;
  b.max_power = 300.0;
  segments = {1e-9, 0.0, 0.4e-3, 0.8e-3, 1.2e-3, 1e-9 + 1.2e-3, 1.0, 1.6e-3, 0.8e-3, 1.2e-3};
  b.n_segments = 2;
  b.segments = segments.data();
  c.time_method = 3; // RK4
  return c;
}
} // namespace

int main()
{
  using namespace adamantine_b200;
  std::vector<double> segments;
  adm_config const cfg = problem(segments);
  int const C = cfg.n_cells[0] * cfg.n_cells[1] * cfg.n_cells[2];
  CellData cells;
  cells.active.assign(C, 1);
  cells.material_id.assign(C, 0);
  cells.initial_state.assign(C, 0);

  ThermalPhysics phys(cfg);
  phys.set_cells(cells);
  phys.setup();
  ThermalOperator &op = phys.get_thermal_operator();
  int64_t nodes[3], pitch = 0;
  phys.node_layout(nodes, pitch);
  std::size_t const n_plain = nodes[0] * nodes[1] * nodes[2];
  expect(op.m() == (std::size_t)(pitch * nodes[1] * nodes[2]) && op.n() == op.m(), "m() = n() = padded length",
         (double)op.m());
  expect(phys.get_fe_degree() == 2, "get_fe_degree()", phys.get_fe_degree());

  orc_oracle *o = orc_create(reinterpret_cast<orc_config const *>(&cfg));
  orc_set_cells(o, cells.active.data(), cells.material_id.data(), cells.initial_state.data(), nullptr, nullptr);
  orc_setup(o);

  // initial field: 300 K, a hot spot under the beam start crossing the
  // solidus and liquidus, +-1 K noise
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> noise(-1.0, 1.0);
  std::vector<double> T(n_plain);
  for (int64_t k = 0; k < nodes[2]; ++k)
    for (int64_t j = 0; j < nodes[1]; ++j)
      for (int64_t i = 0; i < nodes[0]; ++i)
      {
        double const x = cfg.extent[0] * i / (nodes[0] - 1), y = cfg.extent[1] * j / (nodes[1] - 1),
                     z = cfg.extent[2] * k / (nodes[2] - 1);
        double const r2 = (x - 0.8e-3) * (x - 0.8e-3) + (y - 0.8e-3) * (y - 0.8e-3) + (z - 1.2e-3) * (z - 1.2e-3);
        T[i + nodes[0] * (j + nodes[1] * k)] = 300.0 + 1700.0 * std::exp(-r2 / (0.4e-3 * 0.4e-3)) + noise(rng);
      }
  auto to_device = [&](std::vector<double> const &plain, DeviceVector &v) {
    std::vector<double> padded(op.m(), 0.0);
    for (int64_t r = 0; r < nodes[1] * nodes[2]; ++r)
      std::copy(plain.begin() + r * nodes[0], plain.begin() + (r + 1) * nodes[0], padded.begin() + r * pitch);
    v.copy_from_host(padded.data());
  };
  auto to_plain = [&](DeviceVector const &v) {
    std::vector<double> padded = v.to_host(), plain(n_plain);
    for (int64_t r = 0; r < nodes[1] * nodes[2]; ++r)
      std::copy(padded.begin() + r * pitch, padded.begin() + r * pitch + nodes[0], plain.begin() + r * nodes[0]);
    return plain;
  };

  // vmult (ThermalOperatorBase::vmult) at t = 2e-4
  DeviceVector src, dst;
  op.initialize_dof_vector(src);
  op.initialize_dof_vector(dst);
  to_device(T, src);
  op.set_time(2e-4);
  orc_set_time(o, 2e-4);
  op.vmult(dst, src);
  std::vector<double> ref(n_plain);
  orc_vmult(o, ref.data(), T.data());
  expect(rel_max(to_plain(dst), ref) <= 1e-12, "vmult vs oracle (<= 1e-12)", rel_max(to_plain(dst), ref));

  // vmult_add onto a seeded base vector
  std::vector<double> base(n_plain);
  for (double &v : base)
    v = noise(rng);
  to_device(base, dst);
  op.vmult_add(dst, src);
  std::vector<double> ref_add = base;
  orc_vmult_add(o, ref_add.data(), T.data());
  expect(rel_max(to_plain(dst), ref_add) <= 1e-12, "vmult_add vs oracle (<= 1e-12)", rel_max(to_plain(dst), ref_add));

  // the lumped inverse mass
  std::vector<double> im(n_plain);
  orc_inverse_mass(o, im.data());
  double const e_im = rel_max(to_plain(op.get_inverse_mass_matrix()), im);
  expect(e_im <= 1e-14, "get_inverse_mass_matrix vs oracle (<= 1e-14)", e_im);

  // ten RK4 steps (ThermalPhysicsInterface::evolve_one_time_step), fresh
  // problems so the phase history starts alike
  ThermalPhysics phys2(cfg);
  phys2.set_cells(cells);
  phys2.setup();
  orc_oracle *o2 = orc_create(reinterpret_cast<orc_config const *>(&cfg));
  orc_set_cells(o2, cells.active.data(), cells.material_id.data(), cells.initial_state.data(), nullptr, nullptr);
  orc_setup(o2);
  DeviceVector y;
  phys2.initialize_dof_vector(0.0, y);
  to_device(T, y);
  std::vector<double> yr = T;
  double t = 1e-5, tr = 1e-5;
  for (int s = 0; s < 10; ++s)
  {
    t = phys2.evolve_one_time_step(t, 2e-6, y);
    tr = orc_evolve_one_time_step(o2, tr, 2e-6, yr.data());
  }
  expect(t == tr, "evolve_one_time_step returns t + dt", t);
  double const e_y = rel_max(to_plain(y), yr);
  expect(e_y <= 1e-9, "10 RK4 steps vs oracle (<= 1e-9)", e_y);

  // the cell state after the steps (set_state_to_material_properties)
  phys2.set_state_to_material_properties();
  orc_set_state_to_material_properties(o2);
  std::vector<double> st = phys2.get_state(), sr(st.size());
  orc_get_cell_state(o2, sr.data());
  double e_s = 0.0;
  for (std::size_t i = 0; i < st.size(); ++i)
    e_s = std::max(e_s, std::fabs(st[i] - sr[i]));
  expect(e_s <= 1e-10, "cell state after the steps (<= 1e-10)", e_s);
  expect(phys.device_error() == 0 && phys2.device_error() == 0, "no device error", 0.0);

  // errors throw, as ASSERT_THROW does, with the ABI's status code
  bool threw = false;
  try
  {
    DeviceVector small(8);
    op.vmult(small, src);
  }
  catch (Error const &e)
  {
    threw = e.code() == ADM_ERR_INVALID;
  }
  expect(threw, "wrong vector length throws Error(ADM_ERR_INVALID)", 0.0);
  threw = false;
  try
  {
    adm_config bad = cfg;
    bad.degree = 5;
    ThermalPhysics nope(bad);
  }
  catch (Error const &e)
  {
    threw = e.code() == ADM_ERR_UNSUPPORTED;
  }
  expect(threw, "unsupported degree throws Error(ADM_ERR_UNSUPPORTED)", 0.0);

  orc_destroy(o);
  orc_destroy(o2);
  std::printf(failures == 0 ? "OK\n" : "%d FAILED\n", failures);
  return failures == 0 ? 0 : 1;
}
