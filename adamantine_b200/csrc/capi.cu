// extern "C" entry points of include/adamantine_b200.h over adm::Thermal.
// No C++ exception crosses the ABI: each call returns a status code and keeps
// the message for adm_last_error().
#include "capi_common.hpp"

#include <algorithm>

#include <string>

namespace
{
thread_local std::string g_last_error;

adm::Thermal *as(adm_thermal *h) { return reinterpret_cast<adm::Thermal *>(h); }
adm::Thermal const *as(adm_thermal const *h)
{
  return reinterpret_cast<adm::Thermal const *>(h);
}
} // namespace

namespace adm
{
// Records a failure message for adm_last_error() (also used by the entry
// points defined in other translation units).
void set_last_error(std::string const &msg) { g_last_error = msg; }
} // namespace adm

extern "C" {

const char *adm_last_error(void) { return g_last_error.c_str(); }

int adm_create(adm_config const *cfg, int device, void *stream, adm_thermal **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(cfg && out, "null argument");
    *out = nullptr;
    auto *t = new adm::Thermal(*cfg, device, reinterpret_cast<cudaStream_t>(stream));
    *out = reinterpret_cast<adm_thermal *>(t);
  });
}

int adm_destroy(adm_thermal *h)
{
  return adm::guard([&] { delete as(h); });
}

int adm_set_cells(adm_thermal *h, uint8_t const *active, uint8_t const *material_id,
                  uint8_t const *initial_state, double const *deposition_cos,
                  double const *deposition_sin)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->set_cells(active, material_id, initial_state, deposition_cos, deposition_sin);
  });
}

int adm_setup(adm_thermal *h)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->setup();
  });
}

int adm_n_nodes(adm_thermal const *h, int64_t *n)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && n, "null argument");
    *n = (int64_t)as(h)->m();
  });
}

int adm_n_cells(adm_thermal const *h, int64_t *n)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && n, "null argument");
    *n = (int64_t)as(h)->n_cells();
  });
}

int adm_get_active_cells(adm_thermal const *h, uint8_t *active)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && active, "null argument");
    auto const &a = as(h)->active_cells();
    std::copy(a.begin(), a.end(), active);
  });
}

int adm_node_layout(adm_thermal const *h, int64_t nodes[3], int64_t *pitch)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && nodes && pitch, "null argument");
    adm::Mesh const &m = as(h)->mesh();
    for (int d = 0; d < 3; ++d)
      nodes[d] = m.nn[d];
    *pitch = m.pitch;
  });
}

int adm_set_time(adm_thermal *h, double t)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->set_time(t);
  });
}

int adm_vmult(adm_thermal *h, double *dst, double const *src)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst && src, "null argument");
    ADM_REQUIRE(dst != src, "vmult needs distinct src and dst");
    as(h)->vmult(dst, src, false);
  });
}

int adm_vmult_add(adm_thermal *h, double *dst, double const *src)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst && src, "null argument");
    ADM_REQUIRE(dst != src, "vmult_add needs distinct src and dst");
    as(h)->vmult(dst, src, true);
  });
}

int adm_vmult_host(adm_thermal *h, double *dst_host, double const *src_host)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst_host && src_host, "null argument");
    as(h)->vmult_host(dst_host, src_host);
  });
}

int adm_compute_inverse_mass_matrix(adm_thermal *h)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->compute_inverse_mass_matrix();
  });
}

int adm_get_inverse_mass_matrix(adm_thermal *h, double *dst)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && dst, "null argument");
    adm::Thermal *t = as(h);
    ADM_CK(cudaMemcpyAsync(dst, t->inverse_mass_matrix(), t->m() * sizeof(double),
                           cudaMemcpyDeviceToDevice, t->stream()));
  });
}

int adm_evolve_one_time_step(adm_thermal *h, double t, double dt, double *solution,
                             double *t_out)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && solution, "null argument");
    double const tn = as(h)->evolve_one_time_step(t, dt, solution);
    if (t_out)
      *t_out = tn;
  });
}

int adm_evolve_one_time_step_host(adm_thermal *h, double t, double dt,
                                  double *solution_host, double *t_out)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && solution_host, "null argument");
    double const tn = as(h)->evolve_one_time_step_host(t, dt, solution_host);
    if (t_out)
      *t_out = tn;
  });
}

int adm_evolve_n_steps(adm_thermal *h, double t, double dt, int32_t n_steps,
                       double *solution, double *t_out)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && solution, "null argument");
    ADM_REQUIRE(n_steps >= 0, "n_steps must be non-negative");
    double const tn = as(h)->evolve_n_steps(t, dt, n_steps, solution);
    if (t_out)
      *t_out = tn;
  });
}

int adm_evaluate_material_properties(adm_thermal *h, double const *temperature,
                                     double *property_values)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && temperature && property_values, "null argument");
    as(h)->evaluate_material_properties(temperature, property_values);
  });
}

int adm_set_state_to_material_properties(adm_thermal *h)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->set_state_to_material_properties();
  });
}

int adm_get_state_from_material_properties(adm_thermal *h)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->get_state_from_material_properties();
  });
}

int adm_get_cell_state(adm_thermal *h, double *state_host)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && state_host, "null argument");
    as(h)->get_cell_state(state_host);
  });
}

int adm_set_cell_state(adm_thermal *h, double const *state_host)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && state_host, "null argument");
    as(h)->set_cell_state(state_host);
  });
}

int adm_get_qp_powder(adm_thermal *h, double *powder_host)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && powder_host, "null argument");
    as(h)->get_qp_powder(powder_host);
  });
}

int adm_mark_has_melted(adm_thermal *h, double threshold, double const *temperature,
                        uint8_t *has_melted_host)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && temperature, "null argument");
    as(h)->mark_has_melted(threshold, temperature, has_melted_host);
  });
}

int adm_activate_cells(adm_thermal *h, int64_t const *cells, int64_t n,
                       double new_temperature, double const *cos_new,
                       double const *sin_new, double *solution)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && solution && (n == 0 || cells), "null argument");
    ADM_REQUIRE(n >= 0, "negative cell count");
    as(h)->activate_cells(cells, n, new_temperature, cos_new, sin_new, solution);
  });
}

int adm_update_material(adm_thermal *h, adm_config const *cfg)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && cfg, "null argument");
    as(h)->update_material(*cfg);
  });
}

int adm_set_schedule(adm_thermal *h, int32_t schedule)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->set_schedule(schedule);
  });
}

int adm_get_schedule(adm_thermal const *h, int32_t *schedule)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && schedule, "null argument");
    *schedule = as(h)->schedule();
  });
}

int adm_set_cells_per_thread(adm_thermal *h, int32_t n)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->set_cells_per_thread(n);
  });
}

int adm_get_cells_per_thread(adm_thermal const *h, int32_t *n)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && n, "null argument");
    *n = as(h)->cells_per_thread();
  });
}

int adm_set_cells_per_block(adm_thermal *h, int32_t n)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->set_cells_per_block(n);
  });
}

int adm_get_cells_per_block(adm_thermal const *h, int32_t *n)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && n, "null argument");
    *n = as(h)->cells_per_block();
  });
}

int adm_autotune_schedules(adm_thermal *h, double const *field, int32_t *schedule, double *ms, int32_t n_ms)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && field, "null argument");
    ADM_REQUIRE(n_ms >= 0, "n_ms must not be negative");
    double t[ADM_N_SCHEDULES] = {0.0, 0.0, 0.0};
    int const c = as(h)->autotune(field, t);
    if (schedule)
      *schedule = c;
    for (int k = 0; ms && k < n_ms && k < ADM_N_SCHEDULES; ++k)
      ms[k] = t[k];
  });
}

int adm_autotune(adm_thermal *h, double const *field, int32_t *schedule, double *ms)
{
  return adm_autotune_schedules(h, field, schedule, ms, 2);
}

int adm_update_beam(adm_thermal *h, int32_t i, adm_source const *beam)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && beam, "null argument");
    as(h)->update_beam(i, *beam);
  });
}

int adm_device_error(adm_thermal *h, int32_t *code)
{
  return adm::guard([&] {
    ADM_REQUIRE(h && code, "null argument");
    *code = as(h)->device_error();
  });
}

int adm_synchronize(adm_thermal *h)
{
  return adm::guard([&] {
    ADM_REQUIRE(h, "null handle");
    as(h)->synchronize();
  });
}

} // extern "C"
