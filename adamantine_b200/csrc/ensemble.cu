// adm::Ensemble: batched time steps of many thermal problems sharing a mesh.
#include "ensemble.hpp"

#include <algorithm>
#include <cstring>

namespace adm
{

namespace
{
// Everything the batched launch takes from member 0 must be the same for all
// members.
void check_compatible(adm_config const &a, adm_config const &b)
{
  bool same = a.dim == b.dim && a.degree == b.degree && a.quadrature == b.quadrature &&
              a.n_states == b.n_states && a.use_table == b.use_table &&
              a.n_boundary_types == b.n_boundary_types && a.time_method == b.time_method &&
              a.n_sources == b.n_sources;
  for (int d = 0; d < 3 && same; ++d)
    same = a.n_cells[d] == b.n_cells[d] && a.origin[d] == b.origin[d] && a.extent[d] == b.extent[d];
  for (int i = 0; i < a.n_boundary_types && same; ++i)
    same = a.boundary_types[i] == b.boundary_types[i];
  for (int i = 0; i < a.n_sources && same; ++i)
    same = a.sources[i].type == b.sources[i].type;
  if (!same)
    throw Error(ADM_ERR_INVALID, "ensemble members must share the mesh, element, quadrature, material "
                                 "states, boundary types, time method and source kinds");
}
} // namespace

Ensemble::Ensemble(adm_config const *cfgs, int n_members, int device, cudaStream_t stream)
{
  if (!cfgs || n_members < 1)
    throw Error(ADM_ERR_INVALID, "an ensemble needs at least one member");
  if (n_members > (1 << 20))
    throw Error(ADM_ERR_INVALID, "too many ensemble members");
  for (int i = 1; i < n_members; ++i)
    check_compatible(cfgs[0], cfgs[i]);
  device_ = device;
  stream_ = stream;
  ADM_CK(cudaSetDevice(device_));
  members_.reserve(n_members);
  for (int i = 0; i < n_members; ++i)
    members_.emplace_back(new Thermal(cfgs[i], device, stream, false));
  Thermal const &m0 = *members_[0];
  stride_ = m0.m();
  deg_ = m0.mesh_.deg;
  ns_ = m0.ns_;
  tab_ = m0.tab_;
  any_source_ = cfgs[0].n_sources > 0;
  size_t const total = stride_ * (size_t)n_members;
  za_.alloc(total);
  zb_.alloc(total);
  acc_.alloc(total);
  // the two-pass schedule writes the accumulator at every node but the row
  // padding, which the streaming update reads
  ADM_CK(cudaMemset(acc_.p, 0, total * sizeof(double)));
  if (tab_.s > 1)
    s_.alloc(total);
  if (cfgs[0].time_method == 2)
    f0_.alloc(total);
  for (int i = 0; i < n_members; ++i)
  {
    size_t const off = stride_ * (size_t)i;
    members_[i]->bind_stage_vectors(za_.p + off, zb_.p + off, s_.p ? s_.p + off : nullptr,
                                    f0_.p ? f0_.p + off : nullptr, acc_.p + off);
  }
  md_d_.alloc(n_members);
}

Ensemble::~Ensemble()
{
  if (step_graph_)
    cudaGraphExecDestroy(step_graph_);
  cudaStreamSynchronize(stream_);
  if (graph_stream_)
  {
    cudaStreamSynchronize(graph_stream_);
    cudaStreamDestroy(graph_stream_);
    cudaEventDestroy(ev_a_);
    cudaEventDestroy(ev_b_);
  }
}

Thermal &Ensemble::member(int i)
{
  if (i < 0 || i >= n_members())
    throw Error(ADM_ERR_INVALID, "member index out of range");
  return *members_[i];
}

void Ensemble::set_cells(int i, uint8_t const *active, uint8_t const *material_id,
                         uint8_t const *initial_state, double const *cosv, double const *sinv)
{
  member(i).set_cells(active, material_id, initial_state, cosv, sinv);
  setup_done_ = false;
}

void Ensemble::drop_graph()
{
  if (step_graph_)
  {
    cudaGraphExecDestroy(step_graph_);
    step_graph_ = nullptr;
  }
}

void Ensemble::setup()
{
  ADM_CK(cudaSetDevice(device_));
  poly_p_ = 2;
  for (auto &m : members_)
  {
    m->setup();
    poly_p_ = std::max(poly_p_, m->poly_p_);
  }
  // colour-major, member-major within a colour: one launch per colour covers
  // the active tiles of every member
  work_.clear();
  for (int col = 0; col < 8; ++col)
  {
    colour_off_[col] = (int)work_.size();
    for (int i = 0; i < n_members(); ++i)
    {
      Thermal const &m = *members_[i];
      for (int k = m.colour_off_[col]; k < m.colour_off_[col + 1]; ++k)
        work_.push_back(TileWork{i, m.work_[k].tile, m.work_[k].xyz});
    }
  }
  colour_off_[8] = (int)work_.size();
  work_d_.alloc(std::max<size_t>(1, work_.size()));
  if (!work_.empty())
    ADM_CK(cudaMemcpyAsync(work_d_.p, work_.data(), work_.size() * sizeof(TileWork),
                           cudaMemcpyHostToDevice, stream_));
  // the atomic schedule's list: member-major, each member's tiles in order
  awork_.clear();
  for (int i = 0; i < n_members(); ++i)
    for (TileWork const &tw : members_[i]->awork_)
      awork_.push_back(TileWork{i, tw.tile, tw.xyz});
  awork_d_.alloc(std::max<size_t>(1, awork_.size()));
  if (!awork_.empty())
    ADM_CK(cudaMemcpyAsync(awork_d_.p, awork_.data(), awork_.size() * sizeof(TileWork),
                           cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  dirty_ = true;
  drop_graph();
  setup_done_ = true;
}

// Member table of the batched launch: each member's own data, with its
// solution at solutions + i * stride().
void Ensemble::bind(double *solutions)
{
  if ((reinterpret_cast<uintptr_t>(solutions) & 15u) != 0)
    throw Error(ADM_ERR_INVALID, "the solutions array must be 16-byte aligned");
  if (!dirty_ && bound_ == solutions)
    return;
  std::vector<MemberData> h(members_.size());
  for (size_t i = 0; i < members_.size(); ++i)
  {
    h[i] = members_[i]->md_;
    h[i].y = solutions + stride_ * i;
  }
  ADM_CK(cudaMemcpyAsync(md_d_.p, h.data(), h.size() * sizeof(MemberData), cudaMemcpyHostToDevice, stream_));
  ADM_CK(cudaStreamSynchronize(stream_));
  bound_ = solutions;
  dirty_ = false;
}

void Ensemble::set_clock(double t, double dt)
{
  int const n = n_members();
  launch_set_clock(md_d_.p, n, t, dt, stream_);
}

void Ensemble::launch_step(double *solutions)
{
  int const n = n_members();
  for (int i = 0; i < tab_.s; ++i)
  {
    // (the atomic schedule's zeroing launch prepares the beams itself)
    if (any_source_ && schedule_ != Thermal::kScheduleAtomic)
    {
      launch_stage_prepare(md_d_.p, n, tab_.c[i], stream_);
    }
    KernelArgs a = members_[0]->stage_args(i);
    a.members = md_d_.p;
    a.y_override = nullptr;
    double const *src = i == 0 ? solutions : (a.src_sel == 1 ? za_.p : zb_.p);
    CUtensorMap const map = brick_map(members_[0]->mesh_, src, n, stride_);
    if (schedule_ == Thermal::kScheduleTwoPass)
    {
      // every member's tiles in one launch (member-major runs per CTA), then
      // the gather pass over every member's nodes
      a.two_pass = 1;
      a.blocked = 1;
      if (!awork_.empty())
      {
        a.work = awork_d_.p;
        launch_tile(deg_, ns_, poly_p_, map, a, (int)awork_.size(), stream_);
        ADM_CK(cudaGetLastError());
      }
      launch_two_pass_gather(deg_, a, n, stream_);
      launch_stage_finalize(a, stride_, n, stream_);
      continue;
    }
    if (schedule_ == Thermal::kScheduleAtomic)
    {
      // member-major list, one contiguous run per CTA: a CTA changes member
      // (and reloads the material constants) at most once or twice
      a.atomic = 1;
      a.blocked = 1;
      launch_zero_keep(acc_.p, stride_ * (size_t)n, stream_, any_source_ ? md_d_.p : nullptr, n, tab_.c[i]);
      if (!awork_.empty())
      {
        a.work = awork_d_.p;
        launch_tile(deg_, ns_, poly_p_, map, a, (int)awork_.size(), stream_);
        ADM_CK(cudaGetLastError());
      }
      launch_stage_finalize(a, stride_, n, stream_);
      continue;
    }
    a.blocked = 1; // each colour's list is member-major
    for (int col = 0; col < 8; ++col)
    {
      int const count = colour_off_[col + 1] - colour_off_[col];
      if (count == 0)
        continue;
      a.work = work_d_.p + colour_off_[col];
      launch_tile(deg_, ns_, poly_p_, map, a, count, stream_);
      ADM_CK(cudaGetLastError());
    }
  }
}

double Ensemble::evolve_one_time_step(double t, double dt, double *solutions)
{
  NvtxRange const nvtx_range("adm::ensemble_step");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  ADM_CK(cudaSetDevice(device_));
  bind(solutions);
  set_clock(t, dt);
  launch_step(solutions);
  set_clock(t + tab_.c[tab_.s - 1] * dt, 0.0);
  return t + dt;
}

double Ensemble::evolve_looped(double t, double dt, double *solutions)
{
  NvtxRange const nvtx_range("adm::ensemble_looped");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  for (int i = 0; i < n_members(); ++i)
    members_[i]->evolve_one_time_step(t, dt, solutions + stride_ * i);
  return t + dt;
}

double Ensemble::evolve_n_steps(double t, double dt, int n, double *solutions)
{
  NvtxRange const nvtx_range("adm::ensemble_n_steps");
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  if (n <= 0)
    return t;
  ADM_CK(cudaSetDevice(device_));
  bind(solutions);
  if (!graph_stream_)
  {
    ADM_CK(cudaStreamCreateWithFlags(&graph_stream_, cudaStreamNonBlocking));
    ADM_CK(cudaEventCreateWithFlags(&ev_a_, cudaEventDisableTiming));
    ADM_CK(cudaEventCreateWithFlags(&ev_b_, cudaEventDisableTiming));
  }
  if (!step_graph_ || graph_solutions_ != solutions)
  {
    drop_graph();
    // the legacy default stream cannot be captured: capture on our own stream
    cudaStream_t const saved = stream_;
    stream_ = graph_stream_;
    cudaGraph_t graph;
    ADM_CK(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    try
    {
      launch_step(solutions);
      int const m = n_members();
      launch_advance_clock(md_d_.p, m, stream_);
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
    graph_solutions_ = solutions;
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
  set_clock((tt - dt) + tab_.c[tab_.s - 1] * dt, 0.0);
  return tt;
}

void Ensemble::update_material(int i, adm_config const &cfg)
{
  Thermal &m = *members_.at((size_t)i);
  m.update_material(cfg);
  if (m.poly_p_ > poly_p_)
  {
    poly_p_ = m.poly_p_;
    drop_graph();
  }
}

void Ensemble::update_beam(int i, int beam, adm_source const &src)
{
  members_.at((size_t)i)->update_beam(beam, src);
  dirty_ = true; // the member table holds a copy of the beam description
  drop_graph();
}

void Ensemble::set_cells_per_thread(int n)
{
  // the members validate n; the looped baseline runs the same kernel variant
  for (auto &m : members_)
    m->set_cells_per_thread(n);
  if (n != cells_per_thread_)
    drop_graph();
  cells_per_thread_ = n;
}

void Ensemble::set_schedule(int schedule)
{
  if (schedule != Thermal::kScheduleColoured && schedule != Thermal::kScheduleAtomic &&
      schedule != Thermal::kScheduleTwoPass)
    throw Error(ADM_ERR_INVALID, "unknown schedule");
  if (schedule != schedule_)
    drop_graph();
  schedule_ = schedule;
  // the looped baseline runs the members with the same schedule
  for (auto &m : members_)
    m->set_schedule(schedule);
}

// Times one batched step with each schedule on a copy of the solutions (the
// members' phase history and clocks restored afterwards) and keeps the faster.
int Ensemble::autotune(double const *solutions, double dt, double *ms_out)
{
  if (!setup_done_)
    throw Error(ADM_ERR_INVALID, "setup() has not been called");
  ADM_CK(cudaSetDevice(device_));
  size_t const total = stride_ * members_.size();
  DevBuf<double> scratch;
  scratch.alloc(total);
  std::vector<Thermal::PhaseSnapshot> snaps;
  for (auto &m : members_)
    snaps.push_back(m->save_phase());
  cudaEvent_t e0, e1;
  ADM_CK(cudaEventCreate(&e0));
  ADM_CK(cudaEventCreate(&e1));
  int const saved = schedule_, saved_cz = cells_per_thread_;
  double best = 0.0;
  int choice = saved, choice_cz = saved_cz;
  int const deg = members_.empty() ? 2 : members_[0]->mesh_.deg;
  // an untimed step of every variant first: the first launches of each
  // kernel and the clock ramp of an idle GPU would otherwise fall on the
  // first variant timed
  for (int sch : {Thermal::kScheduleColoured, Thermal::kScheduleAtomic, Thermal::kScheduleTwoPass})
    for (int cz : {1, 2, 4})
    {
      if (cz != 1 && deg != 1)
        continue;
      schedule_ = sch;
      set_cells_per_thread(cz);
      ADM_CK(cudaMemcpyAsync(scratch.p, solutions, total * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
      evolve_one_time_step(0.0, dt, scratch.p);
      for (size_t k = 0; k < members_.size(); ++k)
        members_[k]->restore_phase(snaps[k]);
    }
  for (int sch : {Thermal::kScheduleColoured, Thermal::kScheduleAtomic, Thermal::kScheduleTwoPass})
    for (int cz : {1, 2, 4})
  {
    if (cz != 1 && deg != 1)
      continue;
    schedule_ = sch;
    set_cells_per_thread(cz);
    ADM_CK(cudaMemcpyAsync(scratch.p, solutions, total * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    evolve_one_time_step(0.0, dt, scratch.p);
    int const reps = 3;
    ADM_CK(cudaEventRecord(e0, stream_));
    for (int r = 0; r < reps; ++r)
      evolve_one_time_step((r + 1) * dt, dt, scratch.p);
    ADM_CK(cudaEventRecord(e1, stream_));
    ADM_CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    ADM_CK(cudaEventElapsedTime(&ms, e0, e1));
    double const per = ms / reps;
    if (ms_out && (cz == 1 || per < ms_out[sch]))
      ms_out[sch] = per;
    if (best == 0.0 || per < best)
    {
      best = per;
      choice = sch;
      choice_cz = cz;
    }
    for (size_t k = 0; k < members_.size(); ++k)
      members_[k]->restore_phase(snaps[k]);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ADM_CK(cudaStreamSynchronize(stream_));
  schedule_ = saved;
  set_schedule(choice);
  set_cells_per_thread(choice_cz);
  return choice;
}

int32_t Ensemble::device_error()
{
  for (auto &m : members_)
  {
    int32_t const e = m->device_error();
    if (e)
      return e;
  }
  return 0;
}

void Ensemble::synchronize() { ADM_CK(cudaStreamSynchronize(stream_)); }

} // namespace adm

// ------------------------------------------------------------ C ABI
#include "capi_common.hpp"
#include "../../include/adamantine_b200_ensemble.h"

namespace
{
adm::Ensemble *as_ens(adm_ensemble *e) { return reinterpret_cast<adm::Ensemble *>(e); }
adm::Ensemble const *as_ens(adm_ensemble const *e) { return reinterpret_cast<adm::Ensemble const *>(e); }
} // namespace

extern "C" {

int adm_ensemble_create(adm_config const *cfgs, int32_t n_members, int device, void *stream,
                        adm_ensemble **out)
{
  return adm::guard([&] {
    ADM_REQUIRE(cfgs && out, "null argument");
    *out = nullptr;
    auto *e = new adm::Ensemble(cfgs, n_members, device, reinterpret_cast<cudaStream_t>(stream));
    *out = reinterpret_cast<adm_ensemble *>(e);
  });
}

int adm_ensemble_destroy(adm_ensemble *e)
{
  return adm::guard([&] { delete as_ens(e); });
}

int adm_ensemble_set_cells(adm_ensemble *e, int32_t member, uint8_t const *active,
                           uint8_t const *material_id, uint8_t const *initial_state,
                           double const *deposition_cos, double const *deposition_sin)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    as_ens(e)->set_cells(member, active, material_id, initial_state, deposition_cos, deposition_sin);
  });
}

int adm_ensemble_setup(adm_ensemble *e)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    as_ens(e)->setup();
  });
}

int adm_ensemble_stride(adm_ensemble const *e, int64_t *stride)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && stride, "null argument");
    *stride = (int64_t)as_ens(e)->stride();
  });
}

int adm_ensemble_n_work_items(adm_ensemble const *e, int64_t *n)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && n, "null argument");
    *n = (int64_t)as_ens(e)->n_work_items();
  });
}

int adm_ensemble_evolve_one_time_step(adm_ensemble *e, double t, double dt, double *solutions,
                                      double *t_out)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && solutions, "null argument");
    double const tn = as_ens(e)->evolve_one_time_step(t, dt, solutions);
    if (t_out)
      *t_out = tn;
  });
}

int adm_ensemble_evolve_looped(adm_ensemble *e, double t, double dt, double *solutions, double *t_out)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && solutions, "null argument");
    double const tn = as_ens(e)->evolve_looped(t, dt, solutions);
    if (t_out)
      *t_out = tn;
  });
}

int adm_ensemble_evolve_n_steps(adm_ensemble *e, double t, double dt, int32_t n_steps, double *solutions,
                                double *t_out)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && solutions, "null argument");
    ADM_REQUIRE(n_steps >= 0, "n_steps must be non-negative");
    double const tn = as_ens(e)->evolve_n_steps(t, dt, n_steps, solutions);
    if (t_out)
      *t_out = tn;
  });
}

int adm_ensemble_update_beam(adm_ensemble *e, int32_t member, int32_t i, adm_source const *beam)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && beam, "null argument");
    ADM_REQUIRE(member >= 0 && member < as_ens(e)->n_members(), "member index out of range");
    as_ens(e)->update_beam(member, i, *beam);
  });
}

int adm_ensemble_update_material(adm_ensemble *e, int32_t member, adm_config const *cfg)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && cfg, "null argument");
    ADM_REQUIRE(member >= 0 && member < as_ens(e)->n_members(), "member index out of range");
    as_ens(e)->update_material(member, *cfg);
  });
}

int adm_ensemble_get_cell_state(adm_ensemble *e, int32_t member, double *state_host)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && state_host, "null argument");
    as_ens(e)->member(member).get_cell_state(state_host);
  });
}

int adm_ensemble_get_inverse_mass_matrix(adm_ensemble *e, int32_t member, double *dst)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && dst, "null argument");
    adm::Thermal &t = as_ens(e)->member(member);
    ADM_CK(cudaMemcpyAsync(dst, t.inverse_mass_matrix(), t.m() * sizeof(double), cudaMemcpyDeviceToDevice,
                           t.stream()));
  });
}

int adm_ensemble_device_error(adm_ensemble *e, int32_t *code)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && code, "null argument");
    *code = as_ens(e)->device_error();
  });
}

int adm_ensemble_set_schedule(adm_ensemble *e, int32_t schedule)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    as_ens(e)->set_schedule(schedule);
  });
}

int adm_ensemble_set_cells_per_thread(adm_ensemble *e, int32_t n)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    as_ens(e)->set_cells_per_thread(n);
  });
}

int adm_ensemble_get_cells_per_thread(adm_ensemble const *e, int32_t *n)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && n, "null argument");
    *n = reinterpret_cast<adm::Ensemble const *>(e)->cells_per_thread();
  });
}

int adm_ensemble_autotune_schedules(adm_ensemble *e, double const *solutions, double dt, int32_t *schedule,
                                    double *ms, int32_t n_ms)
{
  return adm::guard([&] {
    ADM_REQUIRE(e && solutions, "null argument");
    ADM_REQUIRE(n_ms >= 0, "n_ms must not be negative");
    double t[ADM_N_SCHEDULES] = {0.0, 0.0, 0.0};
    int const c = as_ens(e)->autotune(solutions, dt, t);
    if (schedule)
      *schedule = c;
    for (int k = 0; ms && k < n_ms && k < ADM_N_SCHEDULES; ++k)
      ms[k] = t[k];
  });
}

int adm_ensemble_autotune(adm_ensemble *e, double const *solutions, double dt, int32_t *schedule, double *ms)
{
  return adm_ensemble_autotune_schedules(e, solutions, dt, schedule, ms, 2);
}

int adm_ensemble_synchronize(adm_ensemble *e)
{
  return adm::guard([&] {
    ADM_REQUIRE(e, "null handle");
    as_ens(e)->synchronize();
  });
}

} // extern "C"
