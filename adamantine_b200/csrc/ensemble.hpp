// Batched ensemble of thermal problems on one mesh (one GPU).
//
// The reference advances its EnKF ensemble as a loop over independent
// ThermalPhysics objects (application/adamantine.hh:2137-2142). Here every
// member keeps its own physics (material tables, beam parameters, active
// cells, phase history, inverse mass) in an adm::Thermal, but the members'
// node vectors live in shared arrays, member after member, stride() doubles
// apart, and one launch per colour advances the ragged (member, tile) work
// list of all members together.
#pragma once

#include "thermal.hpp"

#include <memory>
#include <vector>

namespace adm
{

class Ensemble
{
public:
  // cfgs: one configuration per member; they must agree on the mesh, the
  // element, the quadrature, the number of material states, the table /
  // polynomial choice, the boundary types, the time-stepping method and the
  // number and kind of heat sources (the values may differ).
  Ensemble(adm_config const *cfgs, int n_members, int device, cudaStream_t stream);
  ~Ensemble();
  Ensemble(Ensemble const &) = delete;
  Ensemble &operator=(Ensemble const &) = delete;

  int n_members() const { return (int)members_.size(); }
  // doubles between two members' node vectors (= one member's m())
  size_t stride() const { return stride_; }
  Thermal &member(int i);
  // Thermal::set_cells of member i (setup() must follow)
  void set_cells(int i, uint8_t const *active, uint8_t const *material_id,
                 uint8_t const *initial_state, double const *cosv, double const *sinv);
  // every member's setup, then the batched work list
  void setup();
  // one RK step of every member in one launch per colour and stage
  double evolve_one_time_step(double t, double dt, double *solutions);
  // the same step as a loop over members, each through its own
  // single-member launches (the reference's ensemble loop)
  double evolve_looped(double t, double dt, double *solutions);
  // n batched steps replayed from one captured CUDA graph
  double evolve_n_steps(double t, double dt, int n, double *solutions);
  // a member's material or beam changed (after an analysis step)
  void update_material(int i, adm_config const &cfg);
  void update_beam(int i, int beam, adm_source const &src);
  // launch schedule of the batched stages (Thermal::kSchedule*) and its
  // autotuner (one timed batched step per schedule on a copy of solutions)
  void set_schedule(int schedule);
  int schedule() const { return schedule_; }
  // FE_Q(1) operator kernel: 1 or 2 cells per thread (members follow)
  void set_cells_per_thread(int n);
  int cells_per_thread() const { return cells_per_thread_; }
  int autotune(double const *solutions, double dt, double *ms_out);
  int32_t device_error();
  size_t n_work_items() const { return work_.size(); }
  cudaStream_t stream() const { return stream_; }
  void synchronize();

private:
  void bind(double *solutions);
  void launch_step(double *solutions);
  void set_clock(double t, double dt);
  void drop_graph();

  std::vector<std::unique_ptr<Thermal>> members_;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  size_t stride_ = 0;
  int deg_ = 1, ns_ = 1, poly_p_ = 2;
  bool any_source_ = false;
  int schedule_ = Thermal::kScheduleColoured;
  int cells_per_thread_ = 1;
  bool setup_done_ = false;
  Thermal::Tableau tab_;

  DevBuf<double> za_, zb_, s_, f0_, acc_;
  DevBuf<MemberData> md_d_;
  DevBuf<TileWork> work_d_, awork_d_;
  std::vector<TileWork> work_, awork_;
  int colour_off_[9] = {0};
  double *bound_ = nullptr; // solutions array the member table points at
  bool dirty_ = true;       // member table must be re-uploaded

  cudaStream_t graph_stream_ = nullptr;
  cudaEvent_t ev_a_ = nullptr, ev_b_ = nullptr;
  cudaGraphExec_t step_graph_ = nullptr;
  double *graph_solutions_ = nullptr;
};

} // namespace adm
