// Host-side C++ layer of the B200 thermal hot path.
//
// adm::Thermal keeps the method names and meaning of the reference's
// ThermalOperatorBase (source/ThermalOperatorBase.hh:14-85) and
// ThermalPhysicsInterface (source/ThermalPhysicsInterface.hh:28-189) over
// project-owned data: a structured box mesh with a fixed full-grid node
// numbering, a per-cell active mask instead of FE_Nothing, device FP64
// vectors and the material/source tables of adm_config. All numerical work is
// done by the kernels of tile_kernel.cuh and aux_kernels.cuh; there is no CPU
// fallback.
#pragma once

#include "../../include/adamantine_b200.h"
#include "device_types.cuh"

#include <cuda.h>
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace adm
{

struct Error : std::runtime_error
{
  int code;
  Error(int c, std::string const &m) : std::runtime_error(m), code(c) {}
};

void check_cuda(cudaError_t e, char const *what, char const *file, int line);

// NVTX range for profilers (nsys / ncu timelines); free when no tool listens.
struct NvtxRange
{
  explicit NvtxRange(char const *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(NvtxRange const &) = delete;
  NvtxRange &operator=(NvtxRange const &) = delete;
};
#define ADM_CK(x) ::adm::check_cuda((x), #x, __FILE__, __LINE__)

template <class T>
struct DevBuf
{
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(DevBuf const &) = delete;
  DevBuf &operator=(DevBuf const &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n), cap(o.cap)
  {
    o.p = nullptr;
    o.n = 0;
    o.cap = 0;
  }
  DevBuf &operator=(DevBuf &&o) noexcept
  {
    if (this != &o)
    {
      release();
      p = o.p;
      n = o.n;
      cap = o.cap;
      o.p = nullptr;
      o.n = 0;
      o.cap = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release()
  {
    if (p)
      cudaFree(p);
    p = nullptr;
    n = 0;
    cap = 0;
  }
  void alloc(size_t count)
  {
    if (count == n && p)
      return;
    release();
    if (count == 0)
      return;
    cudaError_t e = cudaMalloc(&p, count * sizeof(T));
    if (e != cudaSuccess)
    {
      p = nullptr;
      (void)cudaGetLastError();
      throw Error(ADM_ERR_ALLOC, "cudaMalloc of " + std::to_string(count * sizeof(T)) +
                                     " bytes failed: " + cudaGetErrorString(e));
    }
    n = count;
    cap = count;
  }
  // count elements, reusing the allocation when it is large enough (buffers
  // whose size changes with every mesh change: no allocator call, with its
  // implicit device synchronization, once they have grown)
  void ensure(size_t count)
  {
    if (p && count <= cap)
    {
      n = count;
      return;
    }
    alloc(count + count / 4);
    n = count;
  }
  size_t cap = 0;
};

// 1D tables of one quadrature rule for FE_Q(deg) on Gauss-Lobatto nodes.
struct Rule1D
{
  int n = 0;
  double x[3] = {0, 0, 0}, w[3] = {0, 0, 0};
  double S[3][3] = {};   // S[q][i] = phi_i(x_q)
  double D[3][3] = {};   // collocation derivative at the points
  double G[3][3] = {};   // G[q][i] = phi_i'(x_q)
};

// Geometry and cell arrays shared by the single-problem and ensemble paths.
struct Mesh
{
  int deg = 1;
  int nc[3] = {0, 0, 0}, nn[3] = {0, 0, 0}, nt[3] = {0, 0, 0};
  int pitch = 0;
  double h[3] = {0, 0, 0}, origin[3] = {0, 0, 0};
  size_t n_nodes = 0, n_cells = 0, n_tiles = 0;
  int tx = 8, ty = 8, tz = 4;
  Rule1D quad, gauss;
  double glw[3] = {0, 0, 0};
  void init(adm_config const &cfg);
  size_t cell_index(int x, int y, int z) const
  {
    return x + (size_t)nc[0] * (y + (size_t)nc[1] * z);
  }
};

// Host mirror of one member's physics description.
MaterialDesc make_material(adm_config const &cfg);
void check_config(adm_config const &cfg);

// Per-cell info bits, tile masks and colour work lists for a set of members
// sharing one mesh.
struct CellTopology
{
  std::vector<uint32_t> cell_info;
  std::vector<uint32_t> tile_nbr;
  std::vector<uint8_t> tile_active;
  std::vector<int32_t> face_slot;
  int n_slots = 0;
  bool all_tiles_active = true;
};
// domain (optional, one byte per cell): the cells whose region carries
// material; a face of an active cell is a boundary face where the neighbour
// is outside the domain. Without it the domain is the active set. A level
// grid of a refined mesh passes the region of the whole material (its
// active cells are only the leaves of that level).
CellTopology build_topology(Mesh const &mesh, std::vector<uint8_t> const &active,
                            std::vector<uint8_t> const &matid, bool need_slots,
                            std::vector<uint8_t> const *domain = nullptr);

// Tensor map of n_members node vectors laid out member after member,
// member_stride doubles apart (1 member: one vector), for the 4D TMA brick
// loads of the tile kernel.
// tz_cells: cell layers per block (0: the degree's tile depth)
CUtensorMap brick_map(Mesh const &m, double const *base, int n_members, size_t member_stride, int tz_cells = 0);
// Tile kernel launch for one colour's work list.
void launch_tile(int deg, int ns, int p, CUtensorMap const &map, KernelArgs const &a, int n_items,
                 cudaStream_t stream);

// Per-member clock and heat-source-state kernels over a member table.
void launch_set_clock(MemberData *members, int n, double t, double dt, cudaStream_t stream);
void launch_advance_clock(MemberData *members, int n, cudaStream_t stream);
void launch_stage_prepare(MemberData *members, int n, double c, cudaStream_t stream);
// Per-Gauss-point powder ratios [C][NN] from the sparse powder history.
// Stage update of the atomic schedule for n_members members (a.members).
void launch_stage_finalize(KernelArgs const &a, size_t n_nodes, int n_members, cudaStream_t stream);
// Zeroes n doubles with the evict-last L2 policy (cudaMemsetAsync when p is
// not 16-byte aligned or n is odd).
// With members != nullptr the launch also prepares the beam states of
// n_members members for stage coefficient c (launch_stage_prepare).
void launch_zero_keep(double *p, size_t n, cudaStream_t stream, MemberData *members = nullptr, int n_members = 0,
                      double c = 0.0);
// two-pass schedule: the gather pass, and a tile's halo array length
void launch_two_pass_gather(int deg, KernelArgs const &a, int n_members, cudaStream_t stream);
size_t two_pass_halo_size(int deg);
// The per-point powder ratio [C][NN] from the sparse modes; cells with
// skip[c] == 0 are not written (skip may be null).
void launch_expand_powder(uint32_t const *cell_info, int NN, uint8_t const *pmode, double const *pcell,
                          double const *pq, double *out, size_t C, cudaStream_t stream,
                          uint8_t const *skip = nullptr);

class Ensemble;
class Adjoint;
struct Checkpoint;

// Material-deposition boxes on the device ([n][3] corners) with host copies
// of the directions (for the host fallback of the activation).
struct DeviceBoxes
{
  int64_t n = 0;
  double const *lo = nullptr, *hi = nullptr, *cosv = nullptr, *sinv = nullptr;
  std::vector<double> cos_host, sin_host;
};

class Thermal
{
public:
  // own_stage_vectors = false: the RK stage vectors and partial sums are
  // supplied by bind_stage_vectors (the ensemble keeps all members' vectors
  // in shared arrays).
  Thermal(adm_config const &cfg, int device, cudaStream_t stream, bool own_stage_vectors = true);
  ~Thermal();
  Thermal(Thermal const &) = delete;
  Thermal &operator=(Thermal const &) = delete;

  // ---- set-up (ThermalPhysics ctor / setup / reinit)
  void set_cells(uint8_t const *active, uint8_t const *material_id,
                 uint8_t const *initial_state, double const *cosv,
                 double const *sinv);
  void setup();
  // Level grid of a refined mesh: the cells whose region carries material
  // (faces towards them are interior); before setup().
  void set_domain(uint8_t const *domain);

  // ---- ThermalOperatorBase
  size_t m() const { return mesh_.n_nodes; }
  size_t n_cells() const { return mesh_.n_cells; }
  std::vector<uint8_t> const &active_cells() const { return active_; }
  Mesh const &mesh() const { return mesh_; }
  void set_time(double t);
  void vmult(double *dst, double const *src, bool add);
  // A time step driven from outside (refined meshes): set_step_clock(t, dt)
  // once, then vmult_stage(dst, src, c) evaluates dst = A src with the heat
  // sources at t + c dt (computed on the device, so the launches can be
  // captured in a graph and replayed with another clock).
  void set_step_clock(double t, double dt);
  void vmult_stage(double *dst, double const *src, double c);
  void compute_inverse_mass_matrix();
  double const *inverse_mass_matrix() const { return inv_mass_.p; }
  void get_state_from_material_properties();
  void set_state_to_material_properties();

  // ---- ThermalPhysicsInterface
  double evolve_one_time_step(double t, double dt, double *solution);
  double evolve_n_steps(double t, double dt, int n, double *solution);
  void evaluate_material_properties(double const *temperature, double *pv);
  void get_cell_state(double *host);
  void set_cell_state(double const *host);
  // the per-cell state of the listed cells (values [n][n_states]), every
  // other cell's state 0 (as set_cell_state with zeros there)
  void set_cell_state_sparse(int32_t const *cells, double const *values, size_t n);
  // the per-cell state of the listed cells into out [n][n_states] (host)
  void get_cell_state_sparse(int32_t const *cells, size_t n, double *out);
  void get_qp_powder(double *host);
  void mark_has_melted(double threshold, double const *temperature, uint8_t *host);
  // the has_melted flags per cell (host copy) and their replacement (a
  // refined mesh carries them through refinement)
  std::vector<uint8_t> const &has_melted_cells() const { return has_melted_; }
  void set_has_melted(uint8_t const *host);
  void activate_cells(int64_t const *cells, int64_t n, double new_temperature,
                      double const *cos_new, double const *sin_new, double *solution);
  void update_beam(int i, adm_source const &beam);
  // add_material_start/end for the inactive cells that boxes [b0, b1) meet,
  // found and activated on the device (append list, no renumbering);
  // returns the number of activated cells
  int64_t activate_in_boxes(DeviceBoxes const &boxes, int64_t b0, int64_t b1, double new_temperature,
                            double *solution);
  // new material tables of the same shape (ensemble analysis of a
  // material parameter); no counterpart in the reference
  void update_material(adm_config const &cfg);
  // host-buffer variants through persistent device staging vectors
  void vmult_host(double *dst_host, double const *src_host);
  double evolve_one_time_step_host(double t, double dt, double *solution_host);
  int32_t device_error();
  cudaStream_t stream() const { return stream_; }
  int device() const { return device_; }
  void synchronize();
  void bind_stage_vectors(double *za, double *zb, double *s, double *f0, double *acc);

  // Launch schedules of an operator application / RK stage: coloured (one
  // launch per tile colour, node sums by colour order, fused update; bit
  // reproducible) or atomic (one launch over every tile, node sums by
  // atomics, separate update pass; faster when a colour has fewer tiles than
  // the GPU holds CTAs, not bit reproducible run to run).
  static constexpr int kScheduleColoured = 0, kScheduleAtomic = 1, kScheduleTwoPass = 2;
  void set_schedule(int schedule);
  int schedule() const { return schedule_; }
  // FE_Q(1) operator kernel: 1, 2 (stacked in z) or 4 (the column variant)
  // cells per thread
  void set_cells_per_thread(int n);
  void build_atomic_list(std::vector<uint8_t> const &tile_active);
  int cells_per_thread() const { return cells_per_thread_; }
  // FE_Q(2) operator kernel: cells per block, 64 (one tile, every schedule)
  // or 128 (a z-pair of tiles, the atomic schedule)
  void set_cells_per_block(int n);
  int cells_per_block() const { return cells_per_block_ ? cells_per_block_ : mesh_.tx * mesh_.ty * mesh_.tz; }
  // times both schedules on vmults of `field` (phase history restored) and
  // keeps the faster; ms_out[2] (may be null) receives the per-vmult times
  int autotune(double const *field, double *ms_out);

  // device copy of the phase history (powder, face powder, liquid sums) and
  // the clock, to run trial steps without changing the state
  struct PhaseSnapshot
  {
    DevBuf<uint8_t> mode;
    DevBuf<double> cell, q, face, liquid, clock;
  };
  PhaseSnapshot save_phase() const;
  void restore_phase(PhaseSnapshot const &p);

  // stage schedule (Butcher tableau of the configured method)
  struct Tableau
  {
    int s;
    double a[4][4], b[4], c[4];
  };
  static Tableau tableau(int method);

private:
  friend class Ensemble;
  friend class Adjoint;
  friend struct Checkpoint;
  friend class Microstructure;
  friend class Mechanics;
  void rebuild();
  void upload_member();
  KernelArgs base_args() const;
  KernelArgs stage_args(int i) const;
  void launch_pass(KernelArgs args, double const *src);
  void launch_step(double *solution);
  void prepare_stage(double c);
  void set_clock(double t, double dt);

  adm_config cfg_;
  std::vector<std::vector<double>> segments_;
  Mesh mesh_;
  int ns_ = 1;
  int poly_p_ = 2;
  int device_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaStream_t graph_stream_ = nullptr; // capture/replay stream of evolve_n_steps
  cudaEvent_t ev_a_ = nullptr, ev_b_ = nullptr;
  bool adiabatic_only_ = true;
  bool has_rotation_ = false;
  bool setup_done_ = false;
  double op_time_ = 0.0;
  int schedule_ = kScheduleColoured;
  int cells_per_thread_ = 1;
  int cells_per_block_ = 0; // 0: the tile (FE_Q(2): 64 cells)
  Tableau tab_;

  std::vector<uint8_t> active_, matid_, init_state_, has_melted_;
  std::vector<uint8_t> domain_; // empty: the active cells
  std::vector<double> cos_, sin_;
  CellTopology topo_;
  std::vector<TileWork> work_;
  int colour_off_[9] = {0};

  DevBuf<double> za_, zb_, s_, f0_, acc_, inv_mass_;
  // the stage vectors in use: za_ .. acc_ or the bound external ones
  double *za_p_ = nullptr, *zb_p_ = nullptr, *s_p_ = nullptr, *f0_p_ = nullptr, *acc_p_ = nullptr;
  DevBuf<double> stage_in_, stage_out_;
  DevBuf<double> powder_cell_, powder_q_, liquid_sum_, face_powder_;
  DevBuf<double> cos_d_, sin_d_, state_d_, clock_, segs_;
  DevBuf<uint32_t> cell_info_d_, tile_nbr_d_;
  DevBuf<uint8_t> powder_mode_, has_melted_d_;
  DevBuf<int32_t> face_slot_d_, error_d_;
  DevBuf<int32_t> claim_d_; // per-colour work counters of the tile launches (dynamic claiming)
  // stage coefficient whose beam preparation the atomic schedule's zeroing
  // launch does (negative: none pending)
  double fold_prepare_c_ = -1.0;
  DevBuf<double> halo_d_;   // two-pass schedule: per-tile upper-face partial sums
  DevBuf<int64_t> cells_d_;
  // deposition: per-cell mark, append list, material ids
  DevBuf<int32_t> last_box_d_, list_box_d_;
  DevBuf<int64_t> list_d_;
  DevBuf<unsigned long long> count_d_;
  DevBuf<uint8_t> matid_d_;
  // set-up and state-transfer scratch (grow-only: no allocator call per
  // mesh change once grown)
  DevBuf<uint8_t> scratch_u8_;
  DevBuf<int32_t> scratch_i32_;
  DevBuf<double> scratch_f64_;
  DevBuf<MaterialDesc> mat_d_;
  DevBuf<BeamState> beam_state_d_;
  DevBuf<MemberData> member_d_;
  DevBuf<TileWork> work_d_;
  std::vector<TileWork> awork_;  // atomic schedule: every active tile, bottom layers first
  DevBuf<TileWork> awork_d_;
  MemberData md_{};

  // z-slab pipeline of vmult_host: tiles sorted by z layer, copy streams
  static constexpr int kPipeChunks = 8;
  std::vector<TileWork> zwork_;
  DevBuf<TileWork> zwork_d_;
  uint64_t work_version_ = 0, zwork_version_ = ~0ull;
  // 128-cell blocks: z-pairs of tiles with an active tile, bottom first
  std::vector<TileWork> pwork_;
  DevBuf<TileWork> pwork_d_;
  uint64_t pwork_version_ = ~0ull;
  void build_pair_list();
  cudaStream_t copy_in_ = nullptr, copy_out_ = nullptr;
  cudaEvent_t pipe_ev_[2 * kPipeChunks + 2] = {};

  // captured step graph for evolve_n_steps
  cudaGraphExec_t step_graph_ = nullptr;
  double *graph_solution_ = nullptr;
};

} // namespace adm
