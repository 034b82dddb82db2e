/*
 * adamantine_b200.hpp -- header-only C++ adapter over the C ABI with the
 * method names of the reference's interfaces:
 *
 *   ThermalOperator  <-> ThermalOperatorBase<3, MemorySpace::Default>
 *                        (source/ThermalOperatorBase.hh:14-85)
 *   ThermalPhysics   <-> ThermalPhysicsInterface<3, MemorySpace::Default>
 *                        (source/ThermalPhysicsInterface.hh:28-189)
 *
 * deal.II is not part of this library, so the objects those interfaces pass
 * are replaced: DeviceVector stands for LA::distributed::Vector<double,
 * MemorySpace::Default> (a device array in the node layout of adm_node_layout),
 * adm_config for the property tree and the DoFHandler / quadrature set-up.
 * Failures throw adamantine_b200::Error (a std::runtime_error, as the
 * reference's ASSERT_THROW does, source/utils.hh:70-74) carrying the ABI's
 * status code and adm_last_error().
 *
 * Needs the CUDA runtime (cuda_runtime.h, -lcudart) for DeviceVector and
 * links against libadamantine_b200.so.
 */
#ifndef ADAMANTINE_B200_HPP
#define ADAMANTINE_B200_HPP

#include "adamantine_b200.h"

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace adamantine_b200
{

class Error : public std::runtime_error
{
public:
  Error(int code, std::string const &what) : std::runtime_error(what), code_(code) {}
  int code() const { return code_; }

private:
  int code_;
};

inline void check(int rc)
{
  if (rc != ADM_OK)
    throw Error(rc, adm_last_error());
}

inline void check_cuda(cudaError_t e, char const *what)
{
  if (e != cudaSuccess)
    throw Error(ADM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

/* A device vector of node values (FP64) in the library's node layout; owns
 * its cudaMalloc'ed storage. The stand-in for
 * LA::distributed::Vector<double, MemorySpace::Default>. */
class DeviceVector
{
public:
  DeviceVector() = default;
  explicit DeviceVector(std::size_t n) { reinit(n); }
  DeviceVector(DeviceVector const &) = delete;
  DeviceVector &operator=(DeviceVector const &) = delete;
  DeviceVector(DeviceVector &&o) noexcept : p_(o.p_), n_(o.n_)
  {
    o.p_ = nullptr;
    o.n_ = 0;
  }
  DeviceVector &operator=(DeviceVector &&o) noexcept
  {
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
    return *this;
  }
  ~DeviceVector()
  {
    if (p_)
      cudaFree(p_);
  }
  /* Vector::reinit: n entries, all zero. */
  void reinit(std::size_t n)
  {
    if (n != n_)
    {
      if (p_)
        cudaFree(p_);
      p_ = nullptr;
      n_ = 0;
      check_cuda(cudaMalloc(&p_, n * sizeof(double)), "cudaMalloc");
      n_ = n;
    }
    check_cuda(cudaMemset(p_, 0, n * sizeof(double)), "cudaMemset");
  }
  std::size_t size() const { return n_; }
  double *data() { return p_; }
  double const *data() const { return p_; }
  /* Copies from / to host memory (n entries). */
  void copy_from_host(double const *h)
  {
    check_cuda(cudaMemcpy(p_, h, n_ * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
  }
  void copy_to_host(double *h) const
  {
    check_cuda(cudaMemcpy(h, p_, n_ * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
  }
  std::vector<double> to_host() const
  {
    std::vector<double> h(n_);
    copy_to_host(h.data());
    return h;
  }

private:
  double *p_ = nullptr;
  std::size_t n_ = 0;
};

/* ThermalOperatorBase<3, MemorySpace::Default>
 * (source/ThermalOperatorBase.hh:14-85) over a handle: a view, owned by the
 * ThermalPhysics it belongs to (as the reference's ThermalPhysics owns its
 * operator, source/ThermalPhysics.hh:201). */
class ThermalOperator
{
public:
  explicit ThermalOperator(adm_thermal *h) : h_(h) {}

  /* m() / n(): length of a node vector (padding included). */
  std::size_t m() const
  {
    int64_t n = 0;
    check(adm_n_nodes(h_, &n));
    return static_cast<std::size_t>(n);
  }
  std::size_t n() const { return m(); }

  /* dst = A(src) (source/ThermalOperator.templates.hh:176-186). */
  void vmult(DeviceVector &dst, DeviceVector const &src) const
  {
    require_size(dst);
    require_size(src);
    check(adm_vmult(h_, dst.data(), src.data()));
  }
  /* dst += A(src) (source/ThermalOperator.templates.hh:188-225). */
  void vmult_add(DeviceVector &dst, DeviceVector const &src) const
  {
    require_size(dst);
    require_size(src);
    check(adm_vmult_add(h_, dst.data(), src.data()));
  }
  /* ThermalOperatorBase::Tvmult / Tvmult_add are not provided by the
   * reference's operator either (they assert); not offered here. */

  /* source/ThermalOperator.templates.hh:118-164. */
  void compute_inverse_mass_matrix() { check(adm_compute_inverse_mass_matrix(h_)); }
  /* The lumped inverse mass (the reference returns a shared_ptr to its
   * vector); a device copy, refreshed on every call. */
  DeviceVector const &get_inverse_mass_matrix() const
  {
    inv_mass_.reinit(m());
    check(adm_get_inverse_mass_matrix(h_, inv_mass_.data()));
    return inv_mass_;
  }
  /* initialize_dof_vector: a zero vector of the operator's layout. */
  void initialize_dof_vector(DeviceVector &v) const { v.reinit(m()); }
  /* source/ThermalOperator.templates.hh:753-884 and :886-895. */
  void get_state_from_material_properties() { check(adm_get_state_from_material_properties(h_)); }
  void set_state_to_material_properties() { check(adm_set_state_to_material_properties(h_)); }
  /* ThermalOperator::set_time (source/ThermalOperator.hh:296-308). */
  void set_time(double t) { check(adm_set_time(h_, t)); }

  adm_thermal *handle() const { return h_; }

private:
  void require_size(DeviceVector const &v) const
  {
    if (v.size() != m())
      throw Error(ADM_ERR_INVALID, "vector length " + std::to_string(v.size()) + " does not match m() = " +
                                       std::to_string(m()));
  }
  adm_thermal *h_;
  mutable DeviceVector inv_mass_;
};

/* Per-cell input of a problem (lexicographic cells, x fastest; empty arrays
 * take the defaults: cells below material_height active, material 0, the
 * geometry's initial state, no deposition rotation). */
struct CellData
{
  std::vector<uint8_t> active, material_id, initial_state;
  std::vector<double> deposition_cos, deposition_sin;
};

/* ThermalPhysicsInterface<3, MemorySpace::Default>
 * (source/ThermalPhysicsInterface.hh:28-189): owns the handle. */
class ThermalPhysics
{
public:
  /* The ThermalPhysics constructor (source/ThermalPhysics.templates.hh:346-494)
   * on `device`, enqueueing on `stream` (nullptr: the default stream). */
  ThermalPhysics(adm_config const &cfg, int device = 0, cudaStream_t stream = nullptr)
      : cfg_(cfg), h_(create(cfg_, device, stream)), op_(h_)
  {
  }
  ThermalPhysics(ThermalPhysics const &) = delete;
  ThermalPhysics &operator=(ThermalPhysics const &) = delete;
  ~ThermalPhysics()
  {
    if (h_)
      adm_destroy(h_);
  }

  void set_cells(CellData const &c)
  {
    auto u8 = [](std::vector<uint8_t> const &v) { return v.empty() ? nullptr : v.data(); };
    auto f64 = [](std::vector<double> const &v) { return v.empty() ? nullptr : v.data(); };
    check(adm_set_cells(h_, u8(c.active), u8(c.material_id), u8(c.initial_state), f64(c.deposition_cos),
                        f64(c.deposition_sin)));
  }
  /* setup (source/ThermalPhysics.templates.hh:496-506): setup_dofs, the
   * inverse mass and the state broadcast. setup_dofs alone has no separate
   * step here (the node layout is fixed by the mesh). */
  void setup() { check(adm_setup(h_)); }
  void setup_dofs() { setup(); }
  void compute_inverse_mass_matrix() { op_.compute_inverse_mass_matrix(); }

  /* evolve_one_time_step (source/ThermalPhysics.templates.hh:854-888):
   * returns t + dt. */
  double evolve_one_time_step(double t, double dt, DeviceVector &solution)
  {
    double out = 0.0;
    check(adm_evolve_one_time_step(h_, t, dt, solution.data(), &out));
    return out;
  }
  /* initialize_dof_vector(value, vector): every node set to value. */
  void initialize_dof_vector(double value, DeviceVector &v) const
  {
    v.reinit(op_.m());
    if (value != 0.0)
    {
      std::vector<double> h(v.size(), value);
      v.copy_from_host(h.data());
    }
  }
  /* add_material_start + add_material_end
   * (source/ThermalPhysics.templates.hh:595-825): cells become active, their
   * new nodes take new_temperature. */
  void add_material(std::vector<int64_t> const &cells, double new_temperature, DeviceVector &solution,
                    std::vector<double> const &cos_new = {}, std::vector<double> const &sin_new = {})
  {
    check(adm_activate_cells(h_, cells.data(), static_cast<int64_t>(cells.size()), new_temperature,
                             cos_new.empty() ? nullptr : cos_new.data(),
                             sin_new.empty() ? nullptr : sin_new.data(), solution.data()));
  }
  /* update_physics_parameters for heat source i
   * (source/ThermalPhysics.templates.hh:827-852). */
  void update_physics_parameters(int i, adm_source const &beam) { check(adm_update_beam(h_, i, &beam)); }
  /* get_state_from_material_properties / set_state_to_material_properties. */
  void get_state_from_material_properties() { op_.get_state_from_material_properties(); }
  void set_state_to_material_properties() { op_.set_state_to_material_properties(); }
  /* The cell state [n_states][n_cells] (MaterialProperty::get_state). */
  std::vector<double> get_state() const
  {
    int64_t c = 0;
    check(adm_n_cells(h_, &c));
    std::vector<double> s(static_cast<std::size_t>(cfg_.n_states * c));
    check(adm_get_cell_state(h_, s.data()));
    return s;
  }
  void set_state(std::vector<double> const &s) { check(adm_set_cell_state(h_, s.data())); }
  /* mark_has_melted (source/ThermalPhysics.templates.hh:537-593). */
  std::vector<uint8_t> mark_has_melted(double threshold, DeviceVector const &temperature)
  {
    int64_t c = 0;
    check(adm_n_cells(h_, &c));
    std::vector<uint8_t> out(static_cast<std::size_t>(c));
    check(adm_mark_has_melted(h_, threshold, temperature.data(), out.data()));
    return out;
  }
  /* save_checkpoint / load_checkpoint (source/ThermalPhysics.templates.hh
   * :974-1185); load returns the saved time. */
  void save_checkpoint(std::string const &path, double time, DeviceVector const &solution)
  {
    check(adm_save_checkpoint(h_, path.c_str(), time, solution.data()));
  }
  double load_checkpoint(std::string const &path, DeviceVector &solution, bool exact = false)
  {
    double t = 0.0;
    check(adm_load_checkpoint(h_, path.c_str(), exact ? 1 : 0, &t, solution.data()));
    return t;
  }
  unsigned int get_fe_degree() const { return static_cast<unsigned int>(cfg_.degree); }
  ThermalOperator &get_thermal_operator() { return op_; }
  /* Node grid extents (x, y, z) and row pitch of the vector layout. */
  void node_layout(int64_t nodes[3], int64_t &pitch) const { check(adm_node_layout(h_, nodes, &pitch)); }
  int32_t device_error() const
  {
    int32_t code = 0;
    check(adm_device_error(h_, &code));
    return code;
  }
  adm_thermal *handle() const { return h_; }

private:
  static adm_thermal *create(adm_config const &cfg, int device, cudaStream_t stream)
  {
    adm_thermal *h = nullptr;
    check(adm_create(&cfg, device, stream, &h));
    return h;
  }
  adm_config cfg_;
  adm_thermal *h_ = nullptr;
  ThermalOperator op_;
};

} // namespace adamantine_b200

#endif
