/*
 * adamantine_b200 -- C ABI of the B200-native thermal hot path.
 *
 * The library replaces, for one structured box mesh on one GPU, adamantine's
 * matrix-free heat operator (ThermalOperatorBase, source/ThermalOperatorBase.hh:14-85)
 * and its explicit time integration (ThermalPhysicsInterface,
 * source/ThermalPhysicsInterface.hh:28-189). Paths below are inside
 * adamantine v1.1.9.
 *
 * Conventions
 *  - Every call returns an int status (ADM_OK == 0); no C++ exception crosses
 *    the ABI. adm_last_error() gives the message of the last failure of the
 *    calling thread.
 *  - Vectors are FP64 on the device unless the name ends in _host. Their
 *    layout is the full-grid node numbering: node (i, j, k) of the
 *    (degree*nx+1) x (degree*ny+1) x (degree*nz+1) grid lives at
 *    i + pitch * (j + ny_nodes * k), with pitch >= degree*nx+1 (see
 *    adm_node_layout). Padding entries and nodes of inactive cells are not
 *    degrees of freedom: the operator writes 0 there and the time step leaves
 *    them unchanged.
 *  - Cell arrays are lexicographic over (x, y, z) cells, x fastest.
 *  - A handle enqueues all its work on one CUDA stream (the one passed to
 *    adm_create; NULL means the CUDA default stream) and is not thread-safe.
 *    _host variants and the state read-backs synchronize that stream.
 *  - Kernels report faults through a sticky device error word
 *    (adm_device_error) instead of trapping.
 */
#ifndef ADAMANTINE_B200_H
#define ADAMANTINE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ADM_OK 0
#define ADM_ERR_INVALID 1     /* bad argument or state */
#define ADM_ERR_CUDA 2        /* CUDA runtime error */
#define ADM_ERR_UNSUPPORTED 3 /* valid for the reference, not built here */
#define ADM_ERR_DEVICE 4      /* a kernel set the sticky error word */
#define ADM_ERR_ALLOC 5       /* device allocation failed */

/* Heat source (GoldakHeatSource / ElectronBeamHeatSource / CubeHeatSource,
 * source/BeamHeatSourceProperties.hh:55-66, source/CubeHeatSource.cc:14-43).
 * radius_squared is (diameter/2)^2. segments: n_segments x 5 doubles
 * (end_time, power_modifier, x, y, z) as built by ScanPath
 * (source/ScanPath.cc:58-195); host memory, copied by adm_create. */
typedef struct adm_source
{
  int32_t type; /* 0 goldak, 1 electron_beam, 2 cube */
  int32_t n_segments;
  double depth;
  double absorption_efficiency;
  double radius_squared;
  double max_power;
  double cube_start_time;
  double cube_end_time;
  double cube_value;
  double cube_min[3];
  double cube_max[3];
  const double *segments;
} adm_source;

/* Problem description: Geometry (source/Geometry.cc:186-262), MaterialProperty
 * tables (source/MaterialProperty.hh:359-383), Boundary
 * (source/Boundary.cc:12-70), heat sources and the time-stepping method
 * (source/ThermalPhysics.templates.hh:449-471). */
typedef struct adm_config
{
  int32_t dim;        /* must be 3 on the GPU */
  int32_t degree;     /* FE_Q degree: 1 or 2 */
  int32_t quadrature; /* 0 QGauss(degree+1), 1 QGaussLobatto(degree+1) */
  int32_t n_cells[3]; /* x (length), y (width), z (height) */
  double origin[3];
  double extent[3];
  int32_t n_materials; /* 1..4 */
  int32_t n_states;    /* 1 Solid, 2 SolidLiquid, 3 SolidLiquidPowder */
  int32_t use_table;   /* 0 polynomials, 1 12-point tables */
  int32_t p_order;     /* polynomial order, 0..4 */
  double poly[4][8][3][5];      /* [material][state property][state][coef] */
  double table[4][8][3][12][2]; /* [material][state property][state][i][T,v] */
  double props[4][5];  /* liquidus, solidus, latent heat, T_rad_inf, T_conv_inf */
  int32_t n_boundary_types;     /* 6 for a box: ids x-, x+, y-, y+, z-, z+ */
  int32_t boundary_types[8];    /* bits: 1 adiabatic, 2 radiative, 4 convective */
  int32_t n_sources;
  int32_t pad0;
  adm_source sources[4];
  int32_t time_method; /* 0 forward Euler, 1 RK2 midpoint, 2 RK3, 3 RK4 */
  int32_t n_threads;   /* unused on the GPU */
} adm_config;

typedef struct adm_thermal adm_thermal;

/* Message of the last failed call on this thread (never NULL). */
const char *adm_last_error(void);

/* ThermalPhysics constructor (source/ThermalPhysics.templates.hh:346-494).
 * stream: the cudaStream_t for all of the handle's work (NULL: default stream). */
int adm_create(adm_config const *cfg, int device, void *stream,
               adm_thermal **out);
/* ThermalPhysics / ThermalOperator destructors. */
int adm_destroy(adm_thermal *h);

/* Per-cell data (host arrays of n_cells entries, any may be NULL):
 * FE_Q/FE_Nothing activity (ThermalPhysics.templates.hh:472-493), material
 * id, initial state index (Geometry::assign_material_state,
 * source/Geometry.cc:317-353 -> MaterialProperty::set_initial_state,
 * source/MaterialProperty.templates.hh:755-794) and deposition cos/sin
 * (ThermalOperator::set_material_deposition_orientation,
 * source/ThermalOperator.templates.hh:897-940). */
int adm_set_cells(adm_thermal *h, uint8_t const *active,
                  uint8_t const *material_id, uint8_t const *initial_state,
                  double const *deposition_cos, double const *deposition_sin);
/* ThermalPhysics::setup (source/ThermalPhysics.templates.hh:496-506):
 * reinit, compute_inverse_mass_matrix, get_state_from_material_properties. */
int adm_setup(adm_thermal *h);

/* ThermalOperatorBase::m() / n(): length of a node vector (with padding). */
int adm_n_nodes(adm_thermal const *h, int64_t *n);
int adm_n_cells(adm_thermal const *h, int64_t *n);
/* The cells that currently carry material (FE_Q rather than FE_Nothing:
 * the initial set plus every activation), 1 byte per cell, lexicographic
 * (x fastest); host array of adm_n_cells bytes. */
int adm_get_active_cells(adm_thermal const *h, uint8_t *active);
/* Node grid extents (x, y, z) and the row pitch of the vector layout. */
int adm_node_layout(adm_thermal const *h, int64_t nodes[3], int64_t *pitch);

/* ThermalOperatorBase::set_time (source/ThermalOperator.hh:296-308). */
int adm_set_time(adm_thermal *h, double t);
/* ThermalOperatorBase::vmult (source/ThermalOperator.templates.hh:176-186):
 * dst = A(src), source term and face terms included, per-quadrature-point
 * phase state updated. Device pointers. */
int adm_vmult(adm_thermal *h, double *dst, double const *src);
/* ThermalOperatorBase::vmult_add (source/ThermalOperator.templates.hh:188-225). */
int adm_vmult_add(adm_thermal *h, double *dst, double const *src);
/* vmult on host buffers: copy in, apply, copy out, synchronize. With pinned
 * (page-locked) buffers the vector moves in z-slabs on two copy streams and
 * the tiles of each slab run as soon as their nodes have arrived (node sums
 * by atomics), so both copies and the kernel overlap; pageable buffers take
 * the plain path. */
int adm_vmult_host(adm_thermal *h, double *dst_host, double const *src_host);

/* ThermalOperatorBase::compute_inverse_mass_matrix
 * (source/ThermalOperator.templates.hh:118-164). */
int adm_compute_inverse_mass_matrix(adm_thermal *h);
/* ThermalOperatorBase::get_inverse_mass_matrix: copy into a device vector. */
int adm_get_inverse_mass_matrix(adm_thermal *h, double *dst);

/* ThermalPhysicsInterface::evolve_one_time_step
 * (source/ThermalPhysics.templates.hh:854-888): one forward-Euler or
 * Runge-Kutta step of dT/dt = M^-1 A(T) on a device vector; *t_out = t + dt. */
int adm_evolve_one_time_step(adm_thermal *h, double t, double dt,
                             double *solution, double *t_out);
/* The same step on a host vector (copy in, step, copy out). */
int adm_evolve_one_time_step_host(adm_thermal *h, double t, double dt,
                                  double *solution_host, double *t_out);
/* n_steps consecutive steps of size dt on a device vector; the steps are
 * captured once as a CUDA graph and replayed. */
int adm_evolve_n_steps(adm_thermal *h, double t, double dt, int32_t n_steps,
                       double *solution, double *t_out);

/* MaterialProperty::update (source/MaterialProperty.templates.hh:244-437):
 * cell-average temperature -> cell state and property values
 * [8][n_cells] (device pointers). */
int adm_evaluate_material_properties(adm_thermal *h, double const *temperature,
                                     double *property_values);
/* ThermalOperator::set_state_to_material_properties
 * (source/ThermalOperator.templates.hh:886-895): per-cell means of the
 * quadrature-point liquid/powder ratios. */
int adm_set_state_to_material_properties(adm_thermal *h);
/* ThermalOperator::get_state_from_material_properties
 * (source/ThermalOperator.templates.hh:753-884): broadcast the cell state to
 * the quadrature-point tables. */
int adm_get_state_from_material_properties(adm_thermal *h);
/* MaterialProperty::get_state / set_cell_state: [n_states][n_cells], host. */
int adm_get_cell_state(adm_thermal *h, double *state_host);
int adm_set_cell_state(adm_thermal *h, double const *state_host);
/* Quadrature-point powder ratios [n_cells][(degree+1)^3], host (diagnostic). */
int adm_get_qp_powder(adm_thermal *h, double *powder_host);

/* ThermalPhysics::mark_has_melted (source/ThermalPhysics.templates.hh:537-593):
 * updates and returns the per-cell indicator (host array, may be NULL). */
int adm_mark_has_melted(adm_thermal *h, double threshold,
                        double const *temperature, uint8_t *has_melted_host);

/* ThermalPhysics::add_material_start/end
 * (source/ThermalPhysics.templates.hh:595-825) without DoF renumbering:
 * cells (host array) become active, nodes that were not DoFs get
 * new_temperature in the device vector solution, cos/sin (host, n entries,
 * may be NULL) orient the new cells, the inverse mass is recomputed and the
 * state is averaged to cells and broadcast back. */
int adm_activate_cells(adm_thermal *h, int64_t const *cells, int64_t n,
                       double new_temperature, double const *cos_new,
                       double const *sin_new, double *solution);

/* ThermalPhysics::update_physics_parameters
 * (source/ThermalPhysics.templates.hh:827-852): new beam depth, efficiency,
 * radius and power for source i (segments are ignored). */
int adm_update_beam(adm_thermal *h, int32_t i, adm_source const *beam);

/* Launch schedule of operator applications and RK stages (no counterpart in
 * the reference): ADM_SCHEDULE_COLOURED (default) runs one launch per tile
 * colour, sums shared nodes in colour order and fuses the stage update --
 * bit reproducible; ADM_SCHEDULE_ATOMIC runs every tile in one launch, sums
 * shared nodes with FP64 atomics and updates in a separate pass -- rounding
 * order not reproducible run to run; ADM_SCHEDULE_TWO_PASS runs every tile
 * in one launch without atomics: each node's owner tile writes it (and
 * applies the stage update where no other tile touches it), partial sums of
 * nodes on a tile's upper faces go to a per-tile halo array, and a streaming
 * pass completes the shared nodes in a fixed order -- bit reproducible. */
#define ADM_SCHEDULE_COLOURED 0
#define ADM_SCHEDULE_ATOMIC 1
#define ADM_SCHEDULE_TWO_PASS 2
#define ADM_N_SCHEDULES 3
int adm_set_schedule(adm_thermal *h, int32_t schedule);
int adm_get_schedule(adm_thermal const *h, int32_t *schedule);
/* Cells per thread of the FE_Q(1) operator kernel (no counterpart in the
 * reference): 1 (default) or 2 cells stacked in z per thread, the second
 * sharing the per-tile bookkeeping and one node level in registers; or 4,
 * the column variant: one warp per tile, each thread walking its column of
 * 4 cells and writing each node level out as it completes, with no CTA
 * barrier. FE degree 2 takes 1 only. Results agree to rounding; each
 * variant is bit-reproducible in the coloured and two-pass schedules. */
int adm_set_cells_per_thread(adm_thermal *h, int32_t n);
int adm_get_cells_per_thread(adm_thermal const *h, int32_t *n);
/* Cells per block of the FE_Q(2) operator kernel (no counterpart in the
 * reference): 64 (default, one 8 x 4 x 2 tile per CTA of 192 threads, every
 * schedule) or 128 (a z-pair of tiles per CTA of 384 threads, one CTA per
 * SM, the atomic schedule; the other schedules keep 64). FE_Q(1) takes 128,
 * its tile. */
int adm_set_cells_per_block(adm_thermal *h, int32_t n);
int adm_get_cells_per_block(adm_thermal const *h, int32_t *n);
/* Autotuner: times every schedule and kernel variant (FE degree 1: cells per
 * thread; FE degree 2, atomic schedule: cells per block) on vmults of the
 * device field (the phase history is
 * restored afterwards), keeps the fastest in the handle and returns its
 * schedule in *schedule; ms[2] (may be NULL) receives the best per-vmult
 * times of the coloured and atomic schedules. */
int adm_autotune(adm_thermal *h, double const *field, int32_t *schedule, double *ms);
/* The same autotuner over every schedule; ms (may be NULL) receives up to
 * n_ms of the ADM_N_SCHEDULES best per-vmult times, indexed by schedule. */
int adm_autotune_schedules(adm_thermal *h, double const *field, int32_t *schedule, double *ms, int32_t n_ms);

/* ThermalPhysicsInterface::save_checkpoint
 * (source/ThermalPhysics.templates.hh:1062-1185): the cells' activity,
 * material ids, deposition directions, has_melted flags and state ratios,
 * the time and the device solution vector, plus the per-point phase history,
 * written to one file at path. */
int adm_save_checkpoint(adm_thermal *h, const char *path, double time, double const *solution);
/* ThermalPhysicsInterface::load_checkpoint (:974-1060) into a handle created
 * with the same mesh, element and material states: the cells are set up
 * again, the solution (device) and *time (may be NULL) are restored. exact = 0
 * broadcasts the saved cell states to the points, as the reference does;
 * exact = 1 restores the saved per-point history instead (the continued run
 * is then bit-identical to an uninterrupted one). */
int adm_load_checkpoint(adm_thermal *h, const char *path, int32_t exact, double *time, double *solution);

/* New material tables of the same shape (number of materials and states,
 * table or polynomial) for the handle: polynomial coefficients, tables and
 * the state-independent properties are taken from cfg, nothing else. No
 * counterpart in the reference (whose data assimilation changes beam
 * parameters only); used to perturb material parameters. */
int adm_update_material(adm_thermal *h, adm_config const *cfg);

/* Largest node vector (adm_n_nodes) that adm_vmult_host_static accepts. */
#define ADM_STATIC_SCRATCH_MAX_NODES 1310720

/* vmult on host buffers that allocates nothing (no counterpart in the
 * reference). For callers that hold their vectors in host memory and cannot
 * allocate device memory at the point of the call -- for example code that
 * runs while another part of the program is capturing a CUDA graph (a
 * cudaMalloc there breaks the capture) or a process whose device memory
 * budget is fixed up front. adm_vmult_host allocates its device staging
 * vectors on first use; this entry point stages src and dst in one static
 * device array of 2 x ADM_STATIC_SCRATCH_MAX_NODES doubles (20 MiB, held by
 * every GPU that loads the library until the process exits) and calls no
 * cudaMalloc or cudaFree. The first call on a device looks up that array's
 * device address; make that first call before any stream capture. Vectors
 * longer than the maximum are rejected with ADM_ERR_INVALID. The staged dst
 * is rewritten completely by every call (nodes no active cell touches are
 * cleared to zero). All calls on a device share the array, so calls that
 * overlap on the GPU (other threads, other streams) race; serialize them.
 * Synchronizes the handle's stream. */
int adm_vmult_host_static(adm_thermal *h, double *dst_host, double const *src_host);

/* Sticky device error word: 0 if no kernel reported a fault. Synchronizes. */
int adm_device_error(adm_thermal *h, int32_t *code);
/* Wait for the handle's stream. */
int adm_synchronize(adm_thermal *h);

#ifdef __cplusplus
}
#endif

#endif
