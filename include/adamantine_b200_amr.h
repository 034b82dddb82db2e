/*
 * adamantine_b200 -- refined meshes of the thermal path (C ABI).
 *
 * A forest of octrees over the configuration's coarse box mesh (level 0),
 * refined along the beams' paths as refine_mesh does
 * (application/adamantine.hh:540-681), balanced 2:1 across faces and edges,
 * with the hanging-node constraints of make_hanging_node_constraints
 * (application/adamantine.hh:514-523) and the constrained operator
 * (ThermalOperator::vmult_add, source/ThermalOperator.templates.hh:205-224),
 * inverse mass (:140-160) and refine_and_transfer
 * (application/adamantine.hh:312-539).
 *
 * FE degree 1 or 2; max_level (0..6) bounds the refinement level. The
 * material region is the set of active coarse cells (no activation on a
 * refined mesh). Composite vectors hold the non-hanging nodes ("DoFs"),
 * ordered by their lattice coordinates (z, then y, then x): node positions
 * are integer coordinates on the vertex lattice of level max_level + 1,
 * whose spacing is the coarse cell size / 2^(max_level + 1) along each
 * axis. A hanging node (a node of a fine cell inside a face or edge of a
 * coarser active neighbour, and not one of its nodes) takes the coarse
 * cell's interpolant, read through the constraints on every application
 * and distributed back with the transposed weights.
 *
 * Leaves are listed level by level, cells of a level lexicographic (x
 * fastest), as (level, i, j, k) with i, j, k the cell's indices on the
 * level grid (the coarse mesh refined 2^level times). Per-leaf flag arrays
 * (refine / coarsen) follow the same order.
 */
#ifndef ADAMANTINE_B200_AMR_H
#define ADAMANTINE_B200_AMR_H

#include "adamantine_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- mesh logic on the host (no GPU) */
typedef struct adm_amr_mesh adm_amr_mesh;

/* Uniform level-0 mesh of cfg (its geometry, degree and heat sources). */
int adm_amr_mesh_create(adm_config const *cfg, int max_level, adm_amr_mesh **out);
int adm_amr_mesh_destroy(adm_amr_mesh *h);
/* Coarse-cell data (adm_set_cells meaning; NULL: all active, material 0,
 * state 0). */
int adm_amr_mesh_set_cells(adm_amr_mesh *h, uint8_t const *active, uint8_t const *material_id,
                           uint8_t const *initial_state);
/* refine_mesh (application/adamantine.hh:608-681) with the heat sources of
 * cfg: n_refinements rounds; each flags the leaves whose bounding box meets
 * a beam box (HeatSource::get_bounding_box, scaling 2) at the times
 * time + i (next_refinement_time - time) / n_time_steps, i < n_time_steps,
 * for refinement below level n_refinements, and, with coarsen_after_beam,
 * every other leaf above level 0 for coarsening. Execution: refinement,
 * then coarsening of the families whose eight children are all flagged
 * leaves and whose coarsening keeps the 2:1 balance, then balancing. Ends
 * with adm_amr_mesh_build. */
int adm_amr_mesh_refine_mesh(adm_amr_mesh *h, double time, double next_refinement_time, int n_time_steps,
                             int n_refinements, int coarsen_after_beam);
/* Execute explicit per-leaf flags (one byte per leaf, NULL: none) as
 * above, then adm_amr_mesh_build. */
int adm_amr_mesh_execute(adm_amr_mesh *h, uint8_t const *refine, uint8_t const *coarsen);
/* DoFs and constraints of the current leaves (after set_cells). */
int adm_amr_mesh_build(adm_amr_mesh *h);
int adm_amr_mesh_n_leaves(adm_amr_mesh const *h, int64_t *n);
/* 4 int32 per leaf: level, i, j, k. */
int adm_amr_mesh_leaves(adm_amr_mesh const *h, int32_t *lijk);
/* n_dofs: non-hanging nodes; n_nodes: all distinct nodes of active leaves. */
int adm_amr_mesh_n_dofs(adm_amr_mesh const *h, int64_t *n_dofs, int64_t *n_nodes);
/* 3 int64 lattice coordinates per DoF (x, y, z). */
int adm_amr_mesh_dof_lattice(adm_amr_mesh const *h, int64_t *xyz);
/* Hanging nodes, sorted like DoFs: their lattice coordinates (3 each) and
 * constraint rows in CSR form (ptr: n_hanging + 1; dof, w: n_entries), the
 * masters' DoF indices and weights. With xyz / ptr / dof / w NULL only the
 * counts are returned. */
int adm_amr_mesh_constraints(adm_amr_mesh const *h, int64_t *n_hanging, int64_t *n_entries, int64_t *xyz,
                             int64_t *ptr, int32_t *dof, double *w);

/* ---- the refined thermal problem on the GPU */
typedef struct adm_amr adm_amr;

/* ThermalPhysics on a refined mesh; stream as for adm_create. */
int adm_amr_create(adm_config const *cfg, int max_level, int device, void *stream, adm_amr **out);
int adm_amr_destroy(adm_amr *h);
int adm_amr_set_cells(adm_amr *h, uint8_t const *active, uint8_t const *material_id, uint8_t const *initial_state);
/* Level-0 mesh, level grids, inverse mass; the solution (owned by the
 * handle) set to initial_temperature. */
int adm_amr_setup(adm_amr *h, double initial_temperature);
/* refine_mesh + refine_and_transfer: the solution is interpolated onto the
 * new nodes, cell states carried to children / from first children, the
 * inverse mass recomputed. */
int adm_amr_refine_mesh(adm_amr *h, double time, double next_refinement_time, int n_time_steps, int n_refinements,
                        int coarsen_after_beam);
int adm_amr_execute(adm_amr *h, uint8_t const *refine, uint8_t const *coarsen);
int adm_amr_n_dofs(adm_amr const *h, int64_t *n_dofs, int64_t *n_nodes);
/* Host wall time (ms) of the last refine_mesh / execute, per phase: the
 * snapshot of the old field and cell states, flagging and executing the
 * refinement, nodes and hanging-node constraints, the level grids' set-up,
 * the cell-state transfer, the prolongation tables, the solution transfer,
 * the inverse mass. */
#define ADM_AMR_REMESH_PHASES 8
int adm_amr_remesh_profile(adm_amr const *h, double *ms);
int adm_amr_n_leaves(adm_amr const *h, int64_t *n);
int adm_amr_leaves(adm_amr const *h, int32_t *lijk);
int adm_amr_dof_lattice(adm_amr const *h, int64_t *xyz);
/* Device pointer to the solution (n_dofs doubles); valid until the next
 * mesh change. */
int adm_amr_solution(adm_amr *h, double **y);
/* Device copies of the solution (n_dofs doubles) out of / into the handle. */
int adm_amr_get_solution(adm_amr *h, double *dst);
int adm_amr_set_solution(adm_amr *h, double const *src);
/* ThermalOperatorBase::set_time on every level. */
int adm_amr_set_time(adm_amr *h, double t);
/* dst = C^T (sum over levels of the leaves' operator) C src; device
 * composite vectors of n_dofs doubles. */
int adm_amr_vmult(adm_amr *h, double *dst, double const *src);
/* The composite inverse lumped mass (device, n_dofs doubles). */
int adm_amr_inverse_mass(adm_amr *h, double *dst);
/* One explicit Runge-Kutta step (cfg.time_method) of the solution. */
int adm_amr_evolve_one_time_step(adm_amr *h, double t, double dt, double *t_out);
/* The solution on the level grid of `level` (constraints resolved; host
 * array of that grid's adm_node_layout size) and the grid's layout. */
int adm_amr_level_values(adm_amr *h, int level, double *host);
int adm_amr_level_layout(adm_amr *h, int level, int64_t nodes[3], int64_t *pitch);
/* Cell states of the level grid's cells (ThermalPhysics::
 * set_state_to_material_properties, then the n_states x n_cells ratios,
 * state-major; cells that are not leaves of the level hold 0). */
int adm_amr_level_cell_state(adm_amr *h, int level, double *host);
/* Launch schedule of the level grids (adm_set_schedule's values): the
 * atomic schedule (default) launches once per level and application, the
 * coloured one eight times and the two-pass one a tile launch and a gather,
 * both adding in a fixed order (bit-reproducible). */
int adm_amr_set_schedule(adm_amr *h, int schedule);
/* ThermalPhysics::mark_has_melted on the refined mesh: every leaf whose
 * cell average of the solution exceeds threshold is flagged (flags stay
 * set); refine_and_transfer carries the flags like the cell states. */
int adm_amr_mark_has_melted(adm_amr *h, double threshold);
/* The has_melted flags of a level grid's cells (host array of the grid's
 * cells; cells that are not leaves of the level are 0). */
int adm_amr_level_has_melted(adm_amr *h, int level, uint8_t *host);
int adm_amr_synchronize(adm_amr *h);

#ifdef __cplusplus
}
#endif

#endif
