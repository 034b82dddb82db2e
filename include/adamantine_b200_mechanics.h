/*
 * adamantine_b200 -- thermoelastic displacement on the thermal mesh (C ABI).
 *
 * The mechanical solve the driver runs after the thermal step
 * (application/adamantine.hh:1289-1345): MechanicalPhysics::setup_dofs
 * (source/MechanicalPhysics.cc:280-440) picks the cells that carry
 * displacement (thermally active, solid ratio above 0.99), MechanicalOperator
 * (source/MechanicalOperator.cc:183-486) forms the isotropic elasticity
 * operator
 *   a(u, v) = sum_q JxW (lambda div u div v + mu grad u : grad v^T
 *                        + mu grad u : grad v)
 * (FE_Q(p)^3, QGauss(p + 1)) and the right-hand side
 *   sum_q JxW ((3 lambda + 2 mu) alpha (T - T_ref) div v + f . v),
 * T the thermal field interpolated at the quadrature points, T_ref the
 * material's reference temperature where the cell has melted and the
 * initial temperature elsewhere, f = (0, 0, -rho_s g) with g = 9.80665
 * (GravityForce, source/BodyForce.cc:18-31); MechanicalPhysics::solve
 * (:488-520) runs CG to 1e-12 |rhs|. Displacements on clamped boundary
 * faces are zero (Dirichlet, eliminated: the constrained rows of the
 * operator are the identity).
 *
 * The handle is bound to a thermal handle (same mesh, degree and node
 * layout): displacement vectors are 3 node vectors (x, y, z components)
 * of adm_n_nodes doubles each, consecutive; entries of nodes that carry no
 * displacement are 0.
 *
 * After each solve the stress is updated as MechanicalPhysics::solve and
 * compute_stress do (:520-634): the displacement increment since the last
 * solve gives the strain at every Gauss point of the cells that carry
 * displacement, the trial stress adds C : strain to the stored stress, and
 * where the norm of its deviator minus the back stress reaches the plastic
 * internal variable (initially the elastic limit) the radial return of the
 * combined isotropic-kinematic J2 model updates the stress, the plastic
 * internal variable and the back stress. A cell that starts carrying
 * displacement (material added, or solidified) starts from zero stress and
 * back stress and the elastic limit; the previous displacement is carried
 * over as MechanicalPhysics::setup_dofs does (:296-437: a node keeps it when
 * the last cell touching it in cell order already carried displacement,
 * else it restarts from 0).
 */
#ifndef ADAMANTINE_B200_MECHANICS_H
#define ADAMANTINE_B200_MECHANICS_H

#include "adamantine_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct adm_mech_config
{
  /* per material (the thermal configuration's materials), the solid
   * state's mechanical properties (MaterialProperty mechanical_properties):
   * lame_first_parameter, lame_second_parameter, thermal_expansion_coef,
   * density (solid) */
  double lame_first[4];
  double lame_second[4];
  double thermal_expansion[4];
  double density[4];
  /* reference temperature per material (cells that have melted) and the
   * initial temperature (the others); thermoelastic: 1, elastostatic: 0
   * (no thermal term) */
  double reference_temperature[4];
  double initial_temperature;
  int32_t thermoelastic;
  /* 1: gravity (GravityForce) in the right-hand side */
  int32_t gravity;
  /* bit f: box face f (x-, x+, y-, y+, z-, z+) is clamped */
  int32_t clamped_faces;
  /* CG: relative tolerance (0: 1e-12) and iteration limit (0: the number
   * of displacement DoFs) */
  double rel_tol;
  int32_t max_iter;
  int32_t pad0;
  /* per material, the solid's plastic_modulus, isotropic_hardening (the
   * isotropic share of the hardening, 0..1) and elastic_limit
   * (MaterialProperty mechanical properties; +INFINITY, the reference's
   * default when elastic_limit is not given, keeps the material elastic) */
  double plastic_modulus[4];
  double isotropic_hardening[4];
  double elastic_limit[4];
} adm_mech_config;

typedef struct adm_mechanics adm_mechanics;

/* Preconditioners of the CG (MechanicalPhysics::solve preconditions with
 * algebraic multigrid): the diagonal, or a geometric multigrid V-cycle
 * (the default) over FE_Q(1) levels of the box with half the cells per
 * direction each, Chebyshev smoothing on diag^-1 A and an exact solve of
 * the coarsest level. */
#define ADM_MECH_PRECONDITIONER_JACOBI 0
#define ADM_MECH_PRECONDITIONER_MULTIGRID 1

/* Bound to a set-up thermal handle, which must outlive it. */
int adm_mechanics_create(adm_thermal *thermal, adm_mech_config const *cfg, adm_mechanics **out);
int adm_mechanics_destroy(adm_mechanics *h);
/* MechanicalPhysics::setup_dofs + update_rhs: the cells that carry
 * displacement from the thermal handle's activity and cell states
 * (ThermalPhysics::set_state_to_material_properties is called) and the
 * right-hand side from the temperature (device node vector of the thermal
 * handle) and the thermal handle's has_melted flags. */
int adm_mechanics_setup(adm_mechanics *h, double const *temperature);
/* dst = A src (device displacement vectors, 3 x adm_n_nodes doubles). */
int adm_mechanics_vmult(adm_mechanics *h, double *dst, double const *src);
/* The right-hand side of the last setup (device, 3 x adm_n_nodes). */
int adm_mechanics_rhs(adm_mechanics *h, double *dst);
/* MechanicalPhysics::solve (elastic): displacement (device, 3 x
 * adm_n_nodes), CG iterations and final residual norm. */
int adm_mechanics_solve(adm_mechanics *h, double *displacement, int32_t *iterations, double *residual);
/* Selects the CG preconditioner (ADM_MECH_PRECONDITIONER_*). */
int adm_mechanics_set_preconditioner(adm_mechanics *h, int32_t kind);
/* Levels of the multigrid hierarchy (built at the first multigrid solve
 * after a setup; 0 before) and the free DoFs of its coarsest level. */
int adm_mechanics_multigrid_levels(adm_mechanics const *h, int32_t *n_levels, int64_t *coarsest_dofs);
/* Counts: displacement DoFs (3 per node of a cell that carries
 * displacement, clamped ones included) and cells that carry displacement. */
int adm_mechanics_n_dofs(adm_mechanics const *h, int64_t *n_dofs, int64_t *n_cells);
/* Per node (adm_n_nodes bytes): 0 no displacement, 1 free, 2 clamped. */
int adm_mechanics_node_mask(adm_mechanics const *h, uint8_t *mask);
/* The stress state at the Gauss points (MechanicalPhysics::get_stress_tensor,
 * the back stress and the plastic internal variable), device arrays indexed
 * by q + nq (cell) with nq = (degree + 1)^3 Gauss points per cell
 * (x fastest) and the thermal handle's cell index: stress and back_stress
 * [6][n_cells nq] (components xx, yy, zz, xy, xz, yz), plastic
 * [n_cells nq]; any may be NULL. Values of cells that carry no displacement
 * are those they last had (zero stress and the elastic limit before they
 * ever carried any). */
int adm_mechanics_stress_state(adm_mechanics *h, double *stress, double *back_stress, double *plastic);

#ifdef __cplusplus
}
#endif

#endif
