/*
 * adamantine_b200 -- hand-written adjoint of the explicit time step (C ABI).
 *
 * No counterpart in the reference, which runs the forward problem only; the
 * forward being differentiated is adm_evolve_one_time_step
 * (ThermalPhysicsInterface::evolve_one_time_step,
 * source/ThermalPhysics.templates.hh:854-888) with the operator of
 * source/ThermalOperator.templates.hh:479-751 (cells and faces).
 *
 * Objective: J = sum_{k, p} (T_{n_k}[node_p] - target_{k,p})^2 over the
 * observation steps n_k and the observed nodes. Gradient: dJ/dlog(theta) for
 * theta = (conductivity scale, specific-heat scale, absorptivity, power),
 * i.e. theta * dJ/dtheta, where the conductivities of every state are
 * multiplied by the first, the specific heats by the second and every
 * Goldak / electron-beam source by the product of the last two (cube sources
 * keep their value). Covered: polynomial and table properties, several
 * materials, one to three material states (with the powder history of the
 * cells' and the boundary faces' points), deposition-angle rotation,
 * convective / radiative boundaries and active/inactive interfaces.
 */
#ifndef ADAMANTINE_B200_ADJOINT_H
#define ADAMANTINE_B200_ADJOINT_H

#include "adamantine_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct adm_adjoint adm_adjoint;

/* Adjoint driver over a set-up handle. The handle's phase state at this
 * call (the powder history of the Gauss points and of the boundary faces'
 * points) is the initial state of every objective / gradient run. Cells
 * activated on the handle afterwards (a new face-point layout or a
 * deposition angle) make the later calls fail with ADM_ERR_INVALID: create
 * a new adjoint then. */
int adm_adjoint_create(adm_thermal *h, adm_adjoint **out);
int adm_adjoint_destroy(adm_adjoint *a);
/* Observations (host arrays): n_obs_steps step numbers in [0, n_steps],
 * n_points node indices of the adm_node_layout vector, targets
 * [n_obs_steps][n_points]. */
int adm_adjoint_set_observations(adm_adjoint *a, int32_t n_obs_steps, int32_t const *obs_steps,
                                 int32_t n_points, int64_t const *node_index, double const *targets);
/* Forward run of n_steps from the device vector y0 (unchanged) and the
 * initial phase state: *J, and the final field into y_final (device, may
 * be NULL). */
int adm_adjoint_objective(adm_adjoint *a, double t0, double dt, int32_t n_steps, double const *y0, double *J,
                          double *y_final);
/* Forward run with a checkpoint every checkpoint_every steps, then the
 * backward sweep (each segment recomputed from its checkpoint): *J and
 * grad[4] = dJ/dlog(k scale, c_p scale, absorptivity, power). The handle's
 * phase state ends as after the forward run. checkpoint_every <= 0 picks
 * the longest segment whose stage stores (the stage inputs, and the phase
 * states with three material states) fit in half of the free device
 * memory: the whole run when it fits, so that nothing is recomputed. */
int adm_adjoint_gradient(adm_adjoint *a, double t0, double dt, int32_t n_steps, int32_t checkpoint_every,
                         double const *y0, double *J, double *grad, double *y_final);
/* The checkpoint interval the last adm_adjoint_gradient used. No
 * counterpart in the reference. */
int adm_adjoint_checkpoint_interval(adm_adjoint const *a, int32_t *checkpoint_every);
/* Adjoint values at or below flush times the stage's largest |M^-1 lambda|
 * count as zero in adm_adjoint_gradient, and tiles holding only such values
 * (and no powder adjoint) are skipped. The explicit stencil spreads the
 * adjoint of a misfit at a few points by about one cell per stage with
 * values falling by orders of magnitude per cell, so most tiles hold only
 * negligible values. Default 1e-30 (the dropped terms lie some 14 orders of
 * magnitude below double rounding); 0 skips exact zeros only. 0 <= flush <
 * 1e-3. No counterpart in the reference. */
int adm_adjoint_set_flush(adm_adjoint *a, double flush);
/* The transpose operator: dst = (d r / d T)^T mu at the field y (device
 * vectors), r the vmult residual at the handle's time, with the handle's
 * current phase state as the history input; grad[3] (may be NULL) receives
 * the log-derivatives of mu . r for k scale, c_p scale and source. */
int adm_adjoint_vmult_transpose(adm_adjoint *a, double *dst, double const *y, double const *mu, double *grad);

#ifdef __cplusplus
}
#endif

#endif
