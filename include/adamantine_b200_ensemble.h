/*
 * adamantine_b200 -- batched ensemble and EnKF analysis (C ABI).
 *
 * The reference runs its data-assimilation ensemble as a loop over
 * independent ThermalPhysics objects (application/adamantine.hh:2137-2142)
 * and updates it with DataAssimilator::update_ensemble
 * (source/DataAssimilator.cc:95-189). Here all members of an ensemble advance
 * together in one launch per colour and stage, and the analysis runs on the
 * GPU in FP64. Conventions are those of adamantine_b200.h (status codes,
 * adm_last_error, one stream per handle, device pointers).
 *
 * Ensemble vectors: member k's node vector (same layout as adm_n_nodes /
 * adm_node_layout of a single problem) starts at solutions + k * stride
 * (adm_ensemble_stride, in doubles); the array must be 16-byte aligned.
 */
#ifndef ADAMANTINE_B200_ENSEMBLE_H
#define ADAMANTINE_B200_ENSEMBLE_H

#include "adamantine_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct adm_ensemble adm_ensemble;
typedef struct adm_enkf adm_enkf;

/* create_database_ensemble + one ThermalPhysics per member
 * (source/ensemble_management.cc:213-277, application/adamantine.hh:1663-1730).
 * cfgs: n_members configurations that agree on the mesh, element, quadrature,
 * material states, table/polynomial choice, boundary types, time method and
 * source kinds; material and source values may differ per member. */
int adm_ensemble_create(adm_config const *cfgs, int32_t n_members, int device, void *stream,
                        adm_ensemble **out);
int adm_ensemble_destroy(adm_ensemble *e);
/* adm_set_cells for member k (its own active cells, materials, states). */
int adm_ensemble_set_cells(adm_ensemble *e, int32_t member, uint8_t const *active,
                           uint8_t const *material_id, uint8_t const *initial_state,
                           double const *deposition_cos, double const *deposition_sin);
/* adm_setup of every member, then the batched work list. */
int adm_ensemble_setup(adm_ensemble *e);
/* Doubles between consecutive members' vectors. */
int adm_ensemble_stride(adm_ensemble const *e, int64_t *stride);
/* Number of (member, tile) work items of one batched colour sweep. */
int adm_ensemble_n_work_items(adm_ensemble const *e, int64_t *n);

/* ThermalPhysicsInterface::evolve_one_time_step (source/ThermalPhysics.templates.hh:854-888)
 * for every member: one launch per colour and stage over all members. */
int adm_ensemble_evolve_one_time_step(adm_ensemble *e, double t, double dt, double *solutions,
                                      double *t_out);
/* The same step as the reference's loop over members (each member through
 * its own single-problem launches); the batched step's baseline. */
int adm_ensemble_evolve_looped(adm_ensemble *e, double t, double dt, double *solutions,
                               double *t_out);
/* n_steps batched steps replayed from one captured CUDA graph. */
int adm_ensemble_evolve_n_steps(adm_ensemble *e, double t, double dt, int32_t n_steps,
                                double *solutions, double *t_out);

/* ThermalPhysics::update_physics_parameters (source/ThermalPhysics.templates.hh:827-852)
 * for member k: new depth, efficiency, radius and power of source i. */
int adm_ensemble_update_beam(adm_ensemble *e, int32_t member, int32_t i, adm_source const *beam);
/* New material tables for member k (same shape as at creation); no
 * counterpart in the reference, which augments only beam parameters. */
int adm_ensemble_update_material(adm_ensemble *e, int32_t member, adm_config const *cfg);
/* MaterialProperty::get_state of member k: [n_states][n_cells], host. */
int adm_ensemble_get_cell_state(adm_ensemble *e, int32_t member, double *state_host);
/* Inverse lumped mass of member k into a device vector. */
int adm_ensemble_get_inverse_mass_matrix(adm_ensemble *e, int32_t member, double *dst);
/* Launch schedule of the batched stages (ADM_SCHEDULE_* of adamantine_b200.h). */
int adm_ensemble_set_schedule(adm_ensemble *e, int32_t schedule);
/* Cells per thread of the FE_Q(1) kernel for the batched stages and the
 * members' own (looped) launches (adm_set_cells_per_thread). */
int adm_ensemble_set_cells_per_thread(adm_ensemble *e, int32_t n);
int adm_ensemble_get_cells_per_thread(adm_ensemble const *e, int32_t *n);
/* Autotuner: times one batched step of size dt with each schedule (and, for
 * FE degree 1, each cells-per-thread variant) on a copy of solutions (phase
 * history and clocks restored), keeps the fastest and returns its schedule;
 * ms[2] (may be NULL) receives the best per-step times of the coloured and
 * atomic schedules. */
int adm_ensemble_autotune(adm_ensemble *e, double const *solutions, double dt, int32_t *schedule, double *ms);
/* The same over every schedule; ms (may be NULL) receives up to n_ms of the
 * ADM_N_SCHEDULES best per-step times, indexed by schedule. */
int adm_ensemble_autotune_schedules(adm_ensemble *e, double const *solutions, double dt, int32_t *schedule,
                                    double *ms, int32_t n_ms);
/* First non-zero sticky device error word over the members (synchronizes). */
int adm_ensemble_device_error(adm_ensemble *e, int32_t *code);
int adm_ensemble_synchronize(adm_ensemble *e);

/* Analysis workspace on a device and stream (NULL: default stream). */
int adm_enkf_create(int device, void *stream, adm_enkf **out);
int adm_enkf_destroy(adm_enkf *e);
/* Covariance localization functions (data_assimilation.
 * localization_cutoff_function, source/DataAssimilator.cc:71-91). */
#define ADM_LOC_NONE 0
#define ADM_LOC_STEP 1
#define ADM_LOC_GASPARI_COHN 2

/* DataAssimilator::update_ensemble (source/DataAssimilator.cc:95-189) in
 * FP64 on the device, dense Cholesky of H P H^T + R instead of GMRES:
 *   x_k += P H^T (H P H^T + R)^-1 (obs + perturbations_k - H_k x_k)
 * for the augmented states [x_k; p_k], P their sample covariance (divided
 * by N - 1). All arrays are device memory:
 *   states        N vectors, member k at states + k * stride, n_state entries
 *                 each (updated in place)
 *   params        [N][n_params] augmented parameters (updated; may be NULL
 *                 when n_params == 0)
 *   obs_index     [N][n_obs] state index of observation j for member k
 *                 (calc_Hx with a member-specific map: ragged members see
 *                 the same point at different nodes)
 *   obs           [n_obs] observed values
 *   obs_var       [n_obs] diagonal of R, or NULL when obs_cov is given
 *   obs_cov       [n_obs][n_obs] dense R (row-major), or NULL
 *   perturbations [N][n_obs] the draws e_k ~ N(0, R) of fill_noise_vector
 *                 (:630-670), supplied by the caller
 *   update_mask   [N][n_state] 1 where member k's entry is updated, or NULL
 * 2 <= N <= 64, 1 <= n_obs <= 16384. Synchronizes. Nothing is updated
 * when H P H^T + R is not positive definite (ADM_ERR_DEVICE) or an index is
 * outside [0, n_state) (ADM_ERR_INVALID). */
/* Localization of the analyses of this handle
 * (update_covariance_sparsity_pattern and calc_sample_covariance_sparse,
 * source/DataAssimilator.cc:512-611,690-752): a covariance entry between two
 * state entries whose support points are farther apart than cutoff is zero
 * (the reference's sparsity pattern, whatever the function); within the
 * cutoff it is scaled by 1 (ADM_LOC_NONE, ADM_LOC_STEP) or by the
 * Gaspari-Cohn function of 2 d / cutoff (ADM_LOC_GASPARI_COHN). Parameter
 * rows are not localized. The support point of state entry
 *   i = a + pitch * (b + nodes[1] * c)   (0 <= a < nodes[0], ...)
 * is origin + (a, b, c) * spacing; entries with a >= nodes[0] (row padding)
 * are left unchanged. obs_xyz [n_obs][3] (host) are the support points of
 * the observed entries. The analyses then need n_state == pitch * nodes[1] *
 * nodes[2] and n_obs observations. cutoff covering every pair with
 * ADM_LOC_NONE or ADM_LOC_STEP is the plain analysis; n_obs == 0 removes the
 * localization. */
int adm_enkf_set_localization(adm_enkf *e, int32_t function, double cutoff, int32_t n_obs, double const *obs_xyz,
                              double const *origin, double const *spacing, int64_t const *nodes, int64_t pitch);

int adm_enkf_analysis(adm_enkf *e, int32_t n_members, double *states, int64_t stride,
                      int64_t n_state, double *params, int32_t n_params, int32_t n_obs,
                      int64_t const *obs_index, double const *obs, double const *obs_var,
                      double const *obs_cov, double const *perturbations,
                      uint8_t const *update_mask);

/* Building blocks of the analysis of an ensemble whose members are split over
 * several GPUs (one process per GPU; the caller does the collectives, see
 * adamantine_b200/sharded.py): each rank observes its members
 * (adm_enkf_observe), all-gathers HX, computes the N x N weight matrix
 * redundantly (adm_enkf_gain), all-reduces the per-rank sums of the
 * augmented state (adm_enkf_local_sum), forms its
 * members' contribution to every member's update (adm_enkf_partial_update),
 * reduce-scatters those contributions and applies its share
 * (adm_enkf_apply). The result equals adm_enkf_analysis on all members.
 * Device arrays; each call synchronizes.
 *   hx      [n_members][n_obs]     H_k x_k
 *   w       [n_members][n_members] W = HA^T (HA HA^T/(N-1) + R)^-1 D / (N-1)
 *   sum     [n_state + n_params]   sum of the augmented state (local or all members)
 *   w_rows  [n_local][n_members]   the local members' rows of W
 *   u       [n_members][n_state + n_params] (partial) or [n_local][...] (apply) */
int adm_enkf_observe(adm_enkf *e, int32_t n_members, double const *states, int64_t stride, int64_t n_state,
                     int32_t n_obs, int64_t const *obs_index, double *hx);
/* 2 <= n_members <= 256. */
int adm_enkf_gain(adm_enkf *e, int32_t n_members, int32_t n_obs, double const *hx, double const *obs,
                  double const *obs_var, double const *obs_cov, double const *perturbations, double *w);
int adm_enkf_local_sum(adm_enkf *e, int32_t n_local, double const *states, int64_t stride, int64_t n_state,
                       double const *params, int32_t n_params, double *sum);
/* n_local <= 64 members on this GPU, n_members in the whole ensemble; sum
 * over all members (the mean is sum / n_members). */
int adm_enkf_partial_update(adm_enkf *e, int32_t n_local, int32_t n_members, double const *states, int64_t stride,
                            int64_t n_state, double const *params, int32_t n_params, double const *sum,
                            double const *w_rows, double *u);
/* adm_enkf_partial_update with the handle's localization: the local members
 * are members first_member .. first_member + n_local - 1 of the ensemble,
 * and the observation-space anomalies and weights come from the last
 * adm_enkf_gain on this handle (same members and observations). Without
 * localization it is adm_enkf_partial_update. */
int adm_enkf_partial_update_localized(adm_enkf *e, int32_t n_local, int32_t first_member, int32_t n_members,
                                      double const *states, int64_t stride, int64_t n_state, double const *params,
                                      int32_t n_params, double const *sum, double const *w_rows, double *u);
int adm_enkf_apply(adm_enkf *e, int32_t n_local, double *states, int64_t stride, int64_t n_state, double *params,
                   int32_t n_params, double const *u, uint8_t const *update_mask);

#ifdef __cplusplus
}
#endif

#endif
