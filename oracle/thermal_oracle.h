/*
 * CPU oracle for the adamantine thermal hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker: a plain C++17/OpenMP restatement of the
 * reference's CPU matrix-free heat operator and explicit time step. Only the
 * test suite, the smoke check and the CPU-baseline leg of the benchmark may
 * load it. The product (adamantine_b200) never links, loads or calls it.
 *
 * Restated reference code (paths inside adamantine v1.1.9):
 *   source/ThermalOperator.templates.hh:118-164   inverse lumped mass
 *   source/ThermalOperator.templates.hh:176-225   vmult / vmult_add
 *   source/ThermalOperator.templates.hh:227-413   (face) state ratios
 *   source/ThermalOperator.templates.hh:415-477   1/(rho c_p) + latent heat
 *   source/ThermalOperator.templates.hh:479-617   cell_local_apply
 *   source/ThermalOperator.templates.hh:619-751   face_local_apply
 *   source/ThermalOperator.templates.hh:753-895   get/set state
 *   source/MaterialProperty.hh:529-846            compute_material_property
 *   source/MaterialProperty.templates.hh:244-437  MaterialProperty::update
 *   source/MaterialProperty.templates.hh:537-621  set_state
 *   source/MaterialProperty.templates.hh:1158-1212 table lookup
 *   source/GoldakHeatSource.cc:24-89, ElectronBeamHeatSource.cc:24-93,
 *   source/CubeHeatSource.cc:45-71, ScanPath.cc:197-275
 *   source/ThermalPhysics.templates.hh:43-124,854-888 (time step)
 *
 * The layout of orc_config is identical, field by field, to adm_config in
 * include/adamantine_b200.h; a test checks it.
 */
#ifndef ADAMANTINE_THERMAL_ORACLE_H
#define ADAMANTINE_THERMAL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_source
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
  /* n_segments x 5 doubles: end_time, power_modifier, x, y, z */
  const double *segments;
} orc_source;

typedef struct orc_config
{
  int32_t dim;        /* 2 or 3 */
  int32_t degree;     /* FE_Q degree, 1..4 */
  int32_t quadrature; /* 0 QGauss(degree+1), 1 QGaussLobatto(degree+1) */
  int32_t n_cells[3]; /* 3D: x (length), y (width), z (height); 2D: x, z */
  double origin[3];
  double extent[3];
  int32_t n_materials;
  int32_t n_states; /* 1 Solid, 2 SolidLiquid, 3 SolidLiquidPowder */
  int32_t use_table;
  int32_t p_order;
  double poly[4][8][3][5];
  double table[4][8][3][12][2];
  double props[4][5];
  int32_t n_boundary_types;
  int32_t boundary_types[8];
  int32_t n_sources;
  int32_t pad0;
  orc_source sources[4];
  int32_t time_method; /* 0 forward Euler, 1 RK2 midpoint, 2 RK3, 3 RK4 */
  int32_t n_threads;
} orc_config;

typedef struct orc_oracle orc_oracle;

orc_oracle *orc_create(orc_config const *cfg);
void orc_destroy(orc_oracle *o);
int64_t orc_n_nodes(orc_oracle const *o);
int64_t orc_n_cells(orc_oracle const *o);
int32_t orc_n_qp(orc_oracle const *o);

/* Per-cell arrays (lexicographic cell index, x fastest). */
void orc_set_cells(orc_oracle *o, uint8_t const *active,
                   uint8_t const *material_id, uint8_t const *initial_state,
                   double const *deposition_cos, double const *deposition_sin);
/* Cells whose region carries material (NULL: the active cells). A face of an
 * active cell is a boundary face where the neighbour is outside it: a level
 * grid of a refined mesh passes the whole material region, its active cells
 * being only that level's leaves. Before orc_setup. */
void orc_set_domain(orc_oracle *o, uint8_t const *domain);
/* ThermalPhysics::setup(): inverse mass + get_state_from_material_properties */
void orc_setup(orc_oracle *o);

void orc_set_time(orc_oracle *o, double t);
void orc_vmult(orc_oracle *o, double *dst, double const *src);
void orc_vmult_add(orc_oracle *o, double *dst, double const *src);
void orc_inverse_mass(orc_oracle const *o, double *out);
void orc_node_active(orc_oracle const *o, uint8_t *out);
double orc_evolve_one_time_step(orc_oracle *o, double t, double dt,
                                double *solution);

void orc_set_state_to_material_properties(orc_oracle *o);
void orc_get_state_from_material_properties(orc_oracle *o);
void orc_get_cell_state(orc_oracle const *o, double *out); /* [n_states][C] */
void orc_set_cell_state(orc_oracle *o, double const *in);
void orc_get_qp_powder(orc_oracle const *o, double *out); /* [C][Q] */
void orc_get_qp_liquid(orc_oracle const *o, double *out); /* [C][Q] */
/* MaterialProperty::update: cell-average temperature -> cell state and
 * property values [8][C]. */
void orc_evaluate_material_properties(orc_oracle *o, double const *temperature,
                                      double *property_values);
void orc_mark_has_melted(orc_oracle *o, double threshold,
                         double const *temperature, uint8_t *has_melted);
/* add_material_start/end on the fixed full-grid numbering */
void orc_activate_cells(orc_oracle *o, int64_t const *cells, int64_t n,
                        double new_temperature, double const *cos_new,
                        double const *sin_new, double *solution);

/* Point evaluation of one heat source after orc_set_time. */
void orc_source_values(orc_oracle *o, int32_t beam, double const *points,
                       int64_t n_points, double *out);
/* Beam state after orc_set_time: center[3], alpha, on. */
void orc_source_state(orc_oracle const *o, int32_t beam, double *out5);

#ifdef __cplusplus
}
#endif

#endif
