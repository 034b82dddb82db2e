/*
 * adamantine_b200 -- material deposition (C ABI).
 *
 * Boxes along the scan path (deposition_along_scan_path and
 * merge_deposition_paths, source/material_deposition.cc:129-324) and their
 * activation of cells (get_elements_to_activate, :374-438, with
 * ThermalPhysics::add_material_start/end,
 * source/ThermalPhysics.templates.hh:595-825), driven per time step as
 * application/adamantine.hh:1134-1199 does. The cells a window of boxes
 * meets are found on the device (the structured mesh turns the bounding-box
 * search into index ranges) and appended to a device list; the activation
 * updates the cell data, the new nodes' temperature, the lumped mass and
 * the colour work lists without renumbering nodes.
 */
#ifndef ADAMANTINE_B200_DEPOSITION_H
#define ADAMANTINE_B200_DEPOSITION_H

#include "adamantine_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct adm_deposition adm_deposition;

/* Deposition boxes of the scan paths of the sources (cube sources have none),
 * boxes of deposition_length x deposition_width x deposition_height along
 * the power-on segments, times shifted back by lead_time, in chronological
 * order (ties keep path order). Host function (no GPU): with capacity 0 only
 * *n_boxes is set; otherwise capacity >= *n_boxes and the arrays receive
 * lo/hi [n][3] corners, time, cos and sin of the deposition direction. */
int adm_deposition_boxes(adm_source const *sources, int32_t n_sources, double length, double height, double width,
                         double lead_time, int64_t capacity, double *lo, double *hi, double *time, double *cosv,
                         double *sinv, int64_t *n_boxes);

/* Boxes (host arrays, times sorted) bound to a set-up handle;
 * deposition_time is geometry.deposition_time (minimum window length) and
 * duration the end of the simulation. */
int adm_deposition_create(adm_thermal *h, int64_t n_boxes, double const *lo, double const *hi, double const *time,
                          double const *cosv, double const *sinv, double deposition_time, double duration,
                          adm_deposition **out);
int adm_deposition_destroy(adm_deposition *d);
/* Activate the inactive cells that boxes [b0, b1) meet (closed boxes: a
 * touching face counts); a cell met by several boxes takes the direction of
 * the last one. New nodes of the device vector solution get new_temperature.
 * *n_activated (may be NULL) receives the number of new cells. */
int adm_deposition_activate_range(adm_deposition *d, int64_t b0, int64_t b1, double new_temperature,
                                  double *solution, int64_t *n_activated);
/* The driver's activation at the start of a time step: when time reaches
 * the end of the previous window, the boxes with deposition times in
 * [time - 1e-6 time_step, min(time + max(deposition_time, time_step),
 * duration)) are activated. */
int adm_deposition_step(adm_deposition *d, double time, double time_step, double new_temperature,
                        double *solution, int64_t *n_activated);

#ifdef __cplusplus
}
#endif

#endif
