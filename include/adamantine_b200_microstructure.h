/*
 * adamantine_b200 -- microstructure data of the temperature field (C ABI).
 *
 * Microstructure::set_old_temperature and compute_G_and_R
 * (source/Microstructure.cc:57-63, source/Microstructure.hh:41-207), driven
 * around each time step as application/adamantine.hh:1235-1285 does: save
 * the field before the step, then after it collect, for every support point
 * of every active cell whose node went from above the cell material's
 * liquidus to at or below it, the record
 *   x, y, z, G = |grad T|, cooling rate, R = cooling rate / G
 * with the gradient of the cell's interpolant of the new field at the point
 * and the cooling rate as the reference computes it, old - new / delta_t
 * (the division binds to the new temperature only; R is inf where G is 0).
 * A node shared by several cells gives one record per cell. Records come in
 * the reference's file order: cells lexicographic (x fastest), points of a
 * cell lexicographic.
 */
#ifndef ADAMANTINE_B200_MICROSTRUCTURE_H
#define ADAMANTINE_B200_MICROSTRUCTURE_H

#include "adamantine_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct adm_microstructure adm_microstructure;

/* Bound to a set-up handle, which must outlive it (Microstructure
 * constructor; the file writing stays with the caller). */
int adm_microstructure_create(adm_thermal *h, adm_microstructure **out);
int adm_microstructure_destroy(adm_microstructure *m);
/* Device copy of the field before the step (n_nodes doubles, device
 * pointer). */
int adm_microstructure_set_old_temperature(adm_microstructure *m, double const *old_temperature);
/* Records of the step that produced temperature (device pointer) from the
 * saved field. *n_records receives their number; when records (host,
 * [n][6]) is not NULL and capacity >= *n_records they are written there,
 * otherwise nothing is written (call again with room for *n_records). */
int adm_microstructure_compute_G_and_R(adm_microstructure *m, double const *temperature, double delta_t,
                                       int64_t capacity, double *records, int64_t *n_records);

#ifdef __cplusplus
}
#endif

#endif
