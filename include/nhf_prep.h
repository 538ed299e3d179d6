/* nhflood host preprocessing: NE/NS mesh text -> cell and side tables.
 *
 * Replaces the reference's per-line Python preprocessing
 * (src/nh_flood_2d/preprocess/domain.py): _filter_ne_ns (221-347),
 * create_ne_fdb_compact (83-174) and create_ns_fdb_parallel /
 * _batch_ns_worker (439-470). Host code only; no CUDA. Every array has a
 * sentinel entry 0 (cells and sides are numbered from 1). Returns 0 or -1
 * with the reason in nhp_error(). */
#ifndef NHF_PREP_H
#define NHF_PREP_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct nhp_mesh nhp_mesh;

/* Parse and filter both texts (the files' bytes), build the tables. */
int nhp_prepare(const char *ne_text, size_t ne_len, const char *ns_text, size_t ns_len, nhp_mesh **out);
/* sizes[0] = cells + 1, sizes[1] = sides + 1, sizes[2] = length of the side list. */
int nhp_sizes(const nhp_mesh *m, int64_t sizes[3]);
/* Cell tables: index, x, y, z [cells+1]; type [cells+1] (u8); counts and
 * ptr [cells+1][4] (l, r, b, t); isl [sizes[2]]. NULL skips an array. */
int nhp_copy_cells(const nhp_mesh *m, uint32_t *index, float *x, float *y, float *z, uint8_t *type,
                   uint32_t *counts, uint32_t *ptr, uint32_t *isl);
/* Side tables: index, length, x, y, z [sides+1]; attr (u8); topo [sides+1][3]
 * = (orient, lower, higher). NULL skips an array. */
int nhp_copy_sides(const nhp_mesh *m, uint32_t *index, float *length, float *x, float *y, float *z, uint8_t *attr,
                   uint32_t *topo);
void nhp_free(nhp_mesh *m);
const char *nhp_error(void);

#ifdef __cplusplus
}
#endif
#endif
