/*
 * ORACLE — test infrastructure only, never part of the product path.
 *
 * CPU restatement of the nh-flood-2d compact solver's local-inertial step
 * (src/nh_flood_2d/core/solver_compact.py) together with its device clock
 * (core/clock.py), CFL reduction, positivity limiter, hanging-edge pressure
 * reconstruction (core/pressure.py) and per-block budget diagnostics.
 *
 * The reference itself is Python + Taichi JIT kernels and cannot run here
 * (taichi 1.7.4 / fastdb4py 0.2.4 are not installed). Parity with Taichi's
 * own floating-point lowering is therefore pinned only through the
 * reference tests' known answers (tests/test_oracle_pins.py,
 * tests/test_oracle_physics.py, tests/test_oracle_clock.py,
 * tests/test_oracle_restart.py, tests/test_gate_oracle.py); bit-level
 * agreement with a Taichi CPU run is unpinned. The host-side inputs the
 * step consumes (land parameters, hanging-edge tables, face fractions,
 * still-water depths, gate layout, clock ticks, series and rain rates) are
 * pinned bit for bit to the reference's own code by the golden vectors in
 * tests/golden/ (tests/test_golden_host.py).
 *
 * Differences from the reference that are deliberate (this design's choices):
 *  - budget diagnostics are accumulated as FP64 per-block partials
 *    (fixed pairwise tree inside each 256-cell block, then TwoSum
 *    compensation across steps) instead of exact base-65536 integer digits
 *    (core/device_budget.py:28-57);
 *  - pow(x, 7/3) and exp() are evaluated with the FP64 routines in
 *    mathref.c (published methods, see there) and rounded once to F32.
 *
 * Every array uses the reference's layout: index 0 of cells and sides is the
 * exterior sentinel, face CSR is [e_num][4] in l, r, b, t order, topology is
 * [s_num][3] = (orient, lower, higher).
 */
#ifndef NHF_ORACLE_STEP_REF_H
#define NHF_ORACLE_STEP_REF_H

#include <stdint.h>

#define ORA_TRACE_COLS 10 /* reference 9 columns + wet-cell count */

/* Arithmetic type of the state and the step. The default build is F32, the
 * reference's Taichi default_fp; the precision study compiles the same
 * source with -DORA_REAL_DOUBLE (liboracle_f64.so), where every state array
 * and every step operation is F64 while the clock keeps its F32 dt choice
 * and fixed-point ticks. */
#ifdef ORA_REAL_DOUBLE
typedef double ora_real;
#else
typedef float ora_real;
#endif

typedef struct {
    int32_t e_num, s_num, b_num, n_rates, isl_len;
    int32_t batch_size;
    ora_real g, afa, sita, min_h;
    float min_dt;
    /* cells [e_num] */
    const ora_real *x, *y, *area, *width, *height, *f0, *fc, *k;
    const int32_t *boundary_id, *rain_index;
    const int32_t *face_ptr, *face_count; /* [e_num*4] */
    const int32_t *isl_data;              /* [isl_len] */
    const ora_real *weight;                  /* [e_num] */
    /* sides [s_num] */
    const int32_t *topology; /* [s_num*3] */
    const ora_real *length, *side_n;
    const uint8_t *sbf;
    /* boundaries [max(1,b_num)] */
    const int32_t *kind;
    /* theta < 1 only: open-face fractions [e_num*4] (may be NULL when sita == 1) */
    const ora_real *open_face;
    /* hanging-edge reconstruction (hang_cells == 0 when absent) */
    int32_t hang_cells, hang_edges;
    const int32_t *edge_index; /* [s_num] */
    const ora_real *offsets;      /* [hang_edges*2] */
    const int32_t *slots;      /* [hang_edges*2] */
    const int32_t *hcells;     /* [hang_cells] */
    const int32_t *axes;       /* [hang_cells*2] */
    /* mutable state (caller-owned) */
    ora_real *bed, *depth, *q, *rain_time, *infiltration, *max_depth, *max_speed, *u, *v;
    uint32_t *peak_hi, *peak_lo;
    ora_real *pipe_q; /* [e_num] or NULL (no coupling) */
} ora_mesh;

typedef struct ora_ctx ora_ctx;

ora_ctx *ora_create(const ora_mesh *mesh);
void ora_destroy(ora_ctx *c);
/* reference initialize(): depth = 0, infiltration = f0, dh = -999, sdc */
void ora_initialize(ora_ctx *c);
void ora_set_threads(int n);
void ora_set_clock(ora_ctx *c, const uint32_t now[2]);
void ora_get_clock(const ora_ctx *c, uint32_t now[2]);
void ora_set_active(ora_ctx *c, int active);
void ora_set_forcing(ora_ctx *c, const ora_real *coefficients, const ora_real *rain_rates, int raining);
void ora_apply_initial_levels(ora_ctx *c, const ora_real *targets);
void ora_compute_cfl(ora_ctx *c);
void ora_initial_diagnostics(ora_ctx *c);
void ora_reset_extrema(ora_ctx *c);
/* begin + batch_size x (prepare, pressure, tick, cfl, finish); trace [batch][10] */
void ora_run_batch(ora_ctx *c, const uint32_t target[2], const uint32_t origin[2], uint32_t *trace);
/* one prepared physical step with an externally supplied dt (parity probes) */
void ora_budget_flush(ora_ctx *c, double *totals /* [4+6B] */);
int ora_budget_terms(const ora_ctx *c);
ora_real ora_ndt(const ora_ctx *c);
/* precision study only: replace the CFL candidate of the next step */
void ora_set_ndt(ora_ctx *c, float ndt);
int32_t ora_cfl_arg(const ora_ctx *c);
void ora_limits(const ora_ctx *c, ora_real values[5], int32_t ids[3]);
void ora_reset_limits(ora_ctx *c);
void ora_read_eq(const ora_ctx *c, ora_real *eq /* [e_num*4] */);
void ora_read_flow_depth(const ora_ctx *c, ora_real *out /* [s_num] */);
void ora_read_gradients(const ora_ctx *c, ora_real *out /* [hang_cells*2] */);
/* pressure-only probe for the reference's split-face tests */
void ora_update_pressure(ora_ctx *c);
ora_real ora_pressure_difference(const ora_ctx *c, int side, int lower, int higher, ora_real raw);

/* Gate controller (core/gate.py:35-206). Tables and controller words are
 * caller-owned and stay alive while attached. Exchange terms (gate/pond and
 * gate/river volumes, overtopping) are accumulated per 256 entries of
 * flux_sides; source terms (rain, infiltration, positivity, pipe, boundary,
 * rounding of pond and gate cells) per 256 cells. Terms: 10 count + 8. */
typedef struct {
    int32_t count, n_targets, n_flux;
    const int32_t *cell_gate;  /* [e_num] gate index of each cell, -1 off gates */
    const int32_t *pond;       /* [e_num] 1 on pond cells, 0 at the sentinel */
    const ora_real *closed;    /* [e_num] closed bed */
    const int32_t *targets;    /* [n_targets] gate cells, gate by gate */
    const int32_t *controls;   /* [count] control cell of each gate */
    const int32_t *flux_sides; /* [n_flux] recorded sides in side order */
    uint32_t formal_tick[2];   /* control starts at this clock (formal t = 0) */
    float trigger_level, opening_seconds, open_elevation;
    int32_t *commanded, *flow_seen, *opened; /* [count] */
    uint32_t *command, *first_flow, *opened_at; /* [count*2] hi, lo */
} ora_gate;
void ora_gate_attach(ora_ctx *c, const ora_gate *gate);
/* check + move at the current clock (the run-start check_gates call) */
void ora_gate_check(ora_ctx *c);
int ora_gate_terms(const ora_ctx *c);
/* interval totals since the last flush, in term order; clears them */
void ora_gate_flush(ora_ctx *c, double *totals);

/* mathref.c */
double ora_ln(double x);
double ora_exp(double y);
double ora_pow(double x, double y);
float ora_powf(float x, float y);
float ora_expf(float a);

#endif
