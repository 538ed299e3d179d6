/*
 * nhflood — B200 (sm_100a) local-inertial flood step, C ABI.
 *
 * Drop-in boundary for the Taichi fields, kernels and compiled ti.graph
 * inside the reference's _evolve (nh-flood-2d,
 * src/nh_flood_2d/core/solver_compact.py:179-1008). The reference has no
 * FFI of its own: every entry point below replaces one host call on a
 * Taichi field or kernel, cited beside it. A Python host binds it with
 * ctypes (nhflood/native.py is that binding).
 *
 * Conventions
 *  - Arrays keep the reference's layout: cell and side index 0 is the
 *    exterior sentinel (README.md:407); face CSR is [cells][4] in
 *    l, r, b, t order (preprocess/domain.py:83-174); topology is
 *    [sides][3] = (orient, lower, higher) (preprocess/domain.py:452-460).
 *  - Large arrays are DEVICE pointers owned by the caller (for example
 *    torch CUDA tensors) and must stay alive until nhf_destroy. Scalars,
 *    forcing coefficients, clock words, traces and budget totals are HOST
 *    pointers.
 *  - All device work is ordered after the caller's stream (given at
 *    nhf_create) and the caller's stream is ordered after it, so tensors
 *    written by the caller are visible to the next call and vice versa.
 *  - Every function returns NHF_OK (0) or a negative NHF_E* code; the
 *    message is in nhf_last_error(handle) (or nhf_last_error(NULL) when
 *    creation failed). Device clock statuses are reported, as in the
 *    reference, in column 3 of the batch trace (core/clock.py:42-46).
 *  - One host thread per handle; handles on different streams may run
 *    concurrently.
 */
#ifndef NHFLOOD_H
#define NHFLOOD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NHF_OK 0
#define NHF_EINVAL (-1)
#define NHF_ECUDA (-2)
#define NHF_ENOMEM (-3)
#define NHF_ESTATE (-4)

/* Trace columns: the reference's nine (core/clock.py:35-40) plus the number
 * of wet cells (depth >= min_h, solver_compact.py:359) after the step. */
#define NHF_TRACE_COLS 10
#define NHF_MAX_BATCH 64

/* Clock status values in trace column 3 (core/clock.py:42-46). */
#define NHF_STEP_DONE 0
#define NHF_STEP_COMPLETED 1
#define NHF_STEP_BAD_CFL 2
#define NHF_STEP_BAD_DT 3
#define NHF_STEP_OVERSHOOT 4

/* The physics type of the build. The step computes in F32 as the
 * reference's fields do (libnhflood.so). Compiled with -DNHF_REAL_DOUBLE, the
 * same multi-pass kernels compute in F64 instead (libnhflood_f64.so): the
 * FP64 build the precision study compares the F32 state with. Every array
 * below typed nhf_real is F64 there; the clock (dt, its fixed-point words,
 * the trace) stays F32 in both, and the budget partials are FP64 in both. */
#ifdef NHF_REAL_DOUBLE
typedef double nhf_real;
#else
typedef float nhf_real;
#endif

typedef struct nhf_mesh {
    int32_t e_num;      /* cells including sentinel 0 */
    int32_t s_num;      /* sides including sentinel 0 */
    int32_t b_num;      /* boundaries (level or discharge) */
    int32_t n_rates;    /* unique rain pixels */
    int32_t isl_len;    /* length of isl_data */
    int32_t hang_cells; /* hanging-edge gradient cells (0: aligned mesh) */
    int32_t hang_edges; /* hanging edges */
    /* static cell arrays [e_num], device */
    const nhf_real *x, *y, *area, *width, *height;
    const nhf_real *f0, *fc, *k; /* Horton, m/s and 1/h (hydraulics.py:63-93) */
    const nhf_real *weight;      /* boundary cell weight */
    const int32_t *boundary_id, *rain_index;
    const int32_t *face_ptr, *face_count; /* [e_num*4] */
    const int32_t *isl_data;              /* [isl_len] */
    /* static side arrays [s_num], device */
    const int32_t *topology; /* [s_num*3] */
    const nhf_real *length, *side_n;
    const uint8_t *sbf; /* 1 = closed exterior side */
    /* boundaries [max(1,b_num)], device: 0 level, 1 discharge */
    const int32_t *kind;
    /* theta < 1 only: open-face fractions [e_num*4], device (NULL if theta == 1) */
    const nhf_real *open_face;
    /* hanging-edge reconstruction (core/pressure.py:19-45), device */
    const int32_t *edge_index; /* [s_num] */
    const nhf_real *offsets;   /* [hang_edges*2] */
    const int32_t *slots;      /* [hang_edges*2] */
    const int32_t *hcells;     /* [hang_cells] */
    const int32_t *axes;       /* [hang_cells*2] */
    /* mutable state, device */
    nhf_real *bed, *depth, *q, *rain_time, *infiltration, *max_depth, *max_speed, *u, *v;
    uint32_t *peak_hi, *peak_lo;
} nhf_mesh;

typedef struct nhf_params {
    nhf_real g;       /* 9.81 */
    nhf_real afa;     /* Courant number */
    nhf_real sita;    /* theta time weighting */
    nhf_real min_h;   /* wet threshold */
    float min_dt;     /* F32(1e-4) CFL floor (solver_compact.py:31) */
    int32_t batch_size; /* steps per batch, 1..64 (clock.py:48-51) */
    int32_t path;       /* 0: the lattice form on a uniform grid it covers
                           of at least 2^20 cells, else the fused tiled step
                           when the mesh allows it,
                           else multi-pass; 1: always the multi-pass step;
                           2: the lattice form when the mesh allows it, else
                           multi-pass; 3: the fused tiled step (tile size by
                           mesh size) when the mesh allows it, else multi-pass;
                           256, 512 or 1024: fused tiled step with that tile
                           size when the mesh allows it, else multi-pass */
    int32_t cfl_mode;   /* fused step only. 0: the next step's CFL candidate
                           in the step itself on meshes of less than two
                           waves of tiles, else a separate pass after it;
                           1: always in the step; 2: always a separate pass
                           (ensemble members, whose launches span all
                           members) */
} nhf_params;

typedef struct nhf_handle nhf_handle;

/* Allocate the step's scratch (donor factors, reductions, budget partials,
 * clock control block, trace) and capture nothing yet. `stream` is the
 * caller's cudaStream_t (NULL: legacy default stream). Replaces the field
 * allocation and ti.graph build in solver_compact.py:209-336,894-909. */
int nhf_create(const nhf_mesh *mesh, const nhf_params *params, void *stream, nhf_handle **out);
int nhf_destroy(nhf_handle *h);
const char *nhf_last_error(const nhf_handle *h);
const char *nhf_version(void);
/* sizeof(nhf_real) of this build: 4, or 8 for the FP64 build. */
int nhf_real_bytes(void);

/* initialize() (solver_compact.py:398-410): depth = 0, infiltration = f0,
 * per-side centre distance. */
int nhf_initialize(nhf_handle *h);
/* Clock words (clock.py:60-69): set after a checkpoint restore. */
int nhf_set_clock(nhf_handle *h, const uint32_t now[2]);
int nhf_get_clock(nhf_handle *h, uint32_t now[2]);
/* clock.active[None] = 1 before the first compute_cfl (solver_compact.py:884). */
int nhf_set_active(nhf_handle *h, int32_t active);
/* upload_forcing (solver_compact.py:769-790): coefficients [max(1,b_num)][2]
 * and rain rates [n_rates], both host nhf_real; rain_rates may be NULL to
 * keep the previous rates. */
int nhf_set_forcing(nhf_handle *h, const nhf_real *coefficients, const nhf_real *rain_rates, int32_t raining);
/* apply_initial_levels (solver_compact.py:412-420, 876-883): targets is a
 * device [e_num] nhf_real array; the level diagnostics enter the budget. */
int nhf_apply_initial_levels(nhf_handle *h, const nhf_real *targets);
/* compute_cfl (solver_compact.py:617-641). */
int nhf_compute_cfl(nhf_handle *h);
/* initial_diagnostics (solver_compact.py:657-672). */
int nhf_initial_diagnostics(nhf_handle *h);
/* reset_extrema (solver_compact.py:674-679). */
int nhf_reset_extrema(nhf_handle *h);
/* clock.begin + graph.run + clock.read_trace (clock.py:75-92,187-203;
 * solver_compact.py:939-942): runs batch_size prepare/tick/cfl/finish steps
 * towards `target` ticks with batch origin `origin` (two U32 words each,
 * host) and copies the [batch_size][NHF_TRACE_COLS] trace to `trace` (host).
 * Synchronous. */
int nhf_run_batch(nhf_handle *h, const uint32_t target[2], const uint32_t origin[2], uint32_t *trace);
/* Same batch without the host synchronisation: the trace stays on the
 * device until nhf_read_trace (which synchronises). */
int nhf_run_batch_async(nhf_handle *h, const uint32_t target[2], const uint32_t origin[2]);
int nhf_read_trace(nhf_handle *h, uint32_t *trace);
/* DeviceBudget.flush (device_budget.py:68-84): adds this interval's FP64
 * per-block partials into totals[4 + 6*b_num] (host) and clears them. */
int nhf_budget_flush(nhf_handle *h, double *totals);
int nhf_budget_terms(const nhf_handle *h);
/* ndt_t / cfl_arg_t / flow_depth_t[cfl_arg] (solver_compact.py:644-655). */
int nhf_get_cfl(nhf_handle *h, nhf_real *ndt, int32_t *arg, nhf_real *flow_depth);
/* limit_value_t / limit_ids_t (solver_compact.py:330-331,839,854). */
int nhf_limits(nhf_handle *h, nhf_real values[5], int32_t ids[3]);
int nhf_reset_limits(nhf_handle *h);
/* sample_stations (solver_compact.py:681-687): ids host [n], out host [n][4]
 * = depth, level, u, v. */
int nhf_sample_stations(nhf_handle *h, const int32_t *ids, int32_t n, nhf_real *out);
/* Face flux sums eq_t [e_num][4] (device destination). */
int nhf_read_eq(nhf_handle *h, nhf_real *eq);
/* Hanging-edge gradients [hang_cells][2] (device destination). */
int nhf_read_gradients(nhf_handle *h, nhf_real *gradients);
int nhf_synchronize(nhf_handle *h);
/* The library's own stream (cudaStream_t) on which every batch runs; lets a
 * caller time batches with events on the launching stream. */
void *nhf_stream(nhf_handle *h);
/* Which step form the handle runs ("tiled(...)" or "multipass (reason)"). */
const char *nhf_path(const nhf_handle *h);

/* Gate controller (core/gate.py:35-206; the step graph's check_gates,
 * clear/collect_gate_budget, measure_pond_inventory and finish_gate_bed
 * passes, solver_compact.py:896-906, and the record_flux / record_cell hooks
 * in tick, :523-524 and :595-604). Every array is a DEVICE pointer owned by
 * the caller and alive until nhf_destroy; the controller words are read and
 * restored by the caller directly (snapshot/restore, gate.py:195-215).
 * While attached, every step checks the triggers and moves the gate beds at
 * its start, records the post-limiter exchange volumes and the pond and
 * gate-cell source terms, and moves the beds to the step end before the CFL.
 * Terms (10 count + 8, the reference's order): per gate pond in/out, river
 * in/out; overtopping in/out and the pond's six source terms (rain,
 * infiltration, positivity, pipe, boundary, rounding); per gate the
 * channel's six source terms. Gates run on the multi-pass step (path 1) or on
 * the fused step with 256-cell tiles and the separate CFL pass (path 256,
 * cfl_mode 2); the source terms then come from the fused depth update. */
typedef struct nhf_gate {
    int32_t count;           /* gates */
    int32_t n_targets;       /* gate cells */
    int32_t n_flux;          /* recorded sides */
    const int32_t *cell_gate;  /* [e_num] gate of each cell, -1 off gates */
    const int32_t *pond;       /* [e_num] 1 on pond cells, 0 at the sentinel */
    const nhf_real *closed;    /* [e_num] closed (initial) bed */
    const int32_t *targets;    /* [n_targets] gate cells, gate by gate */
    const int32_t *controls;   /* [count] control cell of each gate */
    const int32_t *flux_sides; /* [n_flux] sides between gate and non-gate cells, or pond and non-pond cells */
    uint32_t formal_tick[2];   /* clock words of formal time 0 (control starts there) */
    float trigger_level, opening_seconds, open_elevation;
    int32_t *commanded, *flow_seen, *opened;     /* [count] controller words */
    uint32_t *command, *first_flow, *opened_at;  /* [count][2] clock words */
} nhf_gate;
int nhf_gate_attach(nhf_handle *h, const nhf_gate *gate);
/* check_gates at run start (solver_compact.py:885-888): trigger check and
 * bed motion at the current clock. */
int nhf_gate_check(nhf_handle *h);
int nhf_gate_terms(const nhf_handle *h);
/* controller.budget.flush: this interval's totals [nhf_gate_terms] (host),
 * FP64 per-block partials merged in block order; clears them. */
int nhf_gate_flush(nhf_handle *h, double *totals);

/* Ensemble (batched) form. The reference runs one domain per process
 * (solver_compact.py:179-1008); an ensemble advances many member handles
 * together, one fused step launch per slot for all of them, each member
 * with its own clock, CFL dt, limiter statistics, budget and extrema.
 * For the single-launch schedules members must run the fused tiled step
 * with one tile size (nhf_params.path = that size, cfl_mode 2), one batch
 * size and one theta class (= 1 or < 1). A batch
 * starts after the work queued so far on `stream` and on every member's
 * creation stream, and those streams wait for the batch. Everything else
 * about a member (forcing, clock, budget flush, stations, CFL read-back)
 * still goes through its own handle between batches. grid_blocks: 0 =
 * persistent grid (resident blocks per SM x SMs), -1 = one block per tile,
 * > 0 = that many blocks; -2 = member graphs: every member runs its own
 * batch graph (its own step form, tile size and CFL placement) on its own
 * stream, all members launched together; members then need to share only
 * the batch size. A member with a gate controller (nhf_gate_attach) runs
 * only in the member-graph schedule: the one-launch step has no gate passes,
 * so creating it with such a member fails with NHF_EINVAL, and a batch of it
 * after a member attached one fails with NHF_ESTATE. */
typedef struct nhf_ensemble nhf_ensemble;
int nhf_ensemble_create(nhf_handle *const *members, int32_t n, int32_t grid_blocks, void *stream,
                        nhf_ensemble **out);
int nhf_ensemble_destroy(nhf_ensemble *e);
const char *nhf_ensemble_last_error(const nhf_ensemble *e);
/* info: members, tile, grid blocks, tiles of all members, batch size,
 * shared bytes per block. */
int nhf_ensemble_info(const nhf_ensemble *e, int32_t info[6]);
void *nhf_ensemble_stream(const nhf_ensemble *e);
/* One batch of every member: targets/origins are host [n][2] tick words
 * (clock.begin per member); trace is host [n][batch_size][NHF_TRACE_COLS]. */
int nhf_ensemble_run_batch(nhf_ensemble *e, const uint32_t *targets, const uint32_t *origins, uint32_t *trace);
int nhf_ensemble_run_batch_async(nhf_ensemble *e, const uint32_t *targets, const uint32_t *origins);
int nhf_ensemble_read_trace(nhf_ensemble *e, uint32_t *trace);

/* No counterpart in the reference: an allocation-free CFL candidate for
 * callers that may not allocate device memory (a host that reserves its HBM
 * budget once at start-up, such as a serving process or a model coupler that
 * hands out fixed pools). Same result as nhf_compute_cfl + nhf_get_cfl on
 * the given state: ndt_out = min over interior sides of
 * afa * L / (sqrt(g h) + |q| / h), arg_out = the lowest side id attaining it
 * (+inf and 0 without interior sides); both outputs are DEVICE pointers, as
 * are all inputs, and the call is asynchronous on `stream`. It allocates
 * nothing: its scratch is a fixed 256 KiB array compiled into the library
 * (held by every device that loads it until exit), which limits it to
 * 67,108,864 sides (larger meshes: NHF_EINVAL). The first call on each
 * device looks up that array's device address and must come before any
 * stream capture; later calls re-check that address and look it up again
 * after a context reset. Calls share the array: calls that overlap on the GPU
 * race. Host pointers are refused (NHF_EINVAL) before any launch.
 * nhf_cfl_noalloc_error() describes the calling thread's last failure. */
int nhf_cfl_noalloc(const int32_t *topology, const float *bed, const float *depth, const float *length,
                    const float *q, int32_t s_num, float afa, float g, void *stream, float *ndt_out,
                    int32_t *arg_out);
const char *nhf_cfl_noalloc_error(void);

#ifdef __cplusplus
}
#endif
#endif
