/*
 * ORACLE — test infrastructure only (see step_ref.h). Only tests/, the smoke
 * check and bench.py's CPU-baseline leg load this library, as a checker or a
 * timed CPU baseline; the product never links it.
 *
 * Restated from the reference (paths relative to the nh-flood-2d repo):
 *   clock          core/clock.py:94-181            (choose, commit)
 *   prepare_step   core/solver_compact.py:364-382
 *   finish_step    core/solver_compact.py:384-391
 *   initialize     core/solver_compact.py:398-410
 *   initial levels core/solver_compact.py:412-420
 *   tick           core/solver_compact.py:422-613
 *   compute_cfl    core/solver_compact.py:617-641
 *   diagnostics    core/solver_compact.py:657-679
 *   pressure       core/pressure.py:65-129
 *   face_discharge, boundary_neighbor_sum  core/solver_compact.py:118-149
 *   gate controller core/gate.py:68-206; its passes in the step graph
 *                  core/solver_compact.py:896-906, hooks 523-524, 595-604
 * Pass structure and operation order follow the reference literally. Scalar
 * constants are F32 (Taichi default_fp); Python-only constant expressions
 * such as (1 - sita) / 2 are folded in F64 first, as Taichi folds them.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "step_ref.h"

#define DONE 0u
#define COMPLETED 1u
#define BAD_CFL 2u
#define BAD_DT 3u
#define OVERSHOOT 4u
#define SNAP_TICKS 1099512u /* ceil(1e-6 * 2**40), clock.py:11 */
#define BLOCK 256

typedef ora_real real;
#ifdef ORA_REAL_DOUBLE
#define R(x) x
#define RABS(x) fabs(x)
#define RSQRT(x) sqrt(x)
#define RPOW(x, y) ora_pow(x, y) /* the FP64 series of mathref.c, as the CUDA FP64 build */
#define REXP(x) ora_exp(x)
#else
#define R(x) x##f
#define RABS(x) fabsf(x)
#define RSQRT(x) sqrtf(x)
#define RPOW(x, y) ora_powf(x, y)
#define REXP(x) ora_expf(x)
#endif

static inline real maxf(real a, real b) { return a > b ? a : b; }
static inline real minf(real a, real b) { return b < a ? b : a; }
static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

struct ora_ctx {
    ora_mesh m;
    int terms, blocks;
    /* clock (clock.py:60-68) */
    uint32_t now[2], next[2], origin[2], step_end[2];
    float dt, local, end_local;  /* the clock's F32 values */
    int active, slot;
    /* scalars */
    real ndt;
    int32_t cfl_arg;
    uint32_t limited_cells, limited_faces;
    real minimum_scale;
    uint32_t wet;
    real limit_value[5];
    int32_t limit_ids[3];
    int raining;
    /* per-boundary */
    real *coefficients, *values, *level_values;
    const real *rain_rates_ext;
    real *rain_rates;
    /* work */
    real *sdc, *dh, *eq, *increment, *rain_depth, *donor_scale, *cfl, *flow_depth, *face_qn, *ssq;
    real *gradients;
    real *diag;      /* [blocks*terms] per-step f32 values per cell collected per block */
    double *acc_sum, *acc_comp; /* [blocks*terms] */
    uint32_t *trace;  /* [batch][10] */
    /* gate controller */
    int gate_on, gterms, gblocks;
    ora_gate gate;
    double *gacc_sum, *gacc_comp; /* [gblocks*gterms] */
};

void ora_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

ora_ctx *ora_create(const ora_mesh *mesh)
{
    ora_ctx *c = (ora_ctx *)calloc(1, sizeof(ora_ctx));
    c->m = *mesh;
    int e = mesh->e_num, s = mesh->s_num, b = mesh->b_num;
    c->terms = 4 + 6 * b;
    c->blocks = (e + BLOCK - 1) / BLOCK;
    int bb = b > 0 ? b : 1;
    c->coefficients = (real *)calloc((size_t)bb * 2, sizeof(real));
    c->values = (real *)calloc(bb, sizeof(real));
    c->level_values = (real *)calloc(bb, sizeof(real));
    c->rain_rates = (real *)calloc(mesh->n_rates > 0 ? mesh->n_rates : 1, sizeof(real));
    c->sdc = (real *)calloc(s, sizeof(real));
    c->dh = (real *)calloc(s, sizeof(real));
    c->eq = (real *)calloc((size_t)e * 4, sizeof(real));
    c->increment = (real *)calloc(e, sizeof(real));
    c->rain_depth = (real *)calloc(e, sizeof(real));
    c->donor_scale = (real *)calloc(e, sizeof(real));
    c->cfl = (real *)calloc(s, sizeof(real));
    c->flow_depth = (real *)calloc(s, sizeof(real));
    c->face_qn = (real *)calloc((size_t)e * 4, sizeof(real));
    c->ssq = (real *)calloc(e, sizeof(real));
    c->gradients = (real *)calloc((size_t)(mesh->hang_cells > 0 ? mesh->hang_cells : 1) * 2, sizeof(real));
    c->acc_sum = (double *)calloc((size_t)c->blocks * c->terms, sizeof(double));
    c->acc_comp = (double *)calloc((size_t)c->blocks * c->terms, sizeof(double));
    c->trace = (uint32_t *)calloc((size_t)mesh->batch_size * ORA_TRACE_COLS, sizeof(uint32_t));
    c->limit_value[0] = INFINITY;
    return c;
}

void ora_destroy(ora_ctx *c)
{
    if (!c) return;
    free(c->coefficients); free(c->values); free(c->level_values); free(c->rain_rates);
    free(c->sdc); free(c->dh); free(c->eq); free(c->increment); free(c->rain_depth);
    free(c->donor_scale); free(c->cfl); free(c->flow_depth); free(c->face_qn); free(c->ssq);
    free(c->gradients); free(c->acc_sum); free(c->acc_comp); free(c->trace);
    free(c->gacc_sum); free(c->gacc_comp);
    free(c);
}

void ora_set_clock(ora_ctx *c, const uint32_t now[2]) { c->now[0] = now[0]; c->now[1] = now[1]; }
void ora_get_clock(const ora_ctx *c, uint32_t now[2]) { now[0] = c->now[0]; now[1] = c->now[1]; }
void ora_set_active(ora_ctx *c, int active) { c->active = active; }
int ora_budget_terms(const ora_ctx *c) { return c->terms; }
real ora_ndt(const ora_ctx *c) { return c->ndt; }
void ora_set_ndt(ora_ctx *c, float ndt) { c->ndt = ndt; }
int32_t ora_cfl_arg(const ora_ctx *c) { return c->cfl_arg; }

void ora_limits(const ora_ctx *c, real values[5], int32_t ids[3])
{
    memcpy(values, c->limit_value, sizeof(c->limit_value));
    memcpy(ids, c->limit_ids, sizeof(c->limit_ids));
}

void ora_reset_limits(ora_ctx *c) { c->limit_value[0] = INFINITY; }

void ora_read_eq(const ora_ctx *c, real *eq) { memcpy(eq, c->eq, sizeof(real) * 4 * (size_t)c->m.e_num); }
void ora_read_flow_depth(const ora_ctx *c, real *out) { memcpy(out, c->flow_depth, sizeof(real) * (size_t)c->m.s_num); }
void ora_read_gradients(const ora_ctx *c, real *out)
{
    if (c->m.hang_cells > 0) memcpy(out, c->gradients, sizeof(real) * 2 * (size_t)c->m.hang_cells);
}

void ora_set_forcing(ora_ctx *c, const real *coefficients, const real *rain_rates, int raining)
{
    int bb = c->m.b_num > 0 ? c->m.b_num : 1;
    if (coefficients) memcpy(c->coefficients, coefficients, sizeof(real) * 2 * (size_t)bb);
    if (rain_rates && c->m.n_rates > 0) memcpy(c->rain_rates, rain_rates, sizeof(real) * (size_t)c->m.n_rates);
    c->raining = raining;
}

/* ---- budget: FP64 per-block partials ------------------------------------ */

/* Canonical pairwise tree over one 256-slot block: stride 128 .. 1,
 * slot i += slot i + stride. */
static double block_tree(double *v)
{
    for (int stride = BLOCK / 2; stride >= 1; stride >>= 1)
        for (int i = 0; i < stride; ++i) v[i] += v[i + stride];
    return v[0];
}

static void acc_add(ora_ctx *c, size_t idx, double p)
{
    double sum = c->acc_sum[idx];
    double s = sum + p;
    double bp = s - sum;
    double err = (sum - (s - bp)) + (p - bp);
    c->acc_comp[idx] += err;
    c->acc_sum[idx] = s;
}

/* Reduce a per-cell diagnostic matrix diag[cell*terms + term] (0 where the
 * reference skips add_diagnostic because value == 0) into the accumulator. */
static void collect(ora_ctx *c, const real *diag)
{
    int T = c->terms, e = c->m.e_num;
#pragma omp parallel for schedule(static)
    for (int blk = 0; blk < c->blocks; ++blk) {
        double v[BLOCK];
        for (int t = 0; t < T; ++t) {
            int any = 0;
            for (int i = 0; i < BLOCK; ++i) {
                int ei = blk * BLOCK + i;
                real val = ei < e ? diag[(size_t)ei * T + t] : R(0.0);
                v[i] = val != R(0.0) ? (double)val : 0.0;
                any |= val != R(0.0);
            }
            if (!any) continue;
            acc_add(c, (size_t)blk * T + t, block_tree(v));
        }
    }
}

void ora_budget_flush(ora_ctx *c, double *totals)
{
    /* Per-term sum over blocks of (sum + comp) pairs, added in block order
     * with Neumaier compensation; the host-side merge. */
    int T = c->terms;
    for (int t = 0; t < T; ++t) {
        double s = 0.0, comp = 0.0;
        for (int blk = 0; blk < c->blocks; ++blk) {
            double parts[2] = {c->acc_sum[(size_t)blk * T + t], c->acc_comp[(size_t)blk * T + t]};
            for (int j = 0; j < 2; ++j) {
                double p = parts[j];
                double n = s + p;
                if (fabs(s) >= fabs(p)) comp += (s - n) + p; else comp += (p - n) + s;
                s = n;
            }
        }
        totals[t] = s + comp;
    }
    memset(c->acc_sum, 0, sizeof(double) * (size_t)c->blocks * T);
    memset(c->acc_comp, 0, sizeof(double) * (size_t)c->blocks * T);
}

/* ---- gate controller (core/gate.py:68-206) ------------------------------ */

void ora_gate_attach(ora_ctx *c, const ora_gate *gate)
{
    c->gate = *gate;
    c->gate_on = 1;
    c->gterms = 10 * gate->count + 8;
    int flux_blocks = (gate->n_flux + BLOCK - 1) / BLOCK;
    c->gblocks = flux_blocks > c->blocks ? flux_blocks : c->blocks;
    free(c->gacc_sum); free(c->gacc_comp);
    c->gacc_sum = (double *)calloc((size_t)c->gblocks * c->gterms, sizeof(double));
    c->gacc_comp = (double *)calloc((size_t)c->gblocks * c->gterms, sizeof(double));
}

int ora_gate_terms(const ora_ctx *c) { return c->gate_on ? c->gterms : 0; }

static void gate_acc_add(ora_ctx *c, int blk, int term, double p)
{
    size_t idx = (size_t)blk * c->gterms + term;
    double sum = c->gacc_sum[idx];
    double s = sum + p;
    double bp = s - sum;
    double err = (sum - (s - bp)) + (p - bp);
    c->gacc_comp[idx] += err;
    c->gacc_sum[idx] = s;
}

/* since_command (gate.py:68-73): clock age of the command in F32 seconds */
static float since_command(const ora_gate *g, int gate, uint32_t hi, uint32_t lo)
{
    uint32_t borrow = lo < g->command[2 * gate + 1] ? 1u : 0u;
    uint32_t high = hi - g->command[2 * gate] - borrow;
    uint32_t low = lo - g->command[2 * gate + 1];
    return (float)high / 256.0f + (float)low * 0x1p-40f;
}

/* move (gate.py:75-86): the working bed of every commanded gate at (hi, lo) */
static void gate_move(ora_ctx *c, uint32_t hi, uint32_t lo)
{
    const ora_gate *g = &c->gate;
    if (!c->active) return;
    for (int slot = 0; slot < g->n_targets; ++slot) {
        int cell = g->targets[slot];
        int gate = g->cell_gate[cell];
        if (g->commanded[gate] != 1) continue;
        float fraction = minf(since_command(g, gate, hi, lo) / g->opening_seconds, 1.0f);
        if (fraction >= 1.0f) {
            c->m.bed[cell] = (real)g->open_elevation;
            if (!g->opened[gate]) {
                g->opened[gate] = 1;
                g->opened_at[2 * gate] = hi; g->opened_at[2 * gate + 1] = lo;
            }
        } else {
            real closed = g->closed[cell];
            c->m.bed[cell] = closed + ((real)g->open_elevation - closed) * (real)fraction;
        }
    }
}

/* check (gate.py:88-99): irreversible command once the control cell is wet
 * and its level exceeds the trigger, from formal time 0 on; then move */
void ora_gate_check(ora_ctx *c)
{
    const ora_gate *g = &c->gate;
    const ora_mesh *m = &c->m;
    if (!c->gate_on || !c->active) return;
    uint32_t hi = c->now[0], lo = c->now[1];
    int formal = hi > g->formal_tick[0] || (hi == g->formal_tick[0] && lo >= g->formal_tick[1]);
    for (int gate = 0; gate < g->count && formal; ++gate) {
        int cell = g->controls[gate];
        if (g->commanded[gate] == 0 && m->depth[cell] >= m->min_h
            && m->bed[cell] + m->depth[cell] > (real)g->trigger_level) {
            g->commanded[gate] = 1;
            g->command[2 * gate] = hi; g->command[2 * gate + 1] = lo;
        }
    }
    gate_move(c, hi, lo);
}

/* record_flux (gate.py:118-140) over the recorded sides after the limiter:
 * term and value pairs of one side; at most two are nonzero. */
static int gate_flux_terms(ora_ctx *c, int si, int terms[2], real values[2])
{
    const ora_gate *g = &c->gate;
    const ora_mesh *m = &c->m;
    int left = m->topology[3 * si + 1], right = m->topology[3 * si + 2];
    real volume = m->q[si] * m->length[si] * c->dt;
    int gl = g->cell_gate[left], gr = g->cell_gate[right];
    int pl = g->pond[left], pr = g->pond[right];
    int term = -1, latch = -1;
    real into = R(0.0);
    if (gl >= 0 && gr < 0) {
        if (pr == 1) { term = 4 * gl; into = volume; latch = gl; }
        else { term = 4 * gl + 2; into = -volume; }
    } else if (gr >= 0 && gl < 0) {
        if (pl == 1) { term = 4 * gr; into = -volume; latch = gr; }
        else { term = 4 * gr + 2; into = volume; }
    } else if (pl != pr) {
        term = 4 * g->count;
        into = pr == 1 ? volume : -volume;
    }
    if (latch >= 0 && volume != R(0.0) && !g->flow_seen[latch]) {
        g->flow_seen[latch] = 1;
        g->first_flow[2 * latch] = c->step_end[0]; g->first_flow[2 * latch + 1] = c->step_end[1];
    }
    terms[0] = term; terms[1] = term + 1;
    values[0] = maxf(into, R(0.0));
    values[1] = maxf(-into, R(0.0));
    return term >= 0;
}

static void gate_record_fluxes(ora_ctx *c)
{
    const ora_gate *g = &c->gate;
    int nblk = (g->n_flux + BLOCK - 1) / BLOCK;
    int T = 4 * g->count + 2;  /* exchange terms */
    real *vals = (real *)calloc((size_t)BLOCK * T, sizeof(real));
    for (int blk = 0; blk < nblk; ++blk) {
        memset(vals, 0, sizeof(real) * (size_t)BLOCK * T);
        for (int i = 0; i < BLOCK; ++i) {
            int p = blk * BLOCK + i;
            if (p >= g->n_flux) break;
            int terms[2]; real values[2];
            if (!gate_flux_terms(c, g->flux_sides[p], terms, values)) continue;
            vals[(size_t)i * T + terms[0]] = values[0];
            vals[(size_t)i * T + terms[1]] = values[1];
        }
        double v[BLOCK];
        for (int t = 0; t < T; ++t) {
            int any = 0;
            for (int i = 0; i < BLOCK; ++i) {
                real val = vals[(size_t)i * T + t];
                v[i] = (double)val;
                any |= val != R(0.0);
            }
            if (any) gate_acc_add(c, blk, t, block_tree(v));
        }
    }
    free(vals);
}

/* source_offset (gate.py:142-149): first of the six source terms of a pond
 * or gate cell, -1 elsewhere */
static int gate_source_offset(const ora_ctx *c, int cell)
{
    const ora_gate *g = &c->gate;
    if (g->pond[cell] == 1) return 4 * g->count + 2;
    if (g->cell_gate[cell] >= 0) return 4 * g->count + 8 + 6 * g->cell_gate[cell];
    return -1;
}

void ora_gate_flush(ora_ctx *c, double *totals)
{
    int T = c->gterms;
    for (int t = 0; t < T; ++t) {
        double s = 0.0, comp = 0.0;
        for (int blk = 0; blk < c->gblocks; ++blk) {
            double parts[2] = {c->gacc_sum[(size_t)blk * T + t], c->gacc_comp[(size_t)blk * T + t]};
            for (int j = 0; j < 2; ++j) {
                double p = parts[j];
                double n = s + p;
                if (fabs(s) >= fabs(p)) comp += (s - n) + p; else comp += (p - n) + s;
                s = n;
            }
        }
        totals[t] = s + comp;
    }
    memset(c->gacc_sum, 0, sizeof(double) * (size_t)c->gblocks * T);
    memset(c->gacc_comp, 0, sizeof(double) * (size_t)c->gblocks * T);
}

/* ---- setup kernels -------------------------------------------------------- */

void ora_initialize(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
    for (int ei = 1; ei < m->e_num; ++ei) {
        m->depth[ei] = R(0.0);
        m->infiltration[ei] = m->f0[ei];
    }
    for (int si = 1; si < m->s_num; ++si) {
        c->dh[si] = -R(999.0);
        int so = m->topology[3 * si], el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        if (so == 2) c->sdc[si] = maxf(RABS(m->x[eh] - m->x[el]), R(0.01));
        else c->sdc[si] = maxf(RABS(m->y[eh] - m->y[el]), R(0.01));
    }
}

void ora_apply_initial_levels(ora_ctx *c, const real *targets)
{
    const ora_mesh *m = &c->m;
    int T = c->terms;
    real *diag = (real *)calloc((size_t)m->e_num * T, sizeof(real));
    for (int ei = 1; ei < m->e_num; ++ei) {
        int bi = m->boundary_id[ei];
        if (bi >= 0 && m->kind[bi] == 0) {
            real previous = m->depth[ei];
            m->depth[ei] = targets[ei];
            diag[(size_t)ei * T + 4 + 5 * bi] = (m->depth[ei] - previous) * m->area[ei];
        }
    }
    collect(c, diag);
    free(diag);
}

static void velocity(const ora_ctx *c, int ei, real *u, real *v)
{
    const ora_mesh *m = &c->m;
    real h = maxf(m->depth[ei], R(0.01));
    *u = R(0.0); *v = R(0.0);
    if (m->depth[ei] >= m->min_h) {
        *u = (c->eq[4 * ei + 0] + c->eq[4 * ei + 1]) / m->height[ei] / h / R(2.0);
        *v = (c->eq[4 * ei + 2] + c->eq[4 * ei + 3]) / m->width[ei] / h / R(2.0);
    }
}

void ora_compute_cfl(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
    if (!c->active) return;
    real ndt = INFINITY;
#pragma omp parallel for schedule(static) reduction(min : ndt)
    for (int si = 1; si < m->s_num; ++si) {
        int el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        c->cfl[si] = INFINITY;
        if (el != 0 && eh != 0) {
            real head = maxf(m->bed[el] + m->depth[el], m->bed[eh] + m->depth[eh]);
            real h = maxf(head - maxf(maxf(m->bed[el], m->bed[eh]), c->dh[si]), R(0.01));
            c->flow_depth[si] = h;
            real val = m->afa * m->length[si] / (RSQRT(m->g * h) + RABS(m->q[si]) / h);
            c->cfl[si] = val;
            ndt = minf(ndt, val);
        }
    }
    c->ndt = ndt;
    int32_t arg = m->s_num;
#pragma omp parallel for schedule(static) reduction(min : arg)
    for (int si = 1; si < m->s_num; ++si) {
        if (c->cfl[si] == c->ndt && m->topology[3 * si + 1] != 0 && m->topology[3 * si + 2] != 0)
            if (si < arg) arg = si;
    }
    c->cfl_arg = arg == m->s_num ? 0 : arg;
}

void ora_initial_diagnostics(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
#pragma omp parallel for schedule(static)
    for (int ei = 1; ei < m->e_num; ++ei) {
        for (int d = 0; d < 4; ++d) {
            real total = R(0.0);
            int p = m->face_ptr[4 * ei + d];
            for (int j = 0; j < m->face_count[4 * ei + d]; ++j) {
                int si = m->isl_data[p + j];
                total += m->q[si] * m->length[si];
            }
            c->eq[4 * ei + d] = total;
        }
        real u, v;
        velocity(c, ei, &u, &v);
        m->u[ei] = u; m->v[ei] = v;
        m->max_speed[ei] = maxf(m->max_speed[ei], RSQRT(u * u + v * v));
        if (m->depth[ei] > m->max_depth[ei]) {
            m->max_depth[ei] = m->depth[ei];
            m->peak_hi[ei] = c->now[0]; m->peak_lo[ei] = c->now[1];
        }
    }
}

void ora_reset_extrema(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
    for (int ei = 1; ei < m->e_num; ++ei) {
        m->max_depth[ei] = m->depth[ei];
        m->max_speed[ei] = RSQRT(m->u[ei] * m->u[ei] + m->v[ei] * m->v[ei]);
        m->peak_hi[ei] = c->now[0]; m->peak_lo[ei] = c->now[1];
    }
}

/* ---- clock (clock.py:94-181) --------------------------------------------- */

static void clock_choose(ora_ctx *c, float candidate, int slot)
{
    uint32_t *row = c->trace + (size_t)slot * ORA_TRACE_COLS;
    c->active = 0; c->dt = 0.0f; c->local = 0.0f; c->end_local = 0.0f;
    uint32_t now_hi = c->now[0], now_lo = c->now[1];
    uint32_t target_hi = c->next[0], target_lo = c->next[1];
    if (!(now_hi < target_hi || (now_hi == target_hi && now_lo < target_lo))) return;
    if (!(candidate >= c->m.min_dt)) { row[3] = BAD_CFL; return; }
    uint32_t borrow = now_lo > target_lo ? 1u : 0u;
    uint32_t rem_hi = target_hi - now_hi - borrow;
    uint32_t rem_lo = target_lo - now_lo;
    float remaining = (float)rem_hi * (1.0f / 256.0f) + (float)rem_lo * 0x1p-40f;
    float chosen = minf(minf(candidate, 1.0f), remaining);
    row[4] = fbits(candidate);
    row[5] = chosen < minf(candidate, 1.0f) ? 1u : 0u;
    uint32_t bits = fbits(chosen);
    int exponent = (int)((bits >> 23) & 255u) - 127;
    uint32_t mantissa = (bits & 0x7fffffu) | 0x800000u;
    uint32_t dt_hi = 0, dt_lo = 0;
    if (!(chosen > 0.0f) || exponent < -40 || exponent > 0) { row[3] = BAD_DT; return; }
    int shift = exponent + 17;
    if (shift >= 0) {
        dt_lo = mantissa << shift;
        if (shift >= 9) dt_hi = mantissa >> (32 - shift);
    } else {
        int right = -shift;
        dt_lo = mantissa >> right;
        uint32_t dropped = mantissa & ((1u << right) - 1u);
        uint32_t half = 1u << (right - 1);
        if (dropped > half || (dropped == half && (dt_lo & 1u) != 0)) dt_lo += 1;
    }
    if (dt_hi == 0 && dt_lo == 0) { row[3] = BAD_DT; return; }
    int dt_exceeds = dt_hi > rem_hi || (dt_hi == rem_hi && dt_lo > rem_lo);
    uint32_t diff_hi, diff_lo;
    if (dt_exceeds) {
        diff_hi = dt_hi - rem_hi - (dt_lo < rem_lo ? 1u : 0u);
        diff_lo = dt_lo - rem_lo;
    } else {
        diff_hi = rem_hi - dt_hi - (rem_lo < dt_lo ? 1u : 0u);
        diff_lo = rem_lo - dt_lo;
    }
    uint32_t end_hi = now_hi, end_lo = now_lo;
    if (diff_hi == 0 && diff_lo < SNAP_TICKS) { end_hi = target_hi; end_lo = target_lo; }
    else if (dt_exceeds) { row[3] = OVERSHOOT; return; }
    else {
        end_lo = now_lo + dt_lo;
        end_hi = now_hi + dt_hi + (end_lo < now_lo ? 1u : 0u);
    }
    uint32_t origin_hi = c->origin[0], origin_lo = c->origin[1];
    uint32_t local_hi = now_hi - origin_hi - (now_lo < origin_lo ? 1u : 0u);
    uint32_t local_lo = now_lo - origin_lo;
    uint32_t end_local_hi = end_hi - origin_hi - (end_lo < origin_lo ? 1u : 0u);
    uint32_t end_local_lo = end_lo - origin_lo;
    c->local = (float)local_hi * (1.0f / 256.0f) + (float)local_lo * 0x1p-40f;
    c->end_local = (float)end_local_hi * (1.0f / 256.0f) + (float)end_local_lo * 0x1p-40f;
    c->dt = chosen;
    c->step_end[0] = end_hi; c->step_end[1] = end_lo;
    c->active = 1;
}

static void prepare_step(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
    clock_choose(c, (float)c->ndt, c->slot);
    if (!c->active) return;
    c->limited_cells = 0; c->limited_faces = 0; c->minimum_scale = R(1.0);
    for (int bi = 0; bi < m->b_num; ++bi) {
        c->values[bi] = c->coefficients[2 * bi] + c->coefficients[2 * bi + 1] * (c->local + c->dt / R(2.0));
        c->level_values[bi] = c->coefficients[2 * bi] + c->coefficients[2 * bi + 1] * c->end_local;
    }
    if (c->ndt < c->limit_value[0]) {
        int si = c->cfl_arg;
        int el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        real h = c->flow_depth[si];
        c->limit_value[0] = c->ndt;
        c->limit_value[1] = m->depth[el]; c->limit_value[2] = m->depth[eh];
        c->limit_value[3] = h;
        c->limit_value[4] = m->q[si] / maxf(h, R(1e-30));
        c->limit_ids[0] = si; c->limit_ids[1] = el; c->limit_ids[2] = eh;
    }
}

static void finish_step(ora_ctx *c)
{
    uint32_t *row = c->trace + (size_t)c->slot * ORA_TRACE_COLS;
    if (c->active) {
        row[6] = c->limited_cells;
        row[7] = c->limited_faces;
        row[8] = fbits((float)c->minimum_scale);
        row[9] = c->wet;
        c->now[0] = c->step_end[0]; c->now[1] = c->step_end[1];
        row[0] = fbits(c->dt);
        row[1] = c->step_end[0]; row[2] = c->step_end[1];
        row[3] = COMPLETED;
    }
    c->slot += 1;
}

/* ---- pressure reconstruction (pressure.py:65-129) ------------------------ */

static void face_difference(const ora_ctx *c, int cell, int direction, int axis,
                            real *value_out, real *distance_out, int *usable_out)
{
    const ora_mesh *m = &c->m;
    real value = R(0.0), distance = R(0.0), total = R(0.0);
    int usable = 1;
    real eta = m->bed[cell] + m->depth[cell];
    int start = m->face_ptr[4 * cell + direction];
    for (int j = 0; j < m->face_count[4 * cell + direction]; ++j) {
        int side = m->isl_data[start + j];
        int other = m->topology[3 * side + 1] + m->topology[3 * side + 2] - cell;
        if (other == 0 || m->depth[other] <= m->min_h) {
            usable = 0;
        } else {
            real weight = m->length[side];
            value += weight * ((m->bed[other] + m->depth[other]) - eta);
            real delta = axis == 1 ? m->y[other] - m->y[cell] : m->x[other] - m->x[cell];
            distance += weight * delta;
            total += weight;
        }
    }
    if (total > R(0.0)) { value /= total; distance /= total; }
    else usable = 0;
    *value_out = value; *distance_out = distance; *usable_out = usable;
}

static real gradient(const ora_ctx *c, int cell, int axis)
{
    int minus = axis == 1 ? 2 : 0, plus = axis == 1 ? 3 : 1;
    real dm, xm, dp, xp; int okm, okp;
    face_difference(c, cell, minus, axis, &dm, &xm, &okm);
    face_difference(c, cell, plus, axis, &dp, &xp, &okp);
    real result = R(0.0);
    if (okm && okp) result = (dp - dm) / (xp - xm);
    else if (okm) result = dm / xm;
    else if (okp) result = dp / xp;
    return result;
}

void ora_update_pressure(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
#pragma omp parallel for schedule(static)
    for (int slot = 0; slot < m->hang_cells; ++slot) {
        int cell = m->hcells[slot];
        for (int axis = 0; axis < 2; ++axis) {
            if (m->axes[2 * slot + axis] == 1) {
                real value = R(0.0);
                if (m->depth[cell] > m->min_h) value = gradient(c, cell, axis);
                c->gradients[2 * slot + axis] = value;
            }
        }
    }
}

real ora_pressure_difference(const ora_ctx *c, int side, int lower, int higher, real raw)
{
    const ora_mesh *m = &c->m;
    real result = raw;
    int index = m->edge_index[side];
    if (index >= 0) {
        if (m->depth[lower] > m->min_h && m->depth[higher] > m->min_h) {
            int axis = m->topology[3 * side] == 2 ? 1 : 0;
            if (m->offsets[2 * index] != R(0.0))
                result -= c->gradients[2 * m->slots[2 * index] + axis] * m->offsets[2 * index];
            if (m->offsets[2 * index + 1] != R(0.0))
                result += c->gradients[2 * m->slots[2 * index + 1] + axis] * m->offsets[2 * index + 1];
        }
    }
    return result;
}

/* ---- tick (solver_compact.py:422-613) ------------------------------------ */

static real face_discharge(const real *qn, const real *lengths, const int32_t *ids, int start, int count)
{
    real result = R(0.0);
    if (count == 1) {
        result = qn[ids[start]];
    } else if (count > 1) {
        real total = R(0.0), width = R(0.0);
        for (int o = 0; o < count; ++o) {
            int side = ids[start + o];
            total += qn[side] * lengths[side];
            width += lengths[side];
        }
        result = total / width;
    }
    return result;
}

static real boundary_neighbor_sum(real q, real left, real right, real lext, real rext)
{
    real result = left + right;
    if (lext > R(0.0) || rext > R(0.0)) {
        if (lext == R(1.0) || rext == R(1.0)) {
            result = R(2.0) * q;
        } else {
            real product = lext * rext;
            result = ((R(1.0) - rext) * left + (R(1.0) - lext) * right
                      + R(2.0) * q * (lext + rext - R(2.0) * product)) / (R(1.0) - product);
        }
    }
    return result;
}

static void tick(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
    if (!c->active) return;
    const real dt = c->dt;
    const int raining = c->raining;
    const int T = c->terms;
    const int theta_one = m->sita == R(1.0);
    const real g = m->g;
    const real neg_g = -g;
    const real sita = m->sita;
    /* (1.0 - sita) / 2.0 folds in F64 (Python constants), then rounds to F32. */
    const real half_rest = (real)((1.0 - (double)m->sita) / 2.0);
    const real seven_thirds = (real)(7.0 / 3.0);

    if (!theta_one) {
#pragma omp parallel for schedule(static)
        for (int ei = 0; ei < m->e_num; ++ei)
            for (int d = 0; d < 4; ++d)
                c->face_qn[4 * ei + d] = face_discharge(m->q, m->length, m->isl_data,
                                                        m->face_ptr[4 * ei + d], m->face_count[4 * ei + d]);
    }

    /* side momentum (solver_compact.py:439-486) */
#pragma omp parallel for schedule(static)
    for (int si = 1; si < m->s_num; ++si) {
        real bf = m->sbf[si] == 1 ? R(0.0) : R(1.0);
        int so = m->topology[3 * si], el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        real hl = m->bed[el] + m->depth[el], hr = m->bed[eh] + m->depth[eh];
        real dx = c->sdc[si];
        real xq = m->q[si];
        real xwh = maxf(hl, hr) - maxf(maxf(m->bed[el], m->bed[eh]), c->dh[si]);
        real difference = hr - hl;
        if (m->hang_cells > 0) difference = ora_pressure_difference(c, si, el, eh, difference);
        real xdq = (neg_g * difference / dx) * maxf(xwh, R(0.0)) * dt;
        real n = m->side_n[si];
        real xf = R(1.0) + g * dt * (n * n) * RABS(xq / RPOW(maxf(xwh, R(0.00001)), seven_thirds));
        int dl = so == 2 ? 0 : 2, dr = so == 2 ? 1 : 3;
        real nb = c->face_qn[4 * el + dl] + c->face_qn[4 * eh + dr];
        if (!theta_one)
            nb = boundary_neighbor_sum(xq, c->face_qn[4 * el + dl], c->face_qn[4 * eh + dr],
                                       m->open_face[4 * el + dl], m->open_face[4 * eh + dr]);
        real new_q = (sita * xq + half_rest * nb + xdq) / xf;
        new_q = xwh < m->min_h ? R(0.0) : new_q;
        new_q *= bf;
        m->q[si] = new_q;
    }

    /* donor factor (solver_compact.py:491-514) */
    uint32_t limited_cells = 0;
    real minimum_scale = c->minimum_scale;
#pragma omp parallel for schedule(static) reduction(+ : limited_cells) reduction(min : minimum_scale)
    for (int ei = 1; ei < m->e_num; ++ei) {
        int bi = m->boundary_id[ei];
        real discharge = R(0.0);
        if (bi >= 0 && m->kind[bi] == 1) discharge = c->values[bi] * m->weight[ei];
        real rainq = R(0.0);
        if (raining) rainq = c->rain_rates[m->rain_index[ei]];
        real pipe = m->pipe_q ? m->pipe_q[ei] : R(0.0);
        real positive = (maxf(pipe, R(0.0)) + maxf(discharge, R(0.0))) * dt;
        real available = m->depth[ei] * m->area[ei] + positive + rainq * dt * m->area[ei];
        real outgoing = (maxf(-pipe, R(0.0)) + maxf(-discharge, R(0.0))) * dt;
        for (int d = 0; d < 4; ++d) {
            int p = m->face_ptr[4 * ei + d];
            for (int j = 0; j < m->face_count[4 * ei + d]; ++j) {
                int side = m->isl_data[p + j];
                real signed_q = m->q[side] * m->length[side];
                if (d == 0 || d == 2) signed_q = -signed_q;
                outgoing += maxf(signed_q, R(0.0)) * dt;
            }
        }
        c->donor_scale[ei] = R(1.0);
        if (outgoing > available && !(bi >= 0 && m->kind[bi] == 0)) {
            real sc = available / outgoing;
            c->donor_scale[ei] = sc;
            limited_cells += 1;
            minimum_scale = minf(minimum_scale, sc);
        }
    }
    c->limited_cells += limited_cells;
    c->minimum_scale = minimum_scale;

    /* side scaling (solver_compact.py:516-522) */
    uint32_t limited_faces = 0;
#pragma omp parallel for schedule(static) reduction(+ : limited_faces)
    for (int si = 1; si < m->s_num; ++si) {
        int el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        int donor = m->q[si] >= R(0.0) ? el : eh;
        if (m->q[si] != R(0.0) && c->donor_scale[donor] < R(1.0)) limited_faces += 1;
        m->q[si] *= c->donor_scale[donor];
    }
    c->limited_faces += limited_faces;
    /* controller.record_flux on the post-limiter volumes (solver_compact.py:523-524) */
    if (c->gate_on) gate_record_fluxes(c);

    /* cell fluxes, sources and depth update (solver_compact.py:525-610);
     * processed per 256-cell budget block. */
    const int B = m->b_num;
    uint32_t wet = 0;
#pragma omp parallel for schedule(static) reduction(+ : wet)
    for (int blk = 0; blk < c->blocks; ++blk) {
        real *diag = (real *)calloc((size_t)BLOCK * T, sizeof(real));
        real gvals[6 * BLOCK];
        int goff[BLOCK];
        for (int i = 0; i < BLOCK; ++i) goff[i] = -1;
        int e0 = blk * BLOCK;
        for (int i = 0; i < BLOCK; ++i) {
            int ei = e0 + i;
            if (ei < 1 || ei >= m->e_num) continue;
            real *dg = diag + (size_t)i * T;
            int bi = m->boundary_id[ei];
            real pq = m->pipe_q ? m->pipe_q[ei] : R(0.0);
            real pipe = maxf(pq, R(0.0)) + minf(pq, R(0.0)) * c->donor_scale[ei];
            real discharge = R(0.0);
            if (bi >= 0 && m->kind[bi] == 1) {
                real requested = c->values[bi] * m->weight[ei];
                discharge = maxf(requested, R(0.0)) + minf(requested, R(0.0)) * c->donor_scale[ei];
                if (discharge * dt != R(0.0)) dg[4 + 5 * B + bi] += discharge * dt;
            }
            c->ssq[ei] = pipe + discharge;
            real rainq = R(0.0);
            if (raining) rainq = c->rain_rates[m->rain_index[ei]];
            if (rainq > R(0.0)) {
                m->rain_time[ei] += dt;
                m->infiltration[ei] = m->fc[ei] + (m->f0[ei] - m->fc[ei])
                    * REXP(-m->k[ei] * m->rain_time[ei] / R(3600.0));
            }
            real fl[4];
            for (int d = 0; d < 4; ++d) {
                real face_flux = R(0.0);
                int p = m->face_ptr[4 * ei + d];
                for (int j = 0; j < m->face_count[4 * ei + d]; ++j) {
                    int si = m->isl_data[p + j];
                    face_flux += m->q[si] * m->length[si];
                }
                fl[d] = face_flux;
            }
            real ql = fl[0], qr = fl[1], qb = fl[2], qt = fl[3];
            real tq = ql - qr + qb - qt + c->ssq[ei];
            c->eq[4 * ei + 0] = ql; c->eq[4 * ei + 1] = qr; c->eq[4 * ei + 2] = qb; c->eq[4 * ei + 3] = qt;
            real ea = m->area[ei];
            real rain_depth = rainq * dt;
            c->increment[ei] = tq * dt / ea + rain_depth;
            c->rain_depth[ei] = rain_depth;

            /* depth update (solver_compact.py:567-610) */
            real previous = m->depth[ei];
            real raw_depth = previous + c->increment[ei];
            real removed = minf(m->infiltration[ei] * dt, maxf(raw_depth, R(0.0)));
            raw_depth -= removed;
            real floor_v = maxf(-raw_depth, R(0.0));
            dg[0] += removed * ea;
            dg[3] += pipe * dt;
            if (bi >= 0 && m->kind[bi] == 0) {
                dg[2] += floor_v * ea;
                real target = maxf(c->level_values[bi] - m->bed[ei], R(0.0));
                int off = 4 + 5 * bi;
                dg[off] += (target - previous) * ea;
                dg[off + 1] += -(ql - qr + qb - qt) * dt;
                dg[off + 2] += -pipe * dt;
                dg[off + 3] += -rain_depth * ea;
                dg[off + 4] += removed * ea;
                m->depth[ei] = target;
            } else {
                dg[1] += floor_v * ea;
                m->depth[ei] = maxf(raw_depth, R(0.0));
            }
            /* controller.record_cell + measure_inventory + collect's rounding
             * term (solver_compact.py:595-604; gate.py:151-193) */
            if (c->gate_on && (goff[i] = gate_source_offset(c, ei)) >= 0) {
                real applied_floor = floor_v, level_exchange = R(0.0);
                if (bi >= 0 && m->kind[bi] == 0) {
                    applied_floor = R(0.0);
                    level_exchange = (m->depth[ei] - previous) * ea - (ql - qr + qb - qt) * dt - pipe * dt
                                     - rain_depth * ea + removed * ea;
                }
                real *gv = gvals + 6 * i;
                gv[0] = rain_depth * ea;
                gv[1] = removed * ea;
                gv[2] = applied_floor * ea;
                gv[3] = pipe * dt;
                gv[4] = (c->ssq[ei] - pipe) * dt + level_exchange;
                real rounding = (m->depth[ei] - previous) - c->increment[ei] + removed - applied_floor;
                gv[5] = rounding * ea - level_exchange;
            }
            real u, v;
            velocity(c, ei, &u, &v);
            m->u[ei] = u; m->v[ei] = v;
            m->max_speed[ei] = maxf(m->max_speed[ei], RSQRT(u * u + v * v));
            if (m->depth[ei] > m->max_depth[ei]) {
                m->max_depth[ei] = m->depth[ei];
                m->peak_hi[ei] = c->step_end[0]; m->peak_lo[ei] = c->step_end[1];
            }
            if (m->depth[ei] >= m->min_h) wet += 1;
        }
        /* one writer per (block, term): fixed pairwise tree */
        double v[BLOCK];
        for (int t = 0; t < T; ++t) {
            int any = 0;
            for (int i = 0; i < BLOCK; ++i) {
                real val = diag[(size_t)i * T + t];
                v[i] = (double)val;
                any |= val != R(0.0);
            }
            if (any) acc_add(c, (size_t)blk * T + t, block_tree(v));
        }
        /* gate source terms: the pond group, then gate by gate */
        for (int grp = -1; c->gate_on && grp < c->gate.count; ++grp) {
            int off = grp < 0 ? 4 * c->gate.count + 2 : 4 * c->gate.count + 8 + 6 * grp;
            int member = 0;
            for (int i = 0; i < BLOCK; ++i) member |= goff[i] == off;
            if (!member) continue;
            for (int k = 0; k < 6; ++k) {
                int any = 0;
                for (int i = 0; i < BLOCK; ++i) {
                    real val = goff[i] == off ? gvals[6 * i + k] : R(0.0);
                    v[i] = (double)val;
                    any |= val != R(0.0);
                }
                if (any) gate_acc_add(c, blk, off + k, block_tree(v));
            }
        }
        free(diag);
    }
    c->wet = wet;
}

void ora_run_batch(ora_ctx *c, const uint32_t target[2], const uint32_t origin[2], uint32_t *trace)
{
    c->next[0] = target[0]; c->next[1] = target[1];
    c->origin[0] = origin[0]; c->origin[1] = origin[1];
    memset(c->trace, 0, sizeof(uint32_t) * (size_t)c->m.batch_size * ORA_TRACE_COLS);
    c->slot = 0;
    for (int s = 0; s < c->m.batch_size; ++s) {
        prepare_step(c);
        if (c->gate_on) ora_gate_check(c);
        if (c->active && c->m.hang_cells > 0) ora_update_pressure(c);
        tick(c);
        if (c->gate_on) gate_move(c, c->step_end[0], c->step_end[1]);  /* finish_gate_bed */
        ora_compute_cfl(c);
        finish_step(c);
    }
    memcpy(trace, c->trace, sizeof(uint32_t) * (size_t)c->m.batch_size * ORA_TRACE_COLS);
}
