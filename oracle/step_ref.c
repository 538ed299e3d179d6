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

static inline float maxf(float a, float b) { return a > b ? a : b; }
static inline float minf(float a, float b) { return b < a ? b : a; }
static inline uint32_t fbits(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float bitsf(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

struct ora_ctx {
    ora_mesh m;
    int terms, blocks;
    /* clock (clock.py:60-68) */
    uint32_t now[2], next[2], origin[2], step_end[2];
    float dt, local, end_local;
    int active, slot;
    /* scalars */
    float ndt;
    int32_t cfl_arg;
    uint32_t limited_cells, limited_faces;
    float minimum_scale;
    uint32_t wet;
    float limit_value[5];
    int32_t limit_ids[3];
    int raining;
    /* per-boundary */
    float *coefficients, *values, *level_values;
    const float *rain_rates_ext;
    float *rain_rates;
    /* work */
    float *sdc, *dh, *eq, *increment, *rain_depth, *donor_scale, *cfl, *flow_depth, *face_qn, *ssq;
    float *gradients;
    float *diag;      /* [blocks*terms] per-step f32 values per cell collected per block */
    double *acc_sum, *acc_comp; /* [blocks*terms] */
    uint32_t *trace;  /* [batch][10] */
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
    c->coefficients = (float *)calloc((size_t)bb * 2, sizeof(float));
    c->values = (float *)calloc(bb, sizeof(float));
    c->level_values = (float *)calloc(bb, sizeof(float));
    c->rain_rates = (float *)calloc(mesh->n_rates > 0 ? mesh->n_rates : 1, sizeof(float));
    c->sdc = (float *)calloc(s, sizeof(float));
    c->dh = (float *)calloc(s, sizeof(float));
    c->eq = (float *)calloc((size_t)e * 4, sizeof(float));
    c->increment = (float *)calloc(e, sizeof(float));
    c->rain_depth = (float *)calloc(e, sizeof(float));
    c->donor_scale = (float *)calloc(e, sizeof(float));
    c->cfl = (float *)calloc(s, sizeof(float));
    c->flow_depth = (float *)calloc(s, sizeof(float));
    c->face_qn = (float *)calloc((size_t)e * 4, sizeof(float));
    c->ssq = (float *)calloc(e, sizeof(float));
    c->gradients = (float *)calloc((size_t)(mesh->hang_cells > 0 ? mesh->hang_cells : 1) * 2, sizeof(float));
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
    free(c);
}

void ora_set_clock(ora_ctx *c, const uint32_t now[2]) { c->now[0] = now[0]; c->now[1] = now[1]; }
void ora_get_clock(const ora_ctx *c, uint32_t now[2]) { now[0] = c->now[0]; now[1] = c->now[1]; }
void ora_set_active(ora_ctx *c, int active) { c->active = active; }
int ora_budget_terms(const ora_ctx *c) { return c->terms; }
float ora_ndt(const ora_ctx *c) { return c->ndt; }
int32_t ora_cfl_arg(const ora_ctx *c) { return c->cfl_arg; }

void ora_limits(const ora_ctx *c, float values[5], int32_t ids[3])
{
    memcpy(values, c->limit_value, sizeof(c->limit_value));
    memcpy(ids, c->limit_ids, sizeof(c->limit_ids));
}

void ora_reset_limits(ora_ctx *c) { c->limit_value[0] = INFINITY; }

void ora_read_eq(const ora_ctx *c, float *eq) { memcpy(eq, c->eq, sizeof(float) * 4 * (size_t)c->m.e_num); }
void ora_read_flow_depth(const ora_ctx *c, float *out) { memcpy(out, c->flow_depth, sizeof(float) * (size_t)c->m.s_num); }
void ora_read_gradients(const ora_ctx *c, float *out)
{
    if (c->m.hang_cells > 0) memcpy(out, c->gradients, sizeof(float) * 2 * (size_t)c->m.hang_cells);
}

void ora_set_forcing(ora_ctx *c, const float *coefficients, const float *rain_rates, int raining)
{
    int bb = c->m.b_num > 0 ? c->m.b_num : 1;
    if (coefficients) memcpy(c->coefficients, coefficients, sizeof(float) * 2 * (size_t)bb);
    if (rain_rates && c->m.n_rates > 0) memcpy(c->rain_rates, rain_rates, sizeof(float) * (size_t)c->m.n_rates);
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
static void collect(ora_ctx *c, const float *diag)
{
    int T = c->terms, e = c->m.e_num;
#pragma omp parallel for schedule(static)
    for (int blk = 0; blk < c->blocks; ++blk) {
        double v[BLOCK];
        for (int t = 0; t < T; ++t) {
            int any = 0;
            for (int i = 0; i < BLOCK; ++i) {
                int ei = blk * BLOCK + i;
                float val = ei < e ? diag[(size_t)ei * T + t] : 0.0f;
                v[i] = val != 0.0f ? (double)val : 0.0;
                any |= val != 0.0f;
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

/* ---- setup kernels -------------------------------------------------------- */

void ora_initialize(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
    for (int ei = 1; ei < m->e_num; ++ei) {
        m->depth[ei] = 0.0f;
        m->infiltration[ei] = m->f0[ei];
    }
    for (int si = 1; si < m->s_num; ++si) {
        c->dh[si] = -999.0f;
        int so = m->topology[3 * si], el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        if (so == 2) c->sdc[si] = maxf(fabsf(m->x[eh] - m->x[el]), 0.01f);
        else c->sdc[si] = maxf(fabsf(m->y[eh] - m->y[el]), 0.01f);
    }
}

void ora_apply_initial_levels(ora_ctx *c, const float *targets)
{
    const ora_mesh *m = &c->m;
    int T = c->terms;
    float *diag = (float *)calloc((size_t)m->e_num * T, sizeof(float));
    for (int ei = 1; ei < m->e_num; ++ei) {
        int bi = m->boundary_id[ei];
        if (bi >= 0 && m->kind[bi] == 0) {
            float previous = m->depth[ei];
            m->depth[ei] = targets[ei];
            diag[(size_t)ei * T + 4 + 5 * bi] = (m->depth[ei] - previous) * m->area[ei];
        }
    }
    collect(c, diag);
    free(diag);
}

static void velocity(const ora_ctx *c, int ei, float *u, float *v)
{
    const ora_mesh *m = &c->m;
    float h = maxf(m->depth[ei], 0.01f);
    *u = 0.0f; *v = 0.0f;
    if (m->depth[ei] >= m->min_h) {
        *u = (c->eq[4 * ei + 0] + c->eq[4 * ei + 1]) / m->height[ei] / h / 2.0f;
        *v = (c->eq[4 * ei + 2] + c->eq[4 * ei + 3]) / m->width[ei] / h / 2.0f;
    }
}

void ora_compute_cfl(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
    if (!c->active) return;
    float ndt = INFINITY;
#pragma omp parallel for schedule(static) reduction(min : ndt)
    for (int si = 1; si < m->s_num; ++si) {
        int el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        c->cfl[si] = INFINITY;
        if (el != 0 && eh != 0) {
            float head = maxf(m->bed[el] + m->depth[el], m->bed[eh] + m->depth[eh]);
            float h = maxf(head - maxf(maxf(m->bed[el], m->bed[eh]), c->dh[si]), 0.01f);
            c->flow_depth[si] = h;
            float val = m->afa * m->length[si] / (sqrtf(m->g * h) + fabsf(m->q[si]) / h);
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
            float total = 0.0f;
            int p = m->face_ptr[4 * ei + d];
            for (int j = 0; j < m->face_count[4 * ei + d]; ++j) {
                int si = m->isl_data[p + j];
                total += m->q[si] * m->length[si];
            }
            c->eq[4 * ei + d] = total;
        }
        float u, v;
        velocity(c, ei, &u, &v);
        m->u[ei] = u; m->v[ei] = v;
        m->max_speed[ei] = maxf(m->max_speed[ei], sqrtf(u * u + v * v));
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
        m->max_speed[ei] = sqrtf(m->u[ei] * m->u[ei] + m->v[ei] * m->v[ei]);
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
    clock_choose(c, c->ndt, c->slot);
    if (!c->active) return;
    c->limited_cells = 0; c->limited_faces = 0; c->minimum_scale = 1.0f;
    for (int bi = 0; bi < m->b_num; ++bi) {
        c->values[bi] = c->coefficients[2 * bi] + c->coefficients[2 * bi + 1] * (c->local + c->dt / 2.0f);
        c->level_values[bi] = c->coefficients[2 * bi] + c->coefficients[2 * bi + 1] * c->end_local;
    }
    if (c->ndt < c->limit_value[0]) {
        int si = c->cfl_arg;
        int el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        float h = c->flow_depth[si];
        c->limit_value[0] = c->ndt;
        c->limit_value[1] = m->depth[el]; c->limit_value[2] = m->depth[eh];
        c->limit_value[3] = h;
        c->limit_value[4] = m->q[si] / maxf(h, 1e-30f);
        c->limit_ids[0] = si; c->limit_ids[1] = el; c->limit_ids[2] = eh;
    }
}

static void finish_step(ora_ctx *c)
{
    uint32_t *row = c->trace + (size_t)c->slot * ORA_TRACE_COLS;
    if (c->active) {
        row[6] = c->limited_cells;
        row[7] = c->limited_faces;
        row[8] = fbits(c->minimum_scale);
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
                            float *value_out, float *distance_out, int *usable_out)
{
    const ora_mesh *m = &c->m;
    float value = 0.0f, distance = 0.0f, total = 0.0f;
    int usable = 1;
    float eta = m->bed[cell] + m->depth[cell];
    int start = m->face_ptr[4 * cell + direction];
    for (int j = 0; j < m->face_count[4 * cell + direction]; ++j) {
        int side = m->isl_data[start + j];
        int other = m->topology[3 * side + 1] + m->topology[3 * side + 2] - cell;
        if (other == 0 || m->depth[other] <= m->min_h) {
            usable = 0;
        } else {
            float weight = m->length[side];
            value += weight * ((m->bed[other] + m->depth[other]) - eta);
            float delta = axis == 1 ? m->y[other] - m->y[cell] : m->x[other] - m->x[cell];
            distance += weight * delta;
            total += weight;
        }
    }
    if (total > 0.0f) { value /= total; distance /= total; }
    else usable = 0;
    *value_out = value; *distance_out = distance; *usable_out = usable;
}

static float gradient(const ora_ctx *c, int cell, int axis)
{
    int minus = axis == 1 ? 2 : 0, plus = axis == 1 ? 3 : 1;
    float dm, xm, dp, xp; int okm, okp;
    face_difference(c, cell, minus, axis, &dm, &xm, &okm);
    face_difference(c, cell, plus, axis, &dp, &xp, &okp);
    float result = 0.0f;
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
                float value = 0.0f;
                if (m->depth[cell] > m->min_h) value = gradient(c, cell, axis);
                c->gradients[2 * slot + axis] = value;
            }
        }
    }
}

float ora_pressure_difference(const ora_ctx *c, int side, int lower, int higher, float raw)
{
    const ora_mesh *m = &c->m;
    float result = raw;
    int index = m->edge_index[side];
    if (index >= 0) {
        if (m->depth[lower] > m->min_h && m->depth[higher] > m->min_h) {
            int axis = m->topology[3 * side] == 2 ? 1 : 0;
            if (m->offsets[2 * index] != 0.0f)
                result -= c->gradients[2 * m->slots[2 * index] + axis] * m->offsets[2 * index];
            if (m->offsets[2 * index + 1] != 0.0f)
                result += c->gradients[2 * m->slots[2 * index + 1] + axis] * m->offsets[2 * index + 1];
        }
    }
    return result;
}

/* ---- tick (solver_compact.py:422-613) ------------------------------------ */

static float face_discharge(const float *qn, const float *lengths, const int32_t *ids, int start, int count)
{
    float result = 0.0f;
    if (count == 1) {
        result = qn[ids[start]];
    } else if (count > 1) {
        float total = 0.0f, width = 0.0f;
        for (int o = 0; o < count; ++o) {
            int side = ids[start + o];
            total += qn[side] * lengths[side];
            width += lengths[side];
        }
        result = total / width;
    }
    return result;
}

static float boundary_neighbor_sum(float q, float left, float right, float lext, float rext)
{
    float result = left + right;
    if (lext > 0.0f || rext > 0.0f) {
        if (lext == 1.0f || rext == 1.0f) {
            result = 2.0f * q;
        } else {
            float product = lext * rext;
            result = ((1.0f - rext) * left + (1.0f - lext) * right
                      + 2.0f * q * (lext + rext - 2.0f * product)) / (1.0f - product);
        }
    }
    return result;
}

static void tick(ora_ctx *c)
{
    const ora_mesh *m = &c->m;
    if (!c->active) return;
    const float dt = c->dt;
    const int raining = c->raining;
    const int T = c->terms;
    const int theta_one = m->sita == 1.0f;
    const float g = m->g;
    const float neg_g = -g;
    const float sita = m->sita;
    /* (1.0 - sita) / 2.0 folds in F64 (Python constants), then rounds to F32. */
    const float half_rest = (float)((1.0 - (double)m->sita) / 2.0);
    const float seven_thirds = (float)(7.0 / 3.0);

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
        float bf = m->sbf[si] == 1 ? 0.0f : 1.0f;
        int so = m->topology[3 * si], el = m->topology[3 * si + 1], eh = m->topology[3 * si + 2];
        float hl = m->bed[el] + m->depth[el], hr = m->bed[eh] + m->depth[eh];
        float dx = c->sdc[si];
        float xq = m->q[si];
        float xwh = maxf(hl, hr) - maxf(maxf(m->bed[el], m->bed[eh]), c->dh[si]);
        float difference = hr - hl;
        if (m->hang_cells > 0) difference = ora_pressure_difference(c, si, el, eh, difference);
        float xdq = (neg_g * difference / dx) * maxf(xwh, 0.0f) * dt;
        float n = m->side_n[si];
        float xf = 1.0f + g * dt * (n * n) * fabsf(xq / ora_powf(maxf(xwh, 0.00001f), seven_thirds));
        int dl = so == 2 ? 0 : 2, dr = so == 2 ? 1 : 3;
        float nb = c->face_qn[4 * el + dl] + c->face_qn[4 * eh + dr];
        if (!theta_one)
            nb = boundary_neighbor_sum(xq, c->face_qn[4 * el + dl], c->face_qn[4 * eh + dr],
                                       m->open_face[4 * el + dl], m->open_face[4 * eh + dr]);
        float new_q = (sita * xq + half_rest * nb + xdq) / xf;
        new_q = xwh < m->min_h ? 0.0f : new_q;
        new_q *= bf;
        m->q[si] = new_q;
    }

    /* donor factor (solver_compact.py:491-514) */
    uint32_t limited_cells = 0;
    float minimum_scale = c->minimum_scale;
#pragma omp parallel for schedule(static) reduction(+ : limited_cells) reduction(min : minimum_scale)
    for (int ei = 1; ei < m->e_num; ++ei) {
        int bi = m->boundary_id[ei];
        float discharge = 0.0f;
        if (bi >= 0 && m->kind[bi] == 1) discharge = c->values[bi] * m->weight[ei];
        float rainq = 0.0f;
        if (raining) rainq = c->rain_rates[m->rain_index[ei]];
        float pipe = m->pipe_q ? m->pipe_q[ei] : 0.0f;
        float positive = (maxf(pipe, 0.0f) + maxf(discharge, 0.0f)) * dt;
        float available = m->depth[ei] * m->area[ei] + positive + rainq * dt * m->area[ei];
        float outgoing = (maxf(-pipe, 0.0f) + maxf(-discharge, 0.0f)) * dt;
        for (int d = 0; d < 4; ++d) {
            int p = m->face_ptr[4 * ei + d];
            for (int j = 0; j < m->face_count[4 * ei + d]; ++j) {
                int side = m->isl_data[p + j];
                float signed_q = m->q[side] * m->length[side];
                if (d == 0 || d == 2) signed_q = -signed_q;
                outgoing += maxf(signed_q, 0.0f) * dt;
            }
        }
        c->donor_scale[ei] = 1.0f;
        if (outgoing > available && !(bi >= 0 && m->kind[bi] == 0)) {
            float sc = available / outgoing;
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
        int donor = m->q[si] >= 0.0f ? el : eh;
        if (m->q[si] != 0.0f && c->donor_scale[donor] < 1.0f) limited_faces += 1;
        m->q[si] *= c->donor_scale[donor];
    }
    c->limited_faces += limited_faces;

    /* cell fluxes, sources and depth update (solver_compact.py:525-610);
     * processed per 256-cell budget block. */
    const int B = m->b_num;
    uint32_t wet = 0;
#pragma omp parallel for schedule(static) reduction(+ : wet)
    for (int blk = 0; blk < c->blocks; ++blk) {
        float *diag = (float *)calloc((size_t)BLOCK * T, sizeof(float));
        int e0 = blk * BLOCK;
        for (int i = 0; i < BLOCK; ++i) {
            int ei = e0 + i;
            if (ei < 1 || ei >= m->e_num) continue;
            float *dg = diag + (size_t)i * T;
            int bi = m->boundary_id[ei];
            float pq = m->pipe_q ? m->pipe_q[ei] : 0.0f;
            float pipe = maxf(pq, 0.0f) + minf(pq, 0.0f) * c->donor_scale[ei];
            float discharge = 0.0f;
            if (bi >= 0 && m->kind[bi] == 1) {
                float requested = c->values[bi] * m->weight[ei];
                discharge = maxf(requested, 0.0f) + minf(requested, 0.0f) * c->donor_scale[ei];
                if (discharge * dt != 0.0f) dg[4 + 5 * B + bi] += discharge * dt;
            }
            c->ssq[ei] = pipe + discharge;
            float rainq = 0.0f;
            if (raining) rainq = c->rain_rates[m->rain_index[ei]];
            if (rainq > 0.0f) {
                m->rain_time[ei] += dt;
                m->infiltration[ei] = m->fc[ei] + (m->f0[ei] - m->fc[ei])
                    * ora_expf(-m->k[ei] * m->rain_time[ei] / 3600.0f);
            }
            float fl[4];
            for (int d = 0; d < 4; ++d) {
                float face_flux = 0.0f;
                int p = m->face_ptr[4 * ei + d];
                for (int j = 0; j < m->face_count[4 * ei + d]; ++j) {
                    int si = m->isl_data[p + j];
                    face_flux += m->q[si] * m->length[si];
                }
                fl[d] = face_flux;
            }
            float ql = fl[0], qr = fl[1], qb = fl[2], qt = fl[3];
            float tq = ql - qr + qb - qt + c->ssq[ei];
            c->eq[4 * ei + 0] = ql; c->eq[4 * ei + 1] = qr; c->eq[4 * ei + 2] = qb; c->eq[4 * ei + 3] = qt;
            float ea = m->area[ei];
            float rain_depth = rainq * dt;
            c->increment[ei] = tq * dt / ea + rain_depth;
            c->rain_depth[ei] = rain_depth;

            /* depth update (solver_compact.py:567-610) */
            float previous = m->depth[ei];
            float raw_depth = previous + c->increment[ei];
            float removed = minf(m->infiltration[ei] * dt, maxf(raw_depth, 0.0f));
            raw_depth -= removed;
            float floor_v = maxf(-raw_depth, 0.0f);
            dg[0] += removed * ea;
            dg[3] += pipe * dt;
            if (bi >= 0 && m->kind[bi] == 0) {
                dg[2] += floor_v * ea;
                float target = maxf(c->level_values[bi] - m->bed[ei], 0.0f);
                int off = 4 + 5 * bi;
                dg[off] += (target - previous) * ea;
                dg[off + 1] += -(ql - qr + qb - qt) * dt;
                dg[off + 2] += -pipe * dt;
                dg[off + 3] += -rain_depth * ea;
                dg[off + 4] += removed * ea;
                m->depth[ei] = target;
            } else {
                dg[1] += floor_v * ea;
                m->depth[ei] = maxf(raw_depth, 0.0f);
            }
            float u, v;
            velocity(c, ei, &u, &v);
            m->u[ei] = u; m->v[ei] = v;
            m->max_speed[ei] = maxf(m->max_speed[ei], sqrtf(u * u + v * v));
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
                float val = diag[(size_t)i * T + t];
                v[i] = (double)val;
                any |= val != 0.0f;
            }
            if (any) acc_add(c, (size_t)blk * T + t, block_tree(v));
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
        if (c->active && c->m.hang_cells > 0) ora_update_pressure(c);
        tick(c);
        ora_compute_cfl(c);
        finish_step(c);
    }
    memcpy(trace, c->trace, sizeof(uint32_t) * (size_t)c->m.batch_size * ORA_TRACE_COLS);
}
