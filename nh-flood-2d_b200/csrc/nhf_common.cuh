// Shared device-side definitions of the nhflood step: the control block, the
// kernel parameter block, the device clock (clock.py:94-181) and the small
// reductions used by both step forms (multi-pass and tiled).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/nhflood.h"

namespace nhf {

// The physics type (nhf_real: float, or double in the FP64 build) and its
// constants: RC(0.01) is 0.01f in the F32 build.
typedef nhf_real real;
#define RC(x) (static_cast<nhf::real>(x))
#ifdef NHF_REAL_DOUBLE
typedef unsigned long long scale_bits_t;  // bits of a nonnegative double: same order as the values
__device__ __forceinline__ scale_bits_t real_bits(double v) { return (scale_bits_t)__double_as_longlong(v); }
__device__ __forceinline__ double bits_real(scale_bits_t b) { return __longlong_as_double((long long)b); }
#else
typedef uint32_t scale_bits_t;  // bits of a nonnegative float: same order as the values
__device__ __forceinline__ scale_bits_t real_bits(float v) { return __float_as_uint(v); }
__device__ __forceinline__ float bits_real(scale_bits_t b) { return __uint_as_float(b); }
#endif

constexpr int kBlock = 256;                 // budget block = reference ei // 256
constexpr real kDh = RC(-999.0);            // dh_t without gates (solver_compact.py:405)
constexpr uint32_t kSnapTicks = 1099512u;   // ceil(1e-6 * 2**40) (clock.py:11)
constexpr unsigned long long kCflEmpty = 0xFFFFFFFFFFFFFFFFULL;

// Device control block: the reference's scalar fields (clock words, dt,
// limiter counters, CFL result, limiting-edge snapshot) and the batch trace.
struct Ctl {
    uint32_t now[2], next[2], origin[2], step_end[2];
    float dt, local, end_local;  // the clock's F32 values
    real ndt;
    int32_t active, slot, raining, cfl_arg;
    uint32_t limited_cells, limited_faces;
    scale_bits_t min_scale_bits;
    uint32_t wet;
    unsigned long long cfl_packed;
    uint32_t done_blocks;
    int32_t parity;  // 1: the current depth/q/rain_time live in the second buffers
    real limit_value[5];
    int32_t limit_ids[3];
    uint32_t trace[NHF_MAX_BATCH * NHF_TRACE_COLS];
    unsigned long long cfl_min_bits;  // FP64 build: the CFL minimum's bits, then
    int32_t cfl_arg_min;              // the lowest side id that attains it
};

// Tile plan of the fused step (built on the host by nhf_tiled.cu).
struct TilePlan {
    int32_t n_tiles, tile, max_ext, max_sides, cells_per_thread;
    int32_t split;  // 1: two halo rings and a separate CFL pass; 0: three rings, CFL in the step
    // per tile: n_ext, n_r0, n_r01, n_don, n_sides, n_owned, n_qf, r0_first_offset,
    // n_faces, cbase, sbase, then the pattern's ext, side, face_desc and face_idx offsets, 0
    const int4 *tile_head;     // [n_tiles][4]
    const int32_t *ext_rel;    // relative cell ids by local slot (slot 0 = exterior sentinel)
    const int32_t *side_rel;   // relative side ids by local side
    const uint32_t *side_lohi; // local slots: lower | higher << 16
    const uint32_t *face_desc; // per slot 0..n_r012: start | counts (4 x 4 bits) << 16
    const uint16_t *face_idx;  // local side indices in the reference's CSR order
};

// Lattice form (nhf_lattice.cu) of a uniform mesh: the cells renumbered into
// a padded 2-D lattice (a 2-cell border and tile padding of holes), the
// state kept in lattice order during a batch. Lattice index of real cell
// (i, j): (j + 2) * lx + (i + 2); the west face of a lattice cell is its
// "v" side, the south face its "h" side.
struct LatticePlan {
    int32_t nx, ny, lx, ly, strips, chunks, rows, block_warps, min_blocks, rain_cells, horton;
    int32_t buffer_stride;          // elements from the first to the second buffer of h, qv and qh
    real sdc_v, sdc_h, len_v, len_h, area, width, height;
    const int32_t *cell;            // [lx*ly] global cell id (0: hole, border, padding)
    const int32_t *side_v, *side_h; // [lx*ly] global id of the west / south side (0: none)
    const uint8_t *live;            // [lx*ly] 1 for a real cell
    const int32_t *glat;            // [e_num] lattice index of each cell
    const int32_t *gside;           // [s_num] lattice index << 1 | 1 for a south side
    real *h[2], *qv[2], *qh[2];     // double-buffered depth and side discharges
    real *z, *nv, *nh;              // bed (refreshed each batch), Manning n of the sides
    int16_t *bi;                    // boundary id, -1 for none
    int32_t *rain;                  // rain pixel (rain_cells only)
    real *rain_time, *infil, *max_depth, *max_speed;
    uint32_t *peak_hi, *peak_lo;
    real *f0, *fc, *k;              // Horton (horton only)
    float *terms;                   // [terms][e_num] budget terms of a step by global id, else zero
    uint32_t *touched;              // [blocks] terms some cell of a 256-cell budget block holds
    uint32_t *part;                 // [4][strips*chunks] per-warp limited cells, limited faces, wet cells, min scale bits
    unsigned long long *part_cfl;   // [strips*chunks] per-warp CFL key
    float4 *edge_first;             // [strips][chunks*rows] first column: new depth, bed, west discharge, live
    float2 *edge_last;              // [strips][chunks*rows] last column: new depth (-1: hole), bed
};

// Gate controller (core/gate.py:35-206): the caller's tables and controller
// words plus the library's budget partials [blocks][terms].
struct GateDev {
    int32_t count, n_targets, n_flux, terms, blocks;
    const int32_t *cell_gate, *pond, *targets, *controls, *flux_sides;
    const real *closed;
    uint32_t formal_hi, formal_lo;
    float trigger_level, opening_seconds, open_elevation;
    int32_t *commanded, *flow_seen, *opened;
    uint32_t *command, *first_flow, *opened_at;
    double *acc_sum, *acc_comp;
};

struct Dev {
    nhf_mesh m;
    real g, neg_g, afa, sita, half_rest, seven_thirds, min_h;
    float min_dt;
    int32_t terms, blocks, batch_size, theta_one;
    Ctl *ctl;
    const real *coef;
    real *values, *level_values, *rain_rates, *sdc, *donor_scale, *face_qn, *eq, *gradients;
    double *acc_sum, *acc_comp;
    // second buffers of the double-buffered state (tiled form)
    real *depth_b, *q_b, *rain_time_b;
    float2 *sdn;  // per side {centre distance, Manning n} (tiled form; filled by initialize)
    TilePlan plan;
    LatticePlan lat;
};

__device__ __forceinline__ float maxf(float a, float b) { return a > b ? a : b; }
__device__ __forceinline__ float minf(float a, float b) { return b < a ? b : a; }
__device__ __forceinline__ real rmax(real a, real b) { return a > b ? a : b; }
__device__ __forceinline__ real rmin(real a, real b) { return b < a ? b : a; }

__device__ __forceinline__ const real *cur_depth(const Dev &d, int parity) { return parity ? d.depth_b : d.m.depth; }
__device__ __forceinline__ const real *cur_q(const Dev &d, int parity) { return parity ? d.q_b : d.m.q; }

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v)
{
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_down_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// Canonical pairwise tree over the 256 cells of one budget block:
// slot i += slot i + stride for stride 128 .. 1. Returns the sum in thread 0.
// Must be called by all 256 threads of the block.
__device__ __forceinline__ double block_tree(double v, double *sh)
{
    const int t = threadIdx.x;
    sh[t] = v;
    __syncthreads();
    for (int stride = 128; stride >= 32; stride >>= 1) {
        if (t < stride) sh[t] += sh[t + stride];
        __syncthreads();
    }
    double r = 0.0;
    if (t < 32) {
        r = sh[t];
        for (int stride = 16; stride >= 1; stride >>= 1) r += __shfl_down_sync(0xffffffffu, r, stride);
    }
    __syncthreads();
    return r;
}

// TwoSum: exact error of sum + p accumulated in the compensation word.
__device__ __forceinline__ void acc_add(double *sum, double *comp, double p)
{
    double s0 = *sum;
    double s = s0 + p;
    double bp = s - s0;
    double err = (s0 - (s - bp)) + (p - bp);
    *comp += err;
    *sum = s;
}

// Face depth and CFL value of an interior side (solver_compact.py:628-631):
// h = max(max(eta_l, eta_h) - max(z_l, z_h, dh), 0.01), cfl = afa L / (sqrt(g h) + |q| / h).
__device__ __forceinline__ real cfl_face_depth(real zl, real depth_l, real zh, real depth_h)
{
    real head = rmax(zl + depth_l, zh + depth_h);
    return rmax(head - rmax(rmax(zl, zh), kDh), RC(0.01));
}

__device__ __forceinline__ real cfl_value(real afa, real g, real length, real q, real h)
{
    return afa * length / (sqrt(g * h) + fabs(q) / h);
}

// flow_depth_t[si] (solver_compact.py:628-630) from a depth array; side 0
// keeps the field's initial zero.
__device__ __forceinline__ real flow_depth_of(const nhf_mesh &m, const real *depth, int si)
{
    if (si == 0) return RC(0);
    int el = m.topology[3 * si + 1], eh = m.topology[3 * si + 2];
    real zl = m.bed[el], zh = m.bed[eh];
    real head = rmax(zl + __ldcg(depth + el), zh + __ldcg(depth + eh));
    return rmax(head - rmax(rmax(zl, zh), kDh), RC(0.01));
}

// StepClock.choose (clock.py:94-167)
__device__ __forceinline__ void clock_choose(const Dev &d, Ctl *c, float candidate, int slot)
{
    uint32_t *row = c->trace + slot * NHF_TRACE_COLS;
    c->active = 0; c->dt = 0.0f; c->local = 0.0f; c->end_local = 0.0f;
    uint32_t now_hi = c->now[0], now_lo = c->now[1];
    uint32_t target_hi = c->next[0], target_lo = c->next[1];
    if (!(now_hi < target_hi || (now_hi == target_hi && now_lo < target_lo))) return;
    if (!(candidate >= d.min_dt)) { row[3] = NHF_STEP_BAD_CFL; return; }
    uint32_t borrow = now_lo > target_lo ? 1u : 0u;
    uint32_t rem_hi = target_hi - now_hi - borrow;
    uint32_t rem_lo = target_lo - now_lo;
    float remaining = __uint2float_rn(rem_hi) * (1.0f / 256.0f) + __uint2float_rn(rem_lo) * 0x1p-40f;
    float chosen = minf(minf(candidate, 1.0f), remaining);
    row[4] = __float_as_uint(candidate);
    row[5] = chosen < minf(candidate, 1.0f) ? 1u : 0u;
    uint32_t bits = __float_as_uint(chosen);
    int exponent = (int)((bits >> 23) & 255u) - 127;
    uint32_t mantissa = (bits & 0x7fffffu) | 0x800000u;
    uint32_t dt_hi = 0, dt_lo = 0;
    if (!(chosen > 0.0f) || exponent < -40 || exponent > 0) { row[3] = NHF_STEP_BAD_DT; return; }
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
    if (dt_hi == 0 && dt_lo == 0) { row[3] = NHF_STEP_BAD_DT; return; }
    bool exceeds = dt_hi > rem_hi || (dt_hi == rem_hi && dt_lo > rem_lo);
    uint32_t diff_hi, diff_lo;
    if (exceeds) {
        diff_hi = dt_hi - rem_hi - (dt_lo < rem_lo ? 1u : 0u);
        diff_lo = dt_lo - rem_lo;
    } else {
        diff_hi = rem_hi - dt_hi - (rem_lo < dt_lo ? 1u : 0u);
        diff_lo = rem_lo - dt_lo;
    }
    uint32_t end_hi = now_hi, end_lo = now_lo;
    if (diff_hi == 0 && diff_lo < kSnapTicks) { end_hi = target_hi; end_lo = target_lo; }
    else if (exceeds) { row[3] = NHF_STEP_OVERSHOOT; return; }
    else {
        end_lo = now_lo + dt_lo;
        end_hi = now_hi + dt_hi + (end_lo < now_lo ? 1u : 0u);
    }
    uint32_t origin_hi = c->origin[0], origin_lo = c->origin[1];
    uint32_t local_hi = now_hi - origin_hi - (now_lo < origin_lo ? 1u : 0u);
    uint32_t local_lo = now_lo - origin_lo;
    uint32_t end_local_hi = end_hi - origin_hi - (end_lo < origin_lo ? 1u : 0u);
    uint32_t end_local_lo = end_lo - origin_lo;
    c->local = __uint2float_rn(local_hi) * (1.0f / 256.0f) + __uint2float_rn(local_lo) * 0x1p-40f;
    c->end_local = __uint2float_rn(end_local_hi) * (1.0f / 256.0f) + __uint2float_rn(end_local_lo) * 0x1p-40f;
    c->dt = chosen;
    c->step_end[0] = end_hi; c->step_end[1] = end_lo;
    c->active = 1;
}

// prepare_step (solver_compact.py:364-382) for trace slot c->slot; `depth` and
// `q` are the current state (read through L2: written by other blocks).
__device__ __forceinline__ void prepare_step(const Dev &d, Ctl *c, const real *depth, const real *q)
{
    const nhf_mesh &m = d.m;
    clock_choose(d, c, (float)c->ndt, c->slot);
    if (!c->active) return;
    c->limited_cells = 0; c->limited_faces = 0;
    c->min_scale_bits = real_bits(RC(1.0));
    c->wet = 0;
    for (int bi = 0; bi < m.b_num; ++bi) {
        d.values[bi] = d.coef[2 * bi] + d.coef[2 * bi + 1] * ((real)c->local + (real)c->dt / RC(2.0));
        d.level_values[bi] = d.coef[2 * bi] + d.coef[2 * bi + 1] * (real)c->end_local;
    }
    if (c->ndt < c->limit_value[0]) {
        int si = c->cfl_arg;
        int el = m.topology[3 * si + 1], eh = m.topology[3 * si + 2];
        real h = flow_depth_of(m, depth, si);
        c->limit_value[0] = c->ndt;
        c->limit_value[1] = __ldcg(depth + el); c->limit_value[2] = __ldcg(depth + eh);
        c->limit_value[3] = h;
        c->limit_value[4] = __ldcg(q + si) / rmax(h, RC(1e-30));
        c->limit_ids[0] = si; c->limit_ids[1] = el; c->limit_ids[2] = eh;
    }
}

// finish_step + StepClock.commit (solver_compact.py:384-391, clock.py:173-181)
__device__ __forceinline__ void finish_step(Ctl *c)
{
    uint32_t *row = c->trace + c->slot * NHF_TRACE_COLS;
    if (c->active) {
        row[6] = c->limited_cells;
        row[7] = c->limited_faces;
        row[8] = __float_as_uint((float)bits_real(c->min_scale_bits));
        row[9] = c->wet;
        c->now[0] = c->step_end[0]; c->now[1] = c->step_end[1];
        row[0] = __float_as_uint(c->dt);
        row[1] = c->step_end[0]; row[2] = c->step_end[1];
        row[3] = NHF_STEP_COMPLETED;
    }
    c->slot += 1;
}

// PressureReconstruction.difference (pressure.py:118-129)
__device__ __forceinline__ real pressure_difference(const Dev &d, const real *depth, int side, int lower,
                                                    int higher, real raw)
{
    const nhf_mesh &m = d.m;
    real result = raw;
    int index = m.edge_index[side];
    if (index >= 0 && depth[lower] > d.min_h && depth[higher] > d.min_h) {
        int axis = m.topology[3 * side] == 2 ? 1 : 0;
        real o0 = m.offsets[2 * index], o1 = m.offsets[2 * index + 1];
        if (o0 != RC(0)) result -= d.gradients[2 * m.slots[2 * index] + axis] * o0;
        if (o1 != RC(0)) result += d.gradients[2 * m.slots[2 * index + 1] + axis] * o1;
    }
    return result;
}

// boundary_neighbor_sum (solver_compact.py:135-149)
__device__ __forceinline__ real boundary_neighbor_sum(real q, real left, real right, real lext, real rext)
{
    real result = left + right;
    if (lext > RC(0) || rext > RC(0)) {
        if (lext == RC(1) || rext == RC(1)) {
            result = RC(2) * q;
        } else {
            real product = lext * rext;
            result = ((RC(1) - rext) * left + (RC(1) - lext) * right
                      + RC(2) * q * (lext + rext - RC(2) * product)) / (RC(1) - product);
        }
    }
    return result;
}

// since_command (gate.py:68-73): the command's clock age in F32 seconds.
__device__ __forceinline__ float since_command(const GateDev &g, int gate, uint32_t hi, uint32_t lo)
{
    uint32_t borrow = lo < g.command[2 * gate + 1] ? 1u : 0u;
    uint32_t high = hi - g.command[2 * gate] - borrow;
    uint32_t low = lo - g.command[2 * gate + 1];
    return __uint2float_rn(high) / 256.0f + __uint2float_rn(low) * 0x1p-40f;
}

// move (gate.py:75-86): the threads of one block set the working bed of
// every commanded gate cell to its opening fraction at (hi, lo).
__device__ __forceinline__ void gate_move_beds(const Dev &d, const GateDev &g, uint32_t hi, uint32_t lo)
{
    const nhf_mesh &m = d.m;
    for (int slot = threadIdx.x; slot < g.n_targets; slot += blockDim.x) {
        int cell = g.targets[slot];
        int gate = g.cell_gate[cell];
        if (g.commanded[gate] != 1) continue;
        float fraction = minf(since_command(g, gate, hi, lo) / g.opening_seconds, 1.0f);
        if (fraction >= 1.0f) {
            m.bed[cell] = g.open_elevation;
            if (atomicOr(&g.opened[gate], 1) == 0) {
                g.opened_at[2 * gate] = hi; g.opened_at[2 * gate + 1] = lo;
            }
        } else {
            real closed = g.closed[cell];
            m.bed[cell] = closed + ((real)g.open_elevation - closed) * (real)fraction;
        }
    }
}

// check (gate.py:88-99), the threads of one block over the gates: from
// formal time 0 on, an irreversible command once the control cell is wet
// and its level is strictly above the trigger.
__device__ __forceinline__ void gate_check(const Dev &d, const GateDev &g, uint32_t hi, uint32_t lo)
{
    const nhf_mesh &m = d.m;
    const real *depth = cur_depth(d, d.ctl->parity);
    const bool formal = hi > g.formal_hi || (hi == g.formal_hi && lo >= g.formal_lo);
    for (int gate = threadIdx.x; formal && gate < g.count; gate += blockDim.x) {
        int cell = g.controls[gate];
        if (g.commanded[gate] == 0 && depth[cell] >= d.min_h && m.bed[cell] + depth[cell] > g.trigger_level) {
            g.commanded[gate] = 1;
            g.command[2 * gate] = hi; g.command[2 * gate + 1] = lo;
        }
    }
}

// ---------------------------------------------------------------- host side

struct TiledBuild {
    TilePlan plan{};
    void *device_memory = nullptr;   // owned plan arrays (cudaFree on destroy)
    size_t shared_bytes = 0;
    int patterns = 0;
};

// Build the tile plan from the caller's device arrays (copied to the host
// once). Returns 0 on success; a nonzero value with `why` set when the mesh
// does not fit the tiled form (the caller then keeps the multi-pass form).
// tile_request: 0 picks the tile size by mesh size; 256, 512 or 1024 asks
// for that size only. cfl_mode: 0 separate CFL pass from two waves of tiles
// on, 1 CFL always in the step, 2 always a separate pass.
int tiled_build(const nhf_mesh &m, cudaStream_t s, TiledBuild *out, char *why, size_t why_len,
                int tile_request = 0, int cfl_mode = 0);
// Enqueue one fused step (plus the hanging/theta pre-passes and, for split
// plans, the CFL pass). With a gate controller (256-cell tiles, split plan)
// only the pre-passes and the gate-enabled step: the caller then enqueues
// the controller's passes and tiled_enqueue_cfl.
void tiled_enqueue_step(const Dev &d, const TiledBuild &b, cudaStream_t s, const GateDev *gate = nullptr);
// The separate CFL pass of a split plan (nothing otherwise); with a gate
// controller its last block also runs the next step's check_gates.
void tiled_enqueue_cfl(const Dev &d, const TiledBuild &b, cudaStream_t s, const GateDev *gate = nullptr);
// Enqueue the batch epilogue: bring the state back into the caller's
// buffers and refresh u, v.
void tiled_enqueue_batch_end(const Dev &d, cudaStream_t s);
// Copy the caller's rain_time into the second buffer (batch start).
void tiled_enqueue_batch_start(const Dev &d, cudaStream_t s);

// u, v of every cell from the caller's arrays (after a batch of the tiled or
// lattice form has brought its state back).
void tiled_enqueue_velocity(const Dev &d, cudaStream_t s);

struct LatticeBuild {
    LatticePlan plan{};
    void *device_memory = nullptr;  // owned lattice arrays (cudaFree on destroy)
};
// Plan the lattice form when the mesh is a uniform grid the form covers
// (theta = 1, no hanging edges, at most four boundaries, one side per face,
// uniform cell size, side length and centre distance); 0 on success, else
// nonzero with `why` set. `d` supplies the mesh and the sizes of the budget.
int lattice_build(const Dev &d, cudaStream_t s, LatticeBuild *out, char *why, size_t why_len);
void lattice_enqueue_batch_start(const Dev &d, cudaStream_t s);
// One step: the fused lattice step, then the pass that reduces its budget
// blocks, takes the CFL candidate, commits the step and prepares the next.
void lattice_enqueue_step(const Dev &d, cudaStream_t s);
void lattice_enqueue_batch_end(const Dev &d, cudaStream_t s);

// Ensemble form: several meshes (members) on the fused tiled step with one
// common tile size, advanced together. Work lists are (member, index) pairs:
// step items index tiles, the other lists index chunks of kEnsChunk cells,
// sides or hanging cells of the member.
constexpr int kEnsChunk = 1024;
struct EnsembleLaunch {
    const Dev *devs = nullptr;      // [members], device
    int members = 0, batch = 0, tile = 0, theta_one = 1;
    size_t smem = 0;
    int grid = 0;                   // blocks of the step kernel
    const int2 *step_items = nullptr; int n_step = 0;
    const int2 *hang_items = nullptr; int n_hang = 0;     // chunks of hanging cells
    const int2 *qn_items = nullptr; int n_qn = 0;         // chunks of cells (theta < 1)
    const int2 *cell_items = nullptr; int n_cell = 0;     // chunks of max(cells, sides)
    const uint32_t *words = nullptr;  // [members][4] next, origin (device)
    uint32_t *trace = nullptr;        // [members][batch][NHF_TRACE_COLS] (device)
};
// Resident blocks per SM of the ensemble step kernel for this tile size.
int ensemble_blocks_per_sm(int tile, int theta_one, size_t smem);
void ensemble_enqueue_begin(const EnsembleLaunch &e, cudaStream_t s);
void ensemble_enqueue_batch_start(const EnsembleLaunch &e, cudaStream_t s);
void ensemble_enqueue_step(const EnsembleLaunch &e, cudaStream_t s);
void ensemble_enqueue_batch_end(const EnsembleLaunch &e, cudaStream_t s);

}  // namespace nhf
