// nhflood: local-inertial step of the nh-flood-2d compact solver on sm_100a.
//
// One physical step follows the reference's global passes
// (solver_compact.py:364-391 prepare/finish, 422-613 tick, 617-641 CFL):
//   k_prepare   clock choice, boundary values, limiting-edge snapshot
//   k_pressure  hanging-edge tangential gradients (multi-resolution meshes)
//   k_face_qn   length-weighted face discharge (theta < 1 only)
//   k_sides     theta-weighted momentum with semi-implicit Manning friction
//   k_donor     per-cell positivity donor factor
//   k_scale     q *= donor factor of the upwind cell
//   k_cells     fluxes, rain, Horton, depth update, level cells, extrema,
//               FP64 per-block budget partials, wet count
//   k_cfl       CFL packed (value, side) minimum; the last block commits the
//               clock and writes the trace row
// With a gate controller attached (core/gate.py) the step also runs
//   k_gate_move trigger check and bed motion at the step start (after
//               k_prepare) and bed motion to the step end (before k_cfl)
//   k_gate_flux post-limiter exchange volumes of the recorded sides (after
//               k_scale); k_cells adds the pond and gate-cell source terms
// A batch of up to 64 steps plus the begin/trace copies is captured once into
// a CUDA graph and replayed per batch. Every scalar the steps need (dt, clock
// words, boundary values) lives in a device control block, so the graph is
// static. Arithmetic follows the reference's F32 operation order; the build
// uses --fmad=false so that the CPU restatement reproduces every bit.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "../../include/nhflood.h"
#include "nhf_common.cuh"
#include "nhf_math.cuh"

using namespace nhf;

namespace {

// --------------------------------------------------------------- small kernels

// eq_t[ei][0..3] (one 16-byte store in the F32 build)
__device__ __forceinline__ void store4(real *p, real a, real b, real c, real e)
{
#ifdef NHF_REAL_DOUBLE
    p[0] = a; p[1] = b; p[2] = c; p[3] = e;
#else
    *reinterpret_cast<float4 *>(p) = make_float4(a, b, c, e);
#endif
}

__global__ void k_initialize(Dev d)
{
    const nhf_mesh &m = d.m;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 1 && i < m.e_num) {
        m.depth[i] = RC(0.0);
        m.infiltration[i] = m.f0[i];
    }
    if (i >= 1 && i < m.s_num) {
        int so = m.topology[3 * i], el = m.topology[3 * i + 1], eh = m.topology[3 * i + 2];
        d.sdc[i] = so == 2 ? rmax(fabs(m.x[eh] - m.x[el]), RC(0.01)) : rmax(fabs(m.y[eh] - m.y[el]), RC(0.01));
#ifndef NHF_REAL_DOUBLE
        if (d.sdn) d.sdn[i] = make_float2(d.sdc[i], m.side_n[i]);
#endif
    }
}

// clock.begin on the device (clock.py:75-92): the target and origin words are
// kernel arguments, updated in the instantiated graph before each replay. The
// tiled form also prepares slot 0 here (each fused step prepares the next).
__global__ void k_begin(Dev d, uint32_t next_hi, uint32_t next_lo, uint32_t origin_hi, uint32_t origin_lo,
                        int prepare_first)
{
    Ctl *c = d.ctl;
    int t = threadIdx.x;
    if (t == 0) {
        c->next[0] = next_hi; c->next[1] = next_lo;
        c->origin[0] = origin_hi; c->origin[1] = origin_lo;
        c->slot = 0;
    }
    for (int i = t; i < NHF_MAX_BATCH * NHF_TRACE_COLS; i += blockDim.x) c->trace[i] = 0u;
    __syncthreads();
    if (prepare_first && t == 0) prepare_step(d, c, d.m.depth, d.m.q);
}

// prepare_step (solver_compact.py:364-382), multi-pass form
__global__ void k_prepare(Dev d)
{
    if (threadIdx.x != 0) return;
    prepare_step(d, d.ctl, d.m.depth, d.m.q);
}

// ------------------------------------------------------ pressure (pressure.py)

__device__ void face_difference(const Dev &d, const real *depth, int cell, int direction, int axis,
                                real &value_out, real &distance_out, int &usable_out)
{
    const nhf_mesh &m = d.m;
    real value = RC(0.0), distance = RC(0.0), total = RC(0.0);
    int usable = 1;
    real eta = m.bed[cell] + depth[cell];
    int start = m.face_ptr[4 * cell + direction];
    int count = m.face_count[4 * cell + direction];
    for (int j = 0; j < count; ++j) {
        int side = m.isl_data[start + j];
        int other = m.topology[3 * side + 1] + m.topology[3 * side + 2] - cell;
        if (other == 0 || depth[other] <= d.min_h) {
            usable = 0;
        } else {
            real weight = m.length[side];
            value += weight * ((m.bed[other] + depth[other]) - eta);
            real delta = axis == 1 ? m.y[other] - m.y[cell] : m.x[other] - m.x[cell];
            distance += weight * delta;
            total += weight;
        }
    }
    if (total > RC(0.0)) { value /= total; distance /= total; }
    else usable = 0;
    value_out = value; distance_out = distance; usable_out = usable;
}

__global__ void k_pressure(Dev d)
{
    const nhf_mesh &m = d.m;
    if (!d.ctl->active) return;
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= m.hang_cells) return;
    int cell = m.hcells[slot];
    const real *depth = cur_depth(d, d.ctl->parity);
    for (int axis = 0; axis < 2; ++axis) {
        if (m.axes[2 * slot + axis] != 1) continue;
        real value = RC(0.0);
        if (depth[cell] > d.min_h) {
            int minus = axis == 1 ? 2 : 0, plus = axis == 1 ? 3 : 1;
            real dm, xm, dp, xp; int okm, okp;
            face_difference(d, depth, cell, minus, axis, dm, xm, okm);
            face_difference(d, depth, cell, plus, axis, dp, xp, okp);
            if (okm && okp) value = (dp - dm) / (xp - xm);
            else if (okm) value = dm / xm;
            else if (okp) value = dp / xp;
        }
        d.gradients[2 * slot + axis] = value;
    }
}

// ----------------------------------------------------------- theta < 1 faces

__global__ void k_face_qn(Dev d)
{
    const nhf_mesh &m = d.m;
    if (!d.ctl->active) return;
    int ei = blockIdx.x * blockDim.x + threadIdx.x;
    if (ei >= m.e_num) return;
    const real *q = cur_q(d, d.ctl->parity);
    for (int dd = 0; dd < 4; ++dd) {
        int start = m.face_ptr[4 * ei + dd], count = m.face_count[4 * ei + dd];
        real result = RC(0.0);
        if (count == 1) {
            result = q[m.isl_data[start]];
        } else if (count > 1) {
            real total = RC(0.0), width = RC(0.0);
            for (int o = 0; o < count; ++o) {
                int side = m.isl_data[start + o];
                total += q[side] * m.length[side];
                width += m.length[side];
            }
            result = total / width;
        }
        d.face_qn[4 * ei + dd] = result;
    }
}

// ------------------------------------------------------------ side momentum

// tick side loop (solver_compact.py:439-486)
template <bool kHanging, bool kThetaOne>
__global__ void k_sides(Dev d)
{
    const nhf_mesh &m = d.m;
    int si = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (si >= m.s_num) return;
    const Ctl *c = d.ctl;
    if (!c->active) return;
    const real dt = c->dt;
    real bf = m.sbf[si] == 1 ? RC(0.0) : RC(1.0);
    int so = m.topology[3 * si], el = m.topology[3 * si + 1], eh = m.topology[3 * si + 2];
    real zl = m.bed[el], zh = m.bed[eh];
    real hl = zl + m.depth[el], hr = zh + m.depth[eh];
    real dx = d.sdc[si];
    real xq = m.q[si];
    real xwh = rmax(hl, hr) - rmax(rmax(zl, zh), kDh);
    real difference = hr - hl;
    if (kHanging) difference = pressure_difference(d, m.depth, si, el, eh, difference);
    real xdq = (d.neg_g * difference / dx) * rmax(xwh, RC(0.0)) * dt;
    real n = m.side_n[si];
    real ratio = RC(0.0);
    // xq / p with p = max(wh, 1e-5) ** f32(7/3) > 0: a zero discharge gives a
    // zero ratio without evaluating the power (identical bits).
    if (xq != RC(0.0)) ratio = xq / nhf::pow_real(rmax(xwh, RC(0.00001)), d.seven_thirds);
    real xf = RC(1.0) + d.g * dt * (n * n) * fabs(ratio);
    int dl = so == 2 ? 0 : 2, dr = so == 2 ? 1 : 3;
    real nb;
    if (kThetaOne) {
        nb = RC(0.0) + RC(0.0);
    } else {
        nb = boundary_neighbor_sum(xq, d.face_qn[4 * el + dl], d.face_qn[4 * eh + dr],
                                   m.open_face[4 * el + dl], m.open_face[4 * eh + dr]);
    }
    real new_q = (d.sita * xq + d.half_rest * nb + xdq) / xf;
    new_q = xwh < d.min_h ? RC(0.0) : new_q;
    new_q *= bf;
    m.q[si] = new_q;
}

// ----------------------------------------------------------- donor factor

// tick cell loop 1 (solver_compact.py:491-514)
__global__ void k_donor(Dev d)
{
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    int ei = blockIdx.x * blockDim.x + threadIdx.x + 1;
    bool valid = ei < m.e_num;
    if (!c->active) return;
    const real dt = c->dt;
    bool limited = false;
    real sc = RC(1.0);
    if (valid) {
        int bi = m.boundary_id[ei];
        real discharge = RC(0.0);
        int kind = bi >= 0 ? m.kind[bi] : -1;
        if (kind == 1) discharge = d.values[bi] * m.weight[ei];
        real rainq = RC(0.0);
        if (c->raining) rainq = d.rain_rates[m.rain_index[ei]];
        real pipe = RC(0.0);
        real positive = (rmax(pipe, RC(0.0)) + rmax(discharge, RC(0.0))) * dt;
        real area = m.area[ei];
        real available = m.depth[ei] * area + positive + rainq * dt * area;
        real outgoing = (rmax(-pipe, RC(0.0)) + rmax(-discharge, RC(0.0))) * dt;
        for (int dd = 0; dd < 4; ++dd) {
            int p = m.face_ptr[4 * ei + dd], cnt = m.face_count[4 * ei + dd];
            for (int j = 0; j < cnt; ++j) {
                int side = m.isl_data[p + j];
                real signed_q = m.q[side] * m.length[side];
                if (dd == 0 || dd == 2) signed_q = -signed_q;
                outgoing += rmax(signed_q, RC(0.0)) * dt;
            }
        }
        if (outgoing > available && kind != 0) {
            sc = available / outgoing;
            limited = true;
        }
        d.donor_scale[ei] = sc;
    }
    unsigned mask = __ballot_sync(0xffffffffu, limited);
    if (mask) {
        scale_bits_t bits = real_bits(sc);  // scale >= 0: bit order is value order
        for (int o = 16; o > 0; o >>= 1) {
            scale_bits_t w = __shfl_down_sync(0xffffffffu, bits, o);
            bits = w < bits ? w : bits;
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(&c->limited_cells, (uint32_t)__popc(mask));
            atomicMin(&c->min_scale_bits, bits);
        }
    }
}

// ------------------------------------------------------------ side scaling

// tick side loop 2 (solver_compact.py:516-522)
__global__ void k_scale(Dev d)
{
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    int si = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (!c->active) return;
    bool counted = false;
    if (si < m.s_num) {
        int el = m.topology[3 * si + 1], eh = m.topology[3 * si + 2];
        real q = m.q[si];
        int donor = q >= RC(0.0) ? el : eh;
        real sc = d.donor_scale[donor];
        counted = q != RC(0.0) && sc < RC(1.0);
        m.q[si] = q * sc;
    }
    unsigned mask = __ballot_sync(0xffffffffu, counted);
    if (mask && (threadIdx.x & 31) == 0) atomicAdd(&c->limited_faces, (uint32_t)__popc(mask));
}

// ------------------------------------------------------------- cell update

// tick cell loops 2 and 3 (solver_compact.py:525-610) for one 256-cell budget
// block; the per-block budget partials have one writer. kGate adds the gate
// controller's record_cell, measure_inventory and rounding collection
// (solver_compact.py:595-604; gate.py:151-193) for pond and gate cells.
template <bool kGate>
__global__ void __launch_bounds__(kBlock) k_cells(Dev d, GateDev g)
{
    __shared__ double sh[kBlock];
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    if (!c->active) return;
    const real dt = c->dt;
    const int T = d.terms;
    const int B = m.b_num;
    const int blk = blockIdx.x;
    const int ei = blk * kBlock + threadIdx.x;
    const bool valid = ei >= 1 && ei < m.e_num;
    real t_removed = RC(0.0), t_pipe = RC(0.0), t_floor = RC(0.0);
    real t_level[5] = {RC(0.0), RC(0.0), RC(0.0), RC(0.0), RC(0.0)};
    real t_discharge = RC(0.0);
    int bi = -1, kind = -1;
    bool wet = false;
    int goff = -1;
    real gv[6] = {RC(0.0), RC(0.0), RC(0.0), RC(0.0), RC(0.0), RC(0.0)};
    if (valid) {
        bi = m.boundary_id[ei];
        kind = bi >= 0 ? m.kind[bi] : -1;
        real sc = d.donor_scale[ei];
        real pq = RC(0.0);
        real pipe = rmax(pq, RC(0.0)) + rmin(pq, RC(0.0)) * sc;
        real discharge = RC(0.0);
        if (kind == 1) {
            real requested = d.values[bi] * m.weight[ei];
            discharge = rmax(requested, RC(0.0)) + rmin(requested, RC(0.0)) * sc;
            t_discharge = discharge * dt;
        }
        real ssq = pipe + discharge;
        real rainq = RC(0.0);
        if (c->raining) rainq = d.rain_rates[m.rain_index[ei]];
        real infil = m.infiltration[ei];
        if (rainq > RC(0.0)) {
            real rt = m.rain_time[ei] + dt;
            m.rain_time[ei] = rt;
            real f0 = m.f0[ei], fc = m.fc[ei];
            real diff = f0 - fc;
            // fc + 0 * e == fc for the finite e in (0, 1]: skip exp when f0 == fc.
            infil = diff == RC(0.0) ? fc + RC(0.0) : fc + diff * nhf::exp_real(-m.k[ei] * rt / RC(3600.0));
            m.infiltration[ei] = infil;
        }
        real fl[4];
        for (int dd = 0; dd < 4; ++dd) {
            real face_flux = RC(0.0);
            int p = m.face_ptr[4 * ei + dd], cnt = m.face_count[4 * ei + dd];
            for (int j = 0; j < cnt; ++j) {
                int si = m.isl_data[p + j];
                face_flux += m.q[si] * m.length[si];
            }
            fl[dd] = face_flux;
        }
        real ql = fl[0], qr = fl[1], qb = fl[2], qt = fl[3];
        real tq = ql - qr + qb - qt + ssq;
        store4(d.eq + 4 * (size_t)ei, ql, qr, qb, qt);
        real ea = m.area[ei];
        real rain_depth = rainq * dt;
        real increment = tq * dt / ea + rain_depth;
        real previous = m.depth[ei];
        real raw_depth = previous + increment;
        real removed = rmin(infil * dt, rmax(raw_depth, RC(0.0)));
        raw_depth -= removed;
        real floor_v = rmax(-raw_depth, RC(0.0));
        t_removed = removed * ea;
        t_pipe = pipe * dt;
        real depth;
        if (kind == 0) {
            t_floor = floor_v * ea;
            real target = rmax(d.level_values[bi] - m.bed[ei], RC(0.0));
            t_level[0] = (target - previous) * ea;
            t_level[1] = -(ql - qr + qb - qt) * dt;
            t_level[2] = -pipe * dt;
            t_level[3] = -rain_depth * ea;
            t_level[4] = removed * ea;
            depth = target;
        } else {
            t_floor = floor_v * ea;
            depth = rmax(raw_depth, RC(0.0));
        }
        m.depth[ei] = depth;
        if (kGate) {
            goff = g.pond[ei] == 1 ? 4 * g.count + 2
                 : (g.cell_gate[ei] >= 0 ? 4 * g.count + 8 + 6 * g.cell_gate[ei] : -1);
            if (goff >= 0) {
                real applied_floor = floor_v, level_exchange = RC(0.0);
                if (kind == 0) {
                    applied_floor = RC(0.0);
                    level_exchange = (depth - previous) * ea - (ql - qr + qb - qt) * dt - pipe * dt
                                     - rain_depth * ea + removed * ea;
                }
                gv[0] = rain_depth * ea;
                gv[1] = removed * ea;
                gv[2] = applied_floor * ea;
                gv[3] = pipe * dt;
                gv[4] = (ssq - pipe) * dt + level_exchange;
                real rounding = (depth - previous) - increment + removed - applied_floor;
                gv[5] = rounding * ea - level_exchange;
            }
        }
        real h = rmax(depth, RC(0.01));
        real u = RC(0.0), v = RC(0.0);
        if (depth >= d.min_h) {
            u = (ql + qr) / m.height[ei] / h / RC(2.0);
            v = (qb + qt) / m.width[ei] / h / RC(2.0);
        }
        m.u[ei] = u; m.v[ei] = v;
        m.max_speed[ei] = rmax(m.max_speed[ei], sqrt(u * u + v * v));
        if (depth > m.max_depth[ei]) {
            m.max_depth[ei] = depth;
            m.peak_hi[ei] = c->step_end[0]; m.peak_lo[ei] = c->step_end[1];
        }
        wet = depth >= d.min_h;
    }
    int wet_count = __syncthreads_count(wet);
    if (threadIdx.x == 0 && wet_count) atomicAdd(&c->wet, (uint32_t)wet_count);

    double *acc_s = d.acc_sum + (size_t)blk * T;
    double *acc_c = d.acc_comp + (size_t)blk * T;
    for (int t = 0; t < T; ++t) {
        real val = RC(0.0);
        if (t == 0) val = t_removed;
        else if (t == 1) val = kind == 0 ? RC(0.0) : t_floor;
        else if (t == 2) val = kind == 0 ? t_floor : RC(0.0);
        else if (t == 3) val = t_pipe;
        else if (t < 4 + 5 * B) { int b = (t - 4) / 5; if (b == bi) val = t_level[(t - 4) % 5]; }
        else { int b = t - 4 - 5 * B; if (b == bi) val = t_discharge; }
        if (!__syncthreads_or(val != RC(0.0))) continue;
        double sum = block_tree((double)val, sh);
        if (threadIdx.x == 0) acc_add(acc_s + t, acc_c + t, sum);
    }
    if (kGate) {
        // the pond group, then gate by gate: six terms each
        for (int grp = -1; grp < g.count; ++grp) {
            const int off = grp < 0 ? 4 * g.count + 2 : 4 * g.count + 8 + 6 * grp;
            if (!__syncthreads_or(goff == off)) continue;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                real val = goff == off ? gv[k] : RC(0.0);
                if (!__syncthreads_or(val != RC(0.0))) continue;
                double sum = block_tree((double)val, sh);
                if (threadIdx.x == 0) {
                    size_t idx = (size_t)blk * g.terms + off + k;
                    acc_add(g.acc_sum + idx, g.acc_comp + idx, sum);
                }
            }
        }
    }
}

// ------------------------------------------------------------ gate control

// check (gate.py:88-99) and move, one block: at_end = 0 is check_gates at
// the step start (irreversible command once the control cell is wet above
// the trigger, from formal time 0 on, then the beds at now); at_end = 1 is
// finish_gate_bed (the beds at the step end).
__global__ void __launch_bounds__(256) k_gate_move(Dev d, GateDev g, int at_end)
{
    const Ctl *c = d.ctl;
    if (!c->active) return;
    const uint32_t hi = at_end ? c->step_end[0] : c->now[0];
    const uint32_t lo = at_end ? c->step_end[1] : c->now[1];
    if (!at_end) {
        gate_check(d, g, hi, lo);
        __syncthreads();
    }
    gate_move_beds(d, g, hi, lo);
}

// record_flux (gate.py:118-140) on the post-limiter volume of each recorded
// side, per 256 entries of the side list; the first nonzero gate-to-pond
// volume latches the gate's first-flow time.
// move_end (fused step): block 0 then also does finish_gate_bed, which the
// volumes do not read.
__global__ void __launch_bounds__(kBlock) k_gate_flux(Dev d, GateDev g, int move_end)
{
    __shared__ double sh[kBlock];
    const nhf_mesh &m = d.m;
    const Ctl *c = d.ctl;
    if (!c->active) return;
    const int p = blockIdx.x * kBlock + threadIdx.x;
    int term = -1;
    real v0 = RC(0.0), v1 = RC(0.0);
    if (p < g.n_flux) {
        int si = g.flux_sides[p];
        int left = m.topology[3 * si + 1], right = m.topology[3 * si + 2];
        real volume = cur_q(d, c->parity)[si] * m.length[si] * c->dt;
        int gl = g.cell_gate[left], gr = g.cell_gate[right];
        int pl = g.pond[left], pr = g.pond[right];
        int latch = -1;
        real into = RC(0.0);
        if (gl >= 0 && gr < 0) {
            if (pr == 1) { term = 4 * gl; into = volume; latch = gl; }
            else { term = 4 * gl + 2; into = -volume; }
        } else if (gr >= 0 && gl < 0) {
            if (pl == 1) { term = 4 * gr; into = -volume; latch = gr; }
            else { term = 4 * gr + 2; into = volume; }
        } else if (pl != pr) {
            term = 4 * g.count;
            into = pr == 1 ? volume : -volume;
        }
        if (latch >= 0 && volume != RC(0.0) && atomicOr(&g.flow_seen[latch], 1) == 0) {
            g.first_flow[2 * latch] = c->step_end[0]; g.first_flow[2 * latch + 1] = c->step_end[1];
        }
        v0 = rmax(into, RC(0.0));
        v1 = rmax(-into, RC(0.0));
    }
    const int T = 4 * g.count + 2;
    for (int t = 0; t < T; ++t) {
        real val = term < 0 ? RC(0.0) : (t == term ? v0 : (t == term + 1 ? v1 : RC(0.0)));
        if (!__syncthreads_or(val != RC(0.0))) continue;
        double sum = block_tree((double)val, sh);
        if (threadIdx.x == 0) {
            size_t idx = (size_t)blockIdx.x * g.terms + t;
            acc_add(g.acc_sum + idx, g.acc_comp + idx, sum);
        }
    }
    if (move_end && blockIdx.x == 0) gate_move_beds(d, g, c->step_end[0], c->step_end[1]);
}

// --------------------------------------------------------------------- CFL

// compute_cfl (solver_compact.py:617-641) + finish_step (384-391).
// Packed key (cfl bits << 32 | side): the minimum is the smallest CFL and,
// among equal values, the lowest side id, as the reference's second pass.
// The FP64 build cannot pack a double and a side id in 64 bits: it takes the
// reference's two passes, the minimum's bits (k_cfl) and then the lowest
// side attaining it (k_cfl_arg).
__global__ void k_cfl(Dev d, int finish)
{
    __shared__ unsigned long long sh[32];
    __shared__ bool last;
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    if (!c->active) {
        if (finish && blockIdx.x == 0 && threadIdx.x == 0) c->slot += 1;
        return;
    }
    unsigned long long best = kCflEmpty;
    for (int si = blockIdx.x * blockDim.x + threadIdx.x + 1; si < m.s_num; si += gridDim.x * blockDim.x) {
        int el = m.topology[3 * si + 1], eh = m.topology[3 * si + 2];
        if (el != 0 && eh != 0) {
            real h = cfl_face_depth(m.bed[el], m.depth[el], m.bed[eh], m.depth[eh]);
            real cfl = cfl_value(d.afa, d.g, m.length[si], m.q[si], h);
#ifdef NHF_REAL_DOUBLE
            unsigned long long key = (unsigned long long)__double_as_longlong(cfl);
#else
            unsigned long long key = ((unsigned long long)__float_as_uint(cfl) << 32) | (unsigned)si;
#endif
            best = key < best ? key : best;
        }
    }
    best = warp_min_u64(best);
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = best;
    __syncthreads();
    if (warp == 0) {
        best = lane < (int)(blockDim.x >> 5) ? sh[lane] : kCflEmpty;
        best = warp_min_u64(best);
        if (lane == 0) {
            if (best != kCflEmpty) atomicMin(&c->cfl_packed, best);
            __threadfence();
            unsigned ticket = atomicAdd(&c->done_blocks, 1u);
            last = ticket == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    unsigned long long packed = atomicExch(&c->cfl_packed, kCflEmpty);
    c->done_blocks = 0;
#ifdef NHF_REAL_DOUBLE
    c->cfl_min_bits = packed;
    c->ndt = packed == kCflEmpty ? __longlong_as_double(0x7ff0000000000000LL) : __longlong_as_double((long long)packed);
    c->cfl_arg_min = m.s_num;
#else
    if (packed == kCflEmpty) {
        c->ndt = __uint_as_float(0x7f800000u);
        c->cfl_arg = 0;
    } else {
        c->ndt = __uint_as_float((uint32_t)(packed >> 32));
        c->cfl_arg = (int32_t)(packed & 0xffffffffu);
    }
    if (finish) finish_step(c);
#endif
}

#ifdef NHF_REAL_DOUBLE
// The lowest interior side whose CFL value equals the minimum (0 when there
// is none), then finish_step.
__global__ void k_cfl_arg(Dev d, int finish)
{
    __shared__ int sh[32];
    __shared__ bool last;
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    if (!c->active) {
        if (finish && blockIdx.x == 0 && threadIdx.x == 0) c->slot += 1;
        return;
    }
    const unsigned long long target = c->cfl_min_bits;
    int best = m.s_num;
    if (target != kCflEmpty) {
        for (int si = blockIdx.x * blockDim.x + threadIdx.x + 1; si < m.s_num; si += gridDim.x * blockDim.x) {
            int el = m.topology[3 * si + 1], eh = m.topology[3 * si + 2];
            if (el != 0 && eh != 0) {
                real h = cfl_face_depth(m.bed[el], m.depth[el], m.bed[eh], m.depth[eh]);
                real cfl = cfl_value(d.afa, d.g, m.length[si], m.q[si], h);
                if ((unsigned long long)__double_as_longlong(cfl) == target && si < best) best = si;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        int w = __shfl_down_sync(0xffffffffu, best, o);
        best = w < best ? w : best;
    }
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = best;
    __syncthreads();
    if (warp == 0) {
        best = lane < (int)(blockDim.x >> 5) ? sh[lane] : m.s_num;
        for (int o = 16; o > 0; o >>= 1) {
            int w = __shfl_down_sync(0xffffffffu, best, o);
            best = w < best ? w : best;
        }
        if (lane == 0) {
            if (best < m.s_num) atomicMin(&c->cfl_arg_min, best);
            __threadfence();
            unsigned ticket = atomicAdd(&c->done_blocks, 1u);
            last = ticket == gridDim.x - 1;
        }
    }
    __syncthreads();
    if (!last || threadIdx.x != 0) return;
    __threadfence();
    c->done_blocks = 0;
    const int arg = atomicExch(&c->cfl_arg_min, m.s_num);
    c->cfl_arg = arg >= m.s_num ? 0 : arg;
    if (finish) finish_step(c);
}
#endif

// ------------------------------------------------------- setup and sampling

// apply_initial_levels (solver_compact.py:412-420)
__global__ void __launch_bounds__(kBlock) k_apply_levels(Dev d, const real *targets)
{
    __shared__ double sh[kBlock];
    const nhf_mesh &m = d.m;
    const int T = d.terms;
    int blk = blockIdx.x, ei = blk * kBlock + threadIdx.x;
    int bi = -1;
    real val = RC(0.0);
    if (ei >= 1 && ei < m.e_num) {
        bi = m.boundary_id[ei];
        if (bi >= 0 && m.kind[bi] == 0) {
            real previous = m.depth[ei];
            m.depth[ei] = targets[ei];
            val = (targets[ei] - previous) * m.area[ei];
        } else {
            bi = -1;
        }
    }
    for (int b = 0; b < m.b_num; ++b) {
        real v = b == bi ? val : RC(0.0);
        if (!__syncthreads_or(v != RC(0.0))) continue;
        double sum = block_tree((double)v, sh);
        int t = 4 + 5 * b;
        if (threadIdx.x == 0) acc_add(d.acc_sum + (size_t)blk * T + t, d.acc_comp + (size_t)blk * T + t, sum);
    }
}

// initial_diagnostics (solver_compact.py:657-672)
__global__ void k_initial_diag(Dev d)
{
    const nhf_mesh &m = d.m;
    int ei = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (ei >= m.e_num) return;
    real fl[4];
    for (int dd = 0; dd < 4; ++dd) {
        real total = RC(0.0);
        int p = m.face_ptr[4 * ei + dd], cnt = m.face_count[4 * ei + dd];
        for (int j = 0; j < cnt; ++j) {
            int si = m.isl_data[p + j];
            total += m.q[si] * m.length[si];
        }
        fl[dd] = total;
    }
    store4(d.eq + 4 * (size_t)ei, fl[0], fl[1], fl[2], fl[3]);
    real depth = m.depth[ei];
    real h = rmax(depth, RC(0.01));
    real u = RC(0.0), v = RC(0.0);
    if (depth >= d.min_h) {
        u = (fl[0] + fl[1]) / m.height[ei] / h / RC(2.0);
        v = (fl[2] + fl[3]) / m.width[ei] / h / RC(2.0);
    }
    m.u[ei] = u; m.v[ei] = v;
    m.max_speed[ei] = rmax(m.max_speed[ei], sqrt(u * u + v * v));
    if (depth > m.max_depth[ei]) {
        m.max_depth[ei] = depth;
        m.peak_hi[ei] = d.ctl->now[0]; m.peak_lo[ei] = d.ctl->now[1];
    }
}

// reset_extrema (solver_compact.py:674-679)
__global__ void k_reset_extrema(Dev d)
{
    const nhf_mesh &m = d.m;
    int ei = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (ei >= m.e_num) return;
    m.max_depth[ei] = m.depth[ei];
    real u = m.u[ei], v = m.v[ei];
    m.max_speed[ei] = sqrt(u * u + v * v);
    m.peak_hi[ei] = d.ctl->now[0]; m.peak_lo[ei] = d.ctl->now[1];
}

// sample_stations (solver_compact.py:681-687)
__global__ void k_sample(Dev d, const int32_t *ids, int n, real *out)
{
    const nhf_mesh &m = d.m;
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int ei = ids[i];
    out[4 * i + 0] = m.depth[ei];
    out[4 * i + 1] = m.bed[ei] + m.depth[ei];
    out[4 * i + 2] = m.u[ei];
    out[4 * i + 3] = m.v[ei];
}

// ndt, flow depth of the limiting side, and the side (an int32 after the two values)
__global__ void k_cfl_edge(Dev d, real *out)
{
    const Ctl *c = d.ctl;
    out[0] = c->ndt;
    out[1] = flow_depth_of(d.m, d.m.depth, c->cfl_arg);
    *reinterpret_cast<int32_t *>(out + 2) = c->cfl_arg;
}

// eq_t from the current discharges (solver_compact.py:548-559 face sums)
__global__ void k_eq(Dev d)
{
    const nhf_mesh &m = d.m;
    int ei = blockIdx.x * blockDim.x + threadIdx.x + 1;
    if (ei >= m.e_num) return;
    real fl[4];
    for (int dd = 0; dd < 4; ++dd) {
        real total = RC(0.0);
        int p = m.face_ptr[4 * ei + dd], cnt = m.face_count[4 * ei + dd];
        for (int j = 0; j < cnt; ++j) {
            int si = m.isl_data[p + j];
            total += m.q[si] * m.length[si];
        }
        fl[dd] = total;
    }
    store4(d.eq + 4 * (size_t)ei, fl[0], fl[1], fl[2], fl[3]);
}

}  // namespace

// ============================================================== host side

#include "nhf_handle.cuh"

namespace {

std::string g_create_error;

int fail(nhf_handle *h, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (h) h->err = buf; else g_create_error = buf;
    return code;
}

#define CK(h, call)                                                                         \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return fail((h), NHF_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_));    \
    } while (0)

inline int grid_for(int n, int b) { return n <= 0 ? 1 : (n + b - 1) / b; }

// compute_cfl, and finish_step when `finish`: one pass, or two in the FP64 build
void enqueue_cfl(nhf_handle *h, cudaStream_t s, int finish)
{
    int gc = grid_for(h->m.s_num - 1, 256);
    if (gc > 148 * 8) gc = 148 * 8;
    k_cfl<<<gc, 256, 0, s>>>(h->dev, finish);
#ifdef NHF_REAL_DOUBLE
    k_cfl_arg<<<gc, 256, 0, s>>>(h->dev, finish);
#endif
}

int enter(nhf_handle *h)
{
    CK(h, cudaEventRecord(h->ev_in, h->user));
    CK(h, cudaStreamWaitEvent(h->s, h->ev_in, 0));
    return NHF_OK;
}

int leave(nhf_handle *h)
{
    CK(h, cudaGetLastError());
    CK(h, cudaEventRecord(h->ev_out, h->s));
    CK(h, cudaStreamWaitEvent(h->user, h->ev_out, 0));
    return NHF_OK;
}

void enqueue_step(nhf_handle *h)
{
    const Dev &d = h->dev;
    const nhf_mesh &m = h->m;
    cudaStream_t s = h->s;
    k_prepare<<<1, 32, 0, s>>>(d);
    if (h->gate_on) k_gate_move<<<1, 256, 0, s>>>(d, h->gate, 0);
    if (m.hang_cells > 0) k_pressure<<<grid_for(m.hang_cells, 256), 256, 0, s>>>(d);
    if (!d.theta_one) k_face_qn<<<grid_for(m.e_num, 256), 256, 0, s>>>(d);
    int gs = grid_for(m.s_num - 1, 256);
    if (m.hang_cells > 0) {
        if (d.theta_one) k_sides<true, true><<<gs, 256, 0, s>>>(d);
        else k_sides<true, false><<<gs, 256, 0, s>>>(d);
    } else {
        if (d.theta_one) k_sides<false, true><<<gs, 256, 0, s>>>(d);
        else k_sides<false, false><<<gs, 256, 0, s>>>(d);
    }
    k_donor<<<grid_for(m.e_num - 1, 256), 256, 0, s>>>(d);
    k_scale<<<gs, 256, 0, s>>>(d);
    if (h->gate_on) {
        if (h->gate.n_flux > 0) k_gate_flux<<<grid_for(h->gate.n_flux, kBlock), kBlock, 0, s>>>(d, h->gate, 0);
        k_cells<true><<<d.blocks, kBlock, 0, s>>>(d, h->gate);
        k_gate_move<<<1, 256, 0, s>>>(d, h->gate, 1);
    } else {
        k_cells<false><<<d.blocks, kBlock, 0, s>>>(d, h->gate);
    }
    enqueue_cfl(h, s, 1);
}

int build_graph(nhf_handle *h)
{
    cudaGraph_t g = nullptr;
    CK(h, cudaStreamBeginCapture(h->s, cudaStreamCaptureModeThreadLocal));
    k_begin<<<1, 256, 0, h->s>>>(h->dev, 0u, 0u, 0u, 0u, (h->tiled || h->lattice) ? 1 : 0);
#ifndef NHF_REAL_DOUBLE
    if (h->lattice) {
        lattice_enqueue_batch_start(h->dev, h->s);
        for (int i = 0; i < h->p.batch_size; ++i) lattice_enqueue_step(h->dev, h->s);
        lattice_enqueue_batch_end(h->dev, h->s);
    } else if (h->tiled) {
        tiled_enqueue_batch_start(h->dev, h->s);
        for (int i = 0; i < h->p.batch_size; ++i) {
            if (h->gate_on) {
                // check_gates (here for the batch's first step; the CFL pass
                // runs it for the next ones), the step with the source terms,
                // the exchange volumes with finish_gate_bed, the CFL pass
                if (i == 0) k_gate_move<<<1, 256, 0, h->s>>>(h->dev, h->gate, 0);
                tiled_enqueue_step(h->dev, h->tb, h->s, &h->gate);
                // the exchange volumes and finish_gate_bed in one launch
                if (h->gate.n_flux > 0)
                    k_gate_flux<<<grid_for(h->gate.n_flux, kBlock), kBlock, 0, h->s>>>(h->dev, h->gate, 1);
                else
                    k_gate_move<<<1, 256, 0, h->s>>>(h->dev, h->gate, 1);
                tiled_enqueue_cfl(h->dev, h->tb, h->s, &h->gate);
            } else {
                tiled_enqueue_step(h->dev, h->tb, h->s);
            }
        }
        tiled_enqueue_batch_end(h->dev, h->s);
    } else
#endif
    {
        for (int i = 0; i < h->p.batch_size; ++i) enqueue_step(h);
    }
    cudaMemcpyAsync(h->h_trace, h->ctl->trace, sizeof(uint32_t) * NHF_TRACE_COLS * h->p.batch_size,
                    cudaMemcpyDeviceToHost, h->s);
    cudaError_t e = cudaStreamEndCapture(h->s, &g);
    if (e != cudaSuccess) return fail(h, NHF_ECUDA, "graph capture failed: %s", cudaGetErrorString(e));
    // Locate the begin kernel node: its arguments carry each batch's words.
    size_t count = 0;
    cudaGraphGetNodes(g, nullptr, &count);
    cudaGraphNode_t *nodes = (cudaGraphNode_t *)malloc(sizeof(cudaGraphNode_t) * (count ? count : 1));
    cudaGraphGetNodes(g, nodes, &count);
    for (size_t i = 0; i < count && !h->begin_node; ++i) {
        cudaGraphNodeType type;
        cudaGraphNodeGetType(nodes[i], &type);
        if (type != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        if (cudaGraphKernelNodeGetParams(nodes[i], &kp) == cudaSuccess && kp.func == (void *)k_begin) {
            h->begin_node = nodes[i];
            h->begin_params = kp;
        }
    }
    free(nodes);
    if (!h->begin_node) { cudaGraphDestroy(g); return fail(h, NHF_ECUDA, "begin node not found in graph"); }
    e = cudaGraphInstantiate(&h->graph, g, 0);
    if (e != cudaSuccess) { cudaGraphDestroy(g); return fail(h, NHF_ECUDA, "graph instantiate failed: %s", cudaGetErrorString(e)); }
    h->graph_def = g;
    return NHF_OK;
}

}  // namespace

namespace nhf {

// One member's own batch graph for the ensemble's member-graph schedule: the
// member's stream waits for `start`, runs its batch towards `target` and
// records `done`; the trace lands in the member's pinned trace buffer.
int member_graph_prepare(nhf_handle *h)
{
    if (!h->graph) return build_graph(h);
    return NHF_OK;
}

int member_graph_launch(nhf_handle *h, const uint32_t target[2], const uint32_t origin[2], cudaEvent_t start,
                        cudaEvent_t done)
{
    int rc = member_graph_prepare(h);
    if (rc) return rc;
    CK(h, cudaStreamWaitEvent(h->s, start, 0));
    Dev d = h->dev;
    uint32_t w[4] = {target[0], target[1], origin[0], origin[1]};
    int prepare_first = (h->tiled || h->lattice) ? 1 : 0;
    void *args[6] = {&d, &w[0], &w[1], &w[2], &w[3], &prepare_first};
    cudaKernelNodeParams kp = h->begin_params;
    kp.kernelParams = args;
    kp.extra = nullptr;
    CK(h, cudaGraphExecKernelNodeSetParams(h->graph, h->begin_node, &kp));
    CK(h, cudaGraphLaunch(h->graph, h->s));
    CK(h, cudaEventRecord(done, h->s));
    return NHF_OK;
}

}  // namespace nhf

extern "C" {

#ifdef NHF_REAL_DOUBLE
const char *nhf_version(void) { return "nhflood-b200 0.2 (sm_100a, FP64 build)"; }
#else
const char *nhf_version(void) { return "nhflood-b200 0.2 (sm_100a)"; }
#endif

int nhf_real_bytes(void) { return (int)sizeof(nhf_real); }

const char *nhf_last_error(const nhf_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int nhf_create(const nhf_mesh *mesh, const nhf_params *params, void *stream, nhf_handle **out)
{
    if (!mesh || !params || !out) return fail(nullptr, NHF_EINVAL, "null argument");
    *out = nullptr;
    if (mesh->e_num < 1 || mesh->s_num < 1 || mesh->b_num < 0 || mesh->n_rates < 0)
        return fail(nullptr, NHF_EINVAL, "invalid mesh sizes");
    if (params->batch_size < 1 || params->batch_size > NHF_MAX_BATCH)
        return fail(nullptr, NHF_EINVAL, "batch_size must be between 1 and %d", NHF_MAX_BATCH);
    if (params->sita != RC(1) && !mesh->open_face)
        return fail(nullptr, NHF_EINVAL, "theta < 1 needs open_face fractions");
    if (mesh->hang_cells > 0 && (!mesh->edge_index || !mesh->offsets || !mesh->slots || !mesh->hcells || !mesh->axes))
        return fail(nullptr, NHF_EINVAL, "hanging geometry arrays missing");
    nhf_handle *h = new nhf_handle();
    h->m = *mesh;
    h->p = *params;
    h->user = (cudaStream_t)stream;
    int rc;
#define CKC(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            rc = fail(nullptr, NHF_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_));          \
            nhf_destroy(h);                                                                         \
            return rc;                                                                              \
        }                                                                                           \
    } while (0)
    CKC(cudaStreamCreateWithFlags(&h->s, cudaStreamNonBlocking));
    CKC(cudaEventCreateWithFlags(&h->ev_in, cudaEventDisableTiming));
    CKC(cudaEventCreateWithFlags(&h->ev_out, cudaEventDisableTiming));
    const int e = mesh->e_num, sn = mesh->s_num, bb = mesh->b_num > 0 ? mesh->b_num : 1;
    const int T = 4 + 6 * mesh->b_num;
    const int blocks = (e + kBlock - 1) / kBlock;
    const int hc = mesh->hang_cells > 0 ? mesh->hang_cells : 1;
    const int nr = mesh->n_rates > 0 ? mesh->n_rates : 1;
    const bool theta_one = params->sita == RC(1);
    // The caller may still be writing the mesh arrays on its stream.
    CKC(cudaEventRecord(h->ev_in, h->user));
    CKC(cudaStreamWaitEvent(h->s, h->ev_in, 0));
#ifdef NHF_REAL_DOUBLE
    h->path = "multipass (FP64 build)";
#else
    // Lattice form when the mesh is a uniform grid it covers (params->path 2,
    // or 0 from 2^20 cells on: on smaller grids a march of a few rows is
    // latency-bound and the tiled step is faster).
    if (params->path == 2 || (params->path == 0 && mesh->e_num - 1 >= (1 << 20))) {
        Dev probe{};
        probe.m = *mesh;
        probe.terms = 4 + 6 * mesh->b_num;
        probe.blocks = (mesh->e_num + kBlock - 1) / kBlock;
        probe.theta_one = params->sita == RC(1) ? 1 : 0;
        char why[256] = {0};
        if (lattice_build(probe, h->s, &h->lb, why, sizeof(why)) == 0) {
            h->lattice = true;
            char buf[160];
            snprintf(buf, sizeof(buf), "lattice(%dx%d,strips=%d,rows=%d,warps=%d,blocks=%d)", h->lb.plan.nx,
                     h->lb.plan.ny, h->lb.plan.strips, h->lb.plan.rows, h->lb.plan.block_warps,
                     h->lb.plan.min_blocks);
            h->path = buf;
        } else {
            if (h->lb.device_memory) { cudaFree(h->lb.device_memory); h->lb.device_memory = nullptr; }
            h->path = std::string("multipass (lattice: ") + why + ")";
        }
    }
    // Fused tiled step when the mesh allows it (params->path 0, or a tile size).
    if (!h->lattice && (params->path == 0 || params->path == 3 || params->path == 256 || params->path == 512 ||
                        params->path == 1024)) {
        char why[256] = {0};
        if (params->cfl_mode < 0 || params->cfl_mode > 2) {
            rc = fail(nullptr, NHF_EINVAL, "cfl_mode must be 0, 1 or 2");
            nhf_destroy(h);
            return rc;
        }
        if (tiled_build(*mesh, h->s, &h->tb, why, sizeof(why), params->path == 3 ? 0 : params->path,
                        params->cfl_mode) == 0) {
            h->tiled = true;
            char buf[160];
            snprintf(buf, sizeof(buf), "tiled(tile=%d,patterns=%d,smem=%zu,cfl=%s)", h->tb.plan.tile,
                     h->tb.patterns, h->tb.shared_bytes, h->tb.plan.split ? "pass" : "fused");
            h->path = buf;
        } else {
            h->path = std::string("multipass (") + why + ")";
        }
    }
#endif
    // scratch layout (bytes, 256-aligned pieces)
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    size_t o_ctl = take(sizeof(Ctl));
    size_t o_coef = take(sizeof(real) * 2 * bb);
    size_t o_val = take(sizeof(real) * bb);
    size_t o_lvl = take(sizeof(real) * bb);
    size_t o_rain = take(sizeof(real) * nr);
    size_t o_sdc = take(sizeof(real) * sn);
    size_t o_donor = take(sizeof(real) * e);
    size_t o_fqn = take(theta_one ? 32 : sizeof(real) * 4 * (size_t)e);
    size_t o_eq = take(sizeof(real) * 4 * (size_t)e);
    size_t o_grad = take(sizeof(real) * 2 * hc);
    size_t o_accs = take(sizeof(double) * (size_t)blocks * T);
    size_t o_accc = take(sizeof(double) * (size_t)blocks * T);
    size_t o_begin = take(sizeof(real) * 4);  // also the staging of nhf_get_cfl's three words
    size_t o_db = h->tiled ? take(sizeof(real) * (size_t)e) : 0;
    size_t o_qb = h->tiled ? take(sizeof(real) * (size_t)sn) : 0;
    size_t o_rb = h->tiled ? take(sizeof(real) * (size_t)e) : 0;
    size_t o_sdn = h->tiled ? take(sizeof(float2) * (size_t)sn) : 0;
    CKC(cudaMalloc(&h->scratch, off));
    CKC(cudaMemsetAsync(h->scratch, 0, off, h->s));
    char *base = (char *)h->scratch;
    h->ctl = (Ctl *)(base + o_ctl);
    h->d_begin = (uint32_t *)(base + o_begin);
    CKC(cudaMallocHost(&h->h_begin, 4 * sizeof(uint32_t)));
    CKC(cudaMallocHost(&h->h_trace, sizeof(uint32_t) * NHF_TRACE_COLS * NHF_MAX_BATCH));
    CKC(cudaMallocHost(&h->h_small, sizeof(real) * (2 * bb + nr + 64)));
    CKC(cudaMallocHost(&h->h_acc, sizeof(double) * 2 * (size_t)blocks * T + 16));
    Dev &d = h->dev;
    d.m = *mesh;
    d.g = params->g;
    d.neg_g = -params->g;
    d.afa = params->afa;
    d.sita = params->sita;
    d.half_rest = (real)((1.0 - (double)params->sita) / 2.0);
    d.seven_thirds = (real)(7.0 / 3.0);
    d.min_h = params->min_h;
    d.min_dt = params->min_dt;
    d.terms = T;
    d.blocks = blocks;
    d.batch_size = params->batch_size;
    d.theta_one = theta_one ? 1 : 0;
    d.ctl = h->ctl;
    d.coef = (const real *)(base + o_coef);
    d.values = (real *)(base + o_val);
    d.level_values = (real *)(base + o_lvl);
    d.rain_rates = (real *)(base + o_rain);
    d.sdc = (real *)(base + o_sdc);
    d.donor_scale = (real *)(base + o_donor);
    d.face_qn = (real *)(base + o_fqn);
    d.eq = (real *)(base + o_eq);
    d.gradients = (real *)(base + o_grad);
    d.acc_sum = (double *)(base + o_accs);
    d.acc_comp = (double *)(base + o_accc);
    if (h->tiled) {
        d.depth_b = (real *)(base + o_db);
        d.q_b = (real *)(base + o_qb);
        d.rain_time_b = (real *)(base + o_rb);
        d.sdn = (float2 *)(base + o_sdn);
        d.plan = h->tb.plan;
    }
#ifndef NHF_REAL_DOUBLE
    if (h->lattice) d.lat = h->lb.plan;
#endif
    // control block initial values
    Ctl init{};
    init.limit_value[0] = __builtin_inff();
    init.cfl_packed = kCflEmpty;
    init.ndt = RC(0);
    init.cfl_min_bits = kCflEmpty;
    init.cfl_arg_min = mesh->s_num;
    CKC(cudaMemcpyAsync(h->ctl, &init, sizeof(Ctl), cudaMemcpyHostToDevice, h->s));
    CKC(cudaStreamSynchronize(h->s));
#undef CKC
    *out = h;
    return NHF_OK;
}

int nhf_destroy(nhf_handle *h)
{
    if (!h) return NHF_OK;
    if (h->s) cudaStreamSynchronize(h->s);
    if (h->graph) cudaGraphExecDestroy(h->graph);
    if (h->graph_def) cudaGraphDestroy(h->graph_def);
    if (h->tb.device_memory) cudaFree(h->tb.device_memory);
    if (h->lb.device_memory) cudaFree(h->lb.device_memory);
    if (h->scratch) cudaFree(h->scratch);
    if (h->h_begin) cudaFreeHost(h->h_begin);
    if (h->h_trace) cudaFreeHost(h->h_trace);
    if (h->h_small) cudaFreeHost(h->h_small);
    if (h->h_acc) cudaFreeHost(h->h_acc);
    if (h->d_ids) cudaFree(h->d_ids);
    if (h->d_samples) cudaFree(h->d_samples);
    if (h->gate_mem) cudaFree(h->gate_mem);
    if (h->h_gacc) cudaFreeHost(h->h_gacc);
    if (h->ev_in) cudaEventDestroy(h->ev_in);
    if (h->ev_out) cudaEventDestroy(h->ev_out);
    if (h->s) cudaStreamDestroy(h->s);
    delete h;
    return NHF_OK;
}

int nhf_initialize(nhf_handle *h)
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    int n = h->m.e_num > h->m.s_num ? h->m.e_num : h->m.s_num;
    k_initialize<<<grid_for(n, 256), 256, 0, h->s>>>(h->dev);
    return leave(h);
}

int nhf_set_clock(nhf_handle *h, const uint32_t now[2])
{
    if (!h || !now) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    memcpy(h->h_small, now, 2 * sizeof(uint32_t));
    CK(h, cudaMemcpyAsync(h->ctl->now, h->h_small, 2 * sizeof(uint32_t), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return leave(h);
}

int nhf_get_clock(nhf_handle *h, uint32_t now[2])
{
    if (!h || !now) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    CK(h, cudaMemcpyAsync(h->h_small, h->ctl->now, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    memcpy(now, h->h_small, 2 * sizeof(uint32_t));
    return leave(h);
}

int nhf_set_active(nhf_handle *h, int32_t active)
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    memcpy(h->h_small, &active, sizeof(int32_t));
    CK(h, cudaMemcpyAsync(&h->ctl->active, h->h_small, sizeof(int32_t), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return leave(h);
}

int nhf_set_forcing(nhf_handle *h, const nhf_real *coefficients, const nhf_real *rain_rates, int32_t raining)
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    const int bb = h->m.b_num > 0 ? h->m.b_num : 1;
    real *stage = h->h_small;
    if (coefficients) {
        memcpy(stage, coefficients, sizeof(real) * 2 * bb);
        CK(h, cudaMemcpyAsync((void *)h->dev.coef, stage, sizeof(real) * 2 * bb, cudaMemcpyHostToDevice, h->s));
    }
    if (rain_rates && h->m.n_rates > 0) {
        memcpy(stage + 2 * bb, rain_rates, sizeof(real) * h->m.n_rates);
        CK(h, cudaMemcpyAsync(h->dev.rain_rates, stage + 2 * bb, sizeof(real) * h->m.n_rates,
                              cudaMemcpyHostToDevice, h->s));
    }
    memcpy(stage + 2 * bb + h->m.n_rates, &raining, sizeof(int32_t));
    CK(h, cudaMemcpyAsync(&h->ctl->raining, stage + 2 * bb + h->m.n_rates, sizeof(int32_t),
                          cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return leave(h);
}

int nhf_apply_initial_levels(nhf_handle *h, const nhf_real *targets)
{
    if (!h || !targets) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    k_apply_levels<<<h->dev.blocks, kBlock, 0, h->s>>>(h->dev, targets);
    return leave(h);
}

int nhf_compute_cfl(nhf_handle *h)
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    enqueue_cfl(h, h->s, 0);
    return leave(h);
}

int nhf_initial_diagnostics(nhf_handle *h)
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    k_initial_diag<<<grid_for(h->m.e_num - 1, 256), 256, 0, h->s>>>(h->dev);
    return leave(h);
}

int nhf_reset_extrema(nhf_handle *h)
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    k_reset_extrema<<<grid_for(h->m.e_num - 1, 256), 256, 0, h->s>>>(h->dev);
    return leave(h);
}

int nhf_run_batch_async(nhf_handle *h, const uint32_t target[2], const uint32_t origin[2])
{
    if (!h || !target || !origin) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    if (!h->graph) { rc = build_graph(h); if (rc) return rc; }
    Dev d = h->dev;
    uint32_t w[4] = {target[0], target[1], origin[0], origin[1]};
    int prepare_first = (h->tiled || h->lattice) ? 1 : 0;
    void *args[6] = {&d, &w[0], &w[1], &w[2], &w[3], &prepare_first};
    cudaKernelNodeParams kp = h->begin_params;
    kp.kernelParams = args;
    kp.extra = nullptr;
    CK(h, cudaGraphExecKernelNodeSetParams(h->graph, h->begin_node, &kp));
    CK(h, cudaGraphLaunch(h->graph, h->s));
    return leave(h);
}

int nhf_read_trace(nhf_handle *h, uint32_t *trace)
{
    if (!h || !trace) return NHF_EINVAL;
    CK(h, cudaStreamSynchronize(h->s));
    memcpy(trace, h->h_trace, sizeof(uint32_t) * NHF_TRACE_COLS * h->p.batch_size);
    return NHF_OK;
}

int nhf_run_batch(nhf_handle *h, const uint32_t target[2], const uint32_t origin[2], uint32_t *trace)
{
    int rc = nhf_run_batch_async(h, target, origin);
    if (rc) return rc;
    return nhf_read_trace(h, trace);
}

int nhf_budget_terms(const nhf_handle *h) { return h ? h->dev.terms : 0; }

int nhf_budget_flush(nhf_handle *h, double *totals)
{
    if (!h || !totals) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    const int T = h->dev.terms, blocks = h->dev.blocks;
    const size_t n = (size_t)blocks * T;
    CK(h, cudaMemcpyAsync(h->h_acc, h->dev.acc_sum, sizeof(double) * n, cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaMemcpyAsync(h->h_acc + n, h->dev.acc_comp, sizeof(double) * n, cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaMemsetAsync(h->dev.acc_sum, 0, sizeof(double) * n, h->s));
    CK(h, cudaMemsetAsync(h->dev.acc_comp, 0, sizeof(double) * n, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    // Host merge: blocks in order, (sum, comp) pairs, Neumaier compensation.
    for (int t = 0; t < T; ++t) {
        double s = 0.0, comp = 0.0;
        for (int b = 0; b < blocks; ++b) {
            double parts[2] = {h->h_acc[(size_t)b * T + t], h->h_acc[n + (size_t)b * T + t]};
            for (int j = 0; j < 2; ++j) {
                double p = parts[j];
                double s2 = s + p;
                if (fabs(s) >= fabs(p)) comp += (s - s2) + p; else comp += (p - s2) + s;
                s = s2;
            }
        }
        totals[t] = s + comp;
    }
    return leave(h);
}

int nhf_gate_attach(nhf_handle *h, const nhf_gate *gate)
{
    if (!h || !gate) return NHF_EINVAL;
#ifdef NHF_REAL_DOUBLE
    return fail(h, NHF_EINVAL, "the FP64 build has no gate controller");
#endif
    if (h->lattice)
        return fail(h, NHF_EINVAL, "gate control runs on the multi-pass step or the fused tiled step, not the "
                                   "lattice form (nhf_params.path = 1, or 256 with cfl_mode 2)");
    if (h->tiled && !(h->tb.plan.tile == 256 && h->tb.plan.split))
        return fail(h, NHF_EINVAL, "gate control runs on the multi-pass step or on the fused step with 256-cell "
                                   "tiles and the separate CFL pass (nhf_params.path = 1, or 256 with cfl_mode 2)");
    if (h->gate_on) return fail(h, NHF_ESTATE, "a gate controller is already attached");
    if (gate->count < 1 || gate->n_targets < 0 || gate->n_flux < 0)
        return fail(h, NHF_EINVAL, "invalid gate sizes");
    if (!gate->cell_gate || !gate->pond || !gate->closed || !gate->controls || !gate->commanded ||
        !gate->command || !gate->flow_seen || !gate->first_flow || !gate->opened || !gate->opened_at ||
        (gate->n_targets > 0 && !gate->targets) || (gate->n_flux > 0 && !gate->flux_sides))
        return fail(h, NHF_EINVAL, "gate array missing");
    if (!(gate->opening_seconds > 0.0f)) return fail(h, NHF_EINVAL, "opening_seconds must be positive");
    GateDev &g = h->gate;
    g.count = gate->count; g.n_targets = gate->n_targets; g.n_flux = gate->n_flux;
    g.terms = 10 * gate->count + 8;
    const int flux_blocks = grid_for(gate->n_flux, kBlock);
    g.blocks = flux_blocks > h->dev.blocks ? flux_blocks : h->dev.blocks;
    g.cell_gate = gate->cell_gate; g.pond = gate->pond; g.targets = gate->targets;
    g.controls = gate->controls; g.flux_sides = gate->flux_sides; g.closed = gate->closed;
    g.formal_hi = gate->formal_tick[0]; g.formal_lo = gate->formal_tick[1];
    g.trigger_level = gate->trigger_level; g.opening_seconds = gate->opening_seconds;
    g.open_elevation = gate->open_elevation;
    g.commanded = gate->commanded; g.flow_seen = gate->flow_seen; g.opened = gate->opened;
    g.command = gate->command; g.first_flow = gate->first_flow; g.opened_at = gate->opened_at;
    const size_t n = (size_t)g.blocks * g.terms;
    int rc = enter(h); if (rc) return rc;
    CK(h, cudaMalloc(&h->gate_mem, 2 * n * sizeof(double)));
    CK(h, cudaMemsetAsync(h->gate_mem, 0, 2 * n * sizeof(double), h->s));
    CK(h, cudaMallocHost(&h->h_gacc, 2 * n * sizeof(double)));
    g.acc_sum = (double *)h->gate_mem;
    g.acc_comp = g.acc_sum + n;
    h->gate_on = true;
    // the step graph is rebuilt with the gate passes at the next batch
    if (h->graph) { cudaGraphExecDestroy(h->graph); h->graph = nullptr; }
    if (h->graph_def) { cudaGraphDestroy(h->graph_def); h->graph_def = nullptr; }
    h->begin_node = nullptr;
    return leave(h);
}

int nhf_gate_check(nhf_handle *h)
{
    if (!h) return NHF_EINVAL;
    if (!h->gate_on) return fail(h, NHF_ESTATE, "no gate controller attached");
    int rc = enter(h); if (rc) return rc;
    k_gate_move<<<1, 256, 0, h->s>>>(h->dev, h->gate, 0);
    return leave(h);
}

int nhf_gate_terms(const nhf_handle *h) { return h && h->gate_on ? h->gate.terms : 0; }

int nhf_gate_flush(nhf_handle *h, double *totals)
{
    if (!h || !totals) return NHF_EINVAL;
    if (!h->gate_on) return fail(h, NHF_ESTATE, "no gate controller attached");
    int rc = enter(h); if (rc) return rc;
    const int T = h->gate.terms, blocks = h->gate.blocks;
    const size_t n = (size_t)blocks * T;
    CK(h, cudaMemcpyAsync(h->h_gacc, h->gate_mem, 2 * n * sizeof(double), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaMemsetAsync(h->gate_mem, 0, 2 * n * sizeof(double), h->s));
    CK(h, cudaStreamSynchronize(h->s));
    for (int t = 0; t < T; ++t) {
        double s = 0.0, comp = 0.0;
        for (int b = 0; b < blocks; ++b) {
            double parts[2] = {h->h_gacc[(size_t)b * T + t], h->h_gacc[n + (size_t)b * T + t]};
            for (int j = 0; j < 2; ++j) {
                double p = parts[j];
                double s2 = s + p;
                if (fabs(s) >= fabs(p)) comp += (s - s2) + p; else comp += (p - s2) + s;
                s = s2;
            }
        }
        totals[t] = s + comp;
    }
    return leave(h);
}

int nhf_get_cfl(nhf_handle *h, nhf_real *ndt, int32_t *arg, nhf_real *flow_depth)
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    real *out = (real *)h->d_begin;  // 3 words of device staging; graph not running
    CK(h, cudaStreamSynchronize(h->s));
    k_cfl_edge<<<1, 1, 0, h->s>>>(h->dev, out);
    CK(h, cudaMemcpyAsync(h->h_small, out, 3 * sizeof(real), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    if (ndt) *ndt = h->h_small[0];
    if (flow_depth) *flow_depth = h->h_small[1];
    if (arg) memcpy(arg, &h->h_small[2], sizeof(int32_t));
    return leave(h);
}

int nhf_limits(nhf_handle *h, nhf_real values[5], int32_t ids[3])
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    CK(h, cudaMemcpyAsync(h->h_small, h->ctl->limit_value, 5 * sizeof(real), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaMemcpyAsync(h->h_small + 5, h->ctl->limit_ids, 3 * sizeof(int32_t), cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    if (values) memcpy(values, h->h_small, 5 * sizeof(real));
    if (ids) memcpy(ids, h->h_small + 5, 3 * sizeof(int32_t));
    return leave(h);
}

int nhf_reset_limits(nhf_handle *h)
{
    if (!h) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    h->h_small[0] = (real)__builtin_inf();
    CK(h, cudaMemcpyAsync(&h->ctl->limit_value[0], h->h_small, sizeof(real), cudaMemcpyHostToDevice, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return leave(h);
}

int nhf_sample_stations(nhf_handle *h, const int32_t *ids, int32_t n, nhf_real *out)
{
    if (!h || n < 0 || (n > 0 && (!ids || !out))) return NHF_EINVAL;
    if (n == 0) return NHF_OK;
    int rc = enter(h); if (rc) return rc;
    if (n > h->ids_cap) {
        if (h->d_ids) cudaFree(h->d_ids);
        if (h->d_samples) cudaFree(h->d_samples);
        h->d_ids = nullptr; h->d_samples = nullptr;
        CK(h, cudaMalloc(&h->d_ids, sizeof(int32_t) * n));
        CK(h, cudaMalloc(&h->d_samples, sizeof(real) * 4 * n));
        h->ids_cap = n;
    }
    for (int i = 0; i < n; ++i)
        if (ids[i] < 1 || ids[i] >= h->m.e_num) return fail(h, NHF_EINVAL, "station cell %d out of range", ids[i]);
    CK(h, cudaMemcpyAsync(h->d_ids, ids, sizeof(int32_t) * n, cudaMemcpyHostToDevice, h->s));
    k_sample<<<grid_for(n, 128), 128, 0, h->s>>>(h->dev, h->d_ids, n, h->d_samples);
    CK(h, cudaMemcpyAsync(out, h->d_samples, sizeof(real) * 4 * n, cudaMemcpyDeviceToHost, h->s));
    CK(h, cudaStreamSynchronize(h->s));
    return leave(h);
}

int nhf_read_eq(nhf_handle *h, nhf_real *eq)
{
    if (!h || !eq) return NHF_EINVAL;
    int rc = enter(h); if (rc) return rc;
    k_eq<<<grid_for(h->m.e_num - 1, 256), 256, 0, h->s>>>(h->dev);
    CK(h, cudaMemcpyAsync(eq, h->dev.eq, sizeof(real) * 4 * (size_t)h->m.e_num, cudaMemcpyDeviceToDevice, h->s));
    return leave(h);
}

int nhf_read_gradients(nhf_handle *h, nhf_real *gradients)
{
    if (!h || !gradients) return NHF_EINVAL;
    if (h->m.hang_cells <= 0) return NHF_OK;
    int rc = enter(h); if (rc) return rc;
    CK(h, cudaMemcpyAsync(gradients, h->dev.gradients, sizeof(real) * 2 * (size_t)h->m.hang_cells,
                          cudaMemcpyDeviceToDevice, h->s));
    return leave(h);
}

void *nhf_stream(nhf_handle *h) { return h ? (void *)h->s : nullptr; }

const char *nhf_path(const nhf_handle *h) { return h ? h->path.c_str() : ""; }

int nhf_synchronize(nhf_handle *h)
{
    if (!h) return NHF_EINVAL;
    CK(h, cudaStreamSynchronize(h->s));
    CK(h, cudaStreamSynchronize(h->user));
    return NHF_OK;
}

}  // extern "C"
