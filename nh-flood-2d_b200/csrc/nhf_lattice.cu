// Lattice form of the fused step, for meshes that are uniform grids.
//
// A uniform NE/NS mesh (one cell size, one side length per orientation,
// one side per face) is a 2-D lattice whatever its numbering. The planner
// below recognises it from the mesh tables and numbers it into a padded
// lattice: a 2-cell border of holes and padding up to whole 32 x 16 tiles.
// During a batch the library keeps its own lattice-ordered copies of the
// state (depth and side discharges double-buffered, rain time, infiltration,
// extrema), gathered from the caller's arrays at the batch start and
// scattered back at its end. Inside the batch every neighbour is found by
// arithmetic: no index tables, rows of 32 cells per warp, coalesced loads.
//
// One step is two launches. k_lattice_step: a block owns a 32 x 16 tile and
// stages depth and bed of the tile and two rings of neighbours, then, as
// the reference's passes do (solver_compact.py:439-613):
//   momentum q* of the sides the donor factors need (rings <= 1),
//   donor factors of rings <= 1,
//   the final discharge of the tile's faces,
//   sources and depth update of the tile's cells, extrema, budget terms.
// k_lattice_cfl: the canonical 256-cell budget trees of the blocks the step
// touched, then compute_cfl (617-641) over the interior sides, and its last
// block commits the step and prepares the next one. Each quantity is
// computed in the reference's operation order with the same expressions as
// the tiled and multi-pass steps, so the three forms and the CPU
// restatement agree bit for bit.
//
// Budget terms are sums over the reference's 256-cell blocks of global ids
// (ei // 256), which a lattice tile does not follow: the step writes each
// nonzero per-cell term into a scratch array by global id and marks its
// block; the CFL pass reduces the marked blocks with the canonical tree and
// clears them.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "nhf_common.cuh"
#include "nhf_math.cuh"

namespace nhf {
namespace {

constexpr int kTX = 32, kTY = 16, kNT = kTX * kTY;  // tile of the step, one thread per cell
constexpr int kRX = kTX + 4, kRY = kTY + 4;         // staged region: the tile and two rings
constexpr int kVX = kRX - 1, kVY = kRY - 2;         // west faces of region x 1..35, rows 1..18
constexpr int kHX = kRX - 2, kHY = kRY - 1;         // south faces of region x 1..34, rows 1..19
constexpr int kDX = kRX - 2, kDY = kRY - 2;         // donor cells: region x 1..34, rows 1..18

// Momentum (solver_compact.py:439-486) of one side from the staged cells
// (a: lower, b: higher); the same expressions as the tiled step's P1.
__device__ __forceinline__ real lattice_momentum(const Dev &d, real dt, real za, real ha, real zb, real hb,
                                                 bool live_a, bool live_b, const real *q_in, const real *n_arr,
                                                 const int32_t *side_ids, size_t L, real sdc)
{
    real hl = za + ha, hr = zb + hb;
    real xwh = rmax(hl, hr) - rmax(rmax(za, zb), kDh);
    real new_q = RC(0);
    if (!(xwh < d.min_h)) {
        real xq = q_in[L];
        real n = n_arr[L];
        const bool exterior = live_a != live_b;
        real dx = exterior ? d.sdc[side_ids[L]] : sdc;
        real bf = exterior ? RC(0) : RC(1);
        real difference = hr - hl;
        real xdq = (d.neg_g * difference / dx) * rmax(xwh, RC(0)) * dt;
        real ratio = RC(0);
        if (xq != RC(0)) ratio = xq / pow_real(rmax(xwh, RC(0.00001)), d.seven_thirds);
        real xf = RC(1) + d.g * dt * (n * n) * fabs(ratio);
        real nb = RC(0) + RC(0);
        new_q = (d.sita * xq + d.half_rest * nb + xdq) / xf;
        new_q *= bf;
    }
    return new_q;
}

// kMinBlocks resident blocks per SM: 2 (64 registers, no spills) or 3 (40
// registers, 12 bytes of spills); LatticePlan.blocks_per_sm picks one.
template <int kMinBlocks>
__global__ void __launch_bounds__(kNT, kMinBlocks) k_lattice_step(const __grid_constant__ Dev d)
{
    __shared__ real sh_h[kRY][kRX], sh_z[kRY][kRX];
    __shared__ real sh_qv[kVY][kVX], sh_qh[kHY][kHX];  // q*, then the final discharge
    __shared__ real sh_s[kDY][kDX];                    // donor factors
    __shared__ uint8_t sh_live[kRY][kRX];
    __shared__ uint32_t sh_cnt[3], sh_minbits;
    const LatticePlan &P = d.lat;
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    if (!c->active) return;
    const int tid = threadIdx.x;
    if (tid == 0) { sh_cnt[0] = sh_cnt[1] = sh_cnt[2] = 0u; sh_minbits = __float_as_uint(1.0f); }
    const int parity = c->parity;
    const real dt = c->dt;
    const int raining = c->raining;
    const real *h_in = P.h[parity];
    real *h_out = P.h[parity ^ 1];
    const real *qv_in = P.qv[parity], *qh_in = P.qh[parity];
    real *qv_out = P.qv[parity ^ 1], *qh_out = P.qh[parity ^ 1];
    const int lx = P.lx;
    // memory index of region cell (rx, ry): (y0 + ry) * lx + (x0 + rx)
    const size_t base = (size_t)blockIdx.y * kTY * lx + (size_t)blockIdx.x * kTX;

    for (int i = tid; i < kRX * kRY; i += kNT) {
        const int rx = i % kRX, ry = i / kRX;
        const size_t L = base + (size_t)ry * lx + rx;
        sh_h[ry][rx] = h_in[L];
        sh_z[ry][rx] = P.z[L];
        sh_live[ry][rx] = P.live[L];
    }
    __syncthreads();

    // momentum of the west faces (region x 1..35) and south faces (x 1..34) of rows 1..18 / 1..19
    for (int i = tid; i < kVX * kVY + kHX * kHY; i += kNT) {
        if (i < kVX * kVY) {
            const int rx = i % kVX + 1, ry = i / kVX + 1;
            const bool la = sh_live[ry][rx - 1], lb = sh_live[ry][rx];
            real q = RC(0);
            if (la || lb)
                q = lattice_momentum(d, dt, sh_z[ry][rx - 1], sh_h[ry][rx - 1], sh_z[ry][rx], sh_h[ry][rx], la, lb,
                                     qv_in, P.nv, P.side_v, base + (size_t)ry * lx + rx, P.sdc_v);
            sh_qv[ry - 1][rx - 1] = q;
        } else {
            const int k = i - kVX * kVY;
            const int rx = k % kHX + 1, ry = k / kHX + 1;
            const bool la = sh_live[ry - 1][rx], lb = sh_live[ry][rx];
            real q = RC(0);
            if (la || lb)
                q = lattice_momentum(d, dt, sh_z[ry - 1][rx], sh_h[ry - 1][rx], sh_z[ry][rx], sh_h[ry][rx], la, lb,
                                     qh_in, P.nh, P.side_h, base + (size_t)ry * lx + rx, P.sdc_h);
            sh_qh[ry - 1][rx - 1] = q;
        }
    }
    __syncthreads();

    // donor factors (solver_compact.py:491-514) of rings <= 1: region x 1..34, rows 1..18
    {
        uint32_t my_limited = 0, my_min = __float_as_uint(1.0f);
        for (int i = tid; i < kDX * kDY; i += kNT) {
            const int rx = i % kDX + 1, ry = i / kDX + 1;
            real sc = RC(0);  // holes: the sentinel's donor factor
            if (sh_live[ry][rx]) {
                const size_t L = base + (size_t)ry * lx + rx;
                const int bi = P.bi[L];
                int kind = -1;
                real discharge = RC(0);
                if (bi >= 0) {
                    kind = m.kind[bi];
                    if (kind == 1) discharge = d.values[bi] * m.weight[P.cell[L]];
                }
                const real rainq = raining ? d.rain_rates[P.rain_cells ? P.rain[L] : 0] : RC(0);
                real pipe = RC(0);
                real positive = (rmax(pipe, RC(0)) + rmax(discharge, RC(0))) * dt;
                real area = P.area;
                real available = sh_h[ry][rx] * area + positive + rainq * dt * area;
                real outgoing = (rmax(-pipe, RC(0)) + rmax(-discharge, RC(0))) * dt;
                const real face[4] = {sh_qv[ry - 1][rx - 1] * P.len_v, sh_qv[ry - 1][rx] * P.len_v,
                                      sh_qh[ry - 1][rx - 1] * P.len_h, sh_qh[ry][rx - 1] * P.len_h};
#pragma unroll
                for (int dd = 0; dd < 4; ++dd) {
                    real signed_q = face[dd];
                    if (dd == 0 || dd == 2) signed_q = -signed_q;
                    outgoing += rmax(signed_q, RC(0)) * dt;
                }
                sc = RC(1);
                if (outgoing > available && kind != 0) {
                    sc = available / outgoing;
                    if (rx >= 2 && rx < 2 + kTX && ry >= 2 && ry < 2 + kTY) {
                        my_limited += 1;
                        uint32_t bits = __float_as_uint(sc);
                        my_min = bits < my_min ? bits : my_min;
                    }
                }
            }
            sh_s[ry - 1][rx - 1] = sc;
        }
        if (my_limited) {
            atomicAdd(&sh_cnt[0], my_limited);
            atomicMin(&sh_minbits, my_min);
        }
    }
    __syncthreads();

    // final discharge (solver_compact.py:516-522) of the faces of the tile's
    // cells: west faces x 2..34 of rows 2..17, south faces x 2..33 of rows 2..18
    {
        uint32_t my_faces = 0;
        constexpr int nv = (kTX + 1) * kTY, nh = kTX * (kTY + 1);
        for (int i = tid; i < nv + nh; i += kNT) {
            if (i < nv) {
                const int rx = i % (kTX + 1) + 2, ry = i / (kTX + 1) + 2;
                const real q = sh_qv[ry - 1][rx - 1];
                const real sc = q >= RC(0) ? sh_s[ry - 1][rx - 2] : sh_s[ry - 1][rx - 1];
                if (rx < 2 + kTX && q != RC(0) && sc < RC(1)) my_faces += 1;
                sh_qv[ry - 1][rx - 1] = q * sc;
            } else {
                const int k = i - nv;
                const int rx = k % kTX + 2, ry = k / kTX + 2;
                const real q = sh_qh[ry - 1][rx - 1];
                const real sc = q >= RC(0) ? sh_s[ry - 2][rx - 1] : sh_s[ry - 1][rx - 1];
                if (ry < 2 + kTY && q != RC(0) && sc < RC(1)) my_faces += 1;
                sh_qh[ry - 1][rx - 1] = q * sc;
            }
        }
        if (my_faces) atomicAdd(&sh_cnt[1], my_faces);
    }
    __syncthreads();

    // sources and depth update (solver_compact.py:525-610) of this thread's cell
    const int rx = tid % kTX + 2, ry = tid / kTX + 2;
    const size_t L = base + (size_t)ry * lx + rx;
    uint32_t wet = 0;
    if (sh_live[ry][rx]) {
        const int g = P.cell[L];
        const int B = m.b_num;
        const int bi = P.bi[L];
        const int kind = bi >= 0 ? m.kind[bi] : -1;
        const real sc = sh_s[ry - 1][rx - 1];
        real pq = RC(0);
        real pipe = rmax(pq, RC(0)) + rmin(pq, RC(0)) * sc;
        real discharge = RC(0), t_discharge = RC(0);
        if (kind == 1) {
            real requested = d.values[bi] * m.weight[g];
            discharge = rmax(requested, RC(0)) + rmin(requested, RC(0)) * sc;
            t_discharge = discharge * dt;
        }
        real ssq = pipe + discharge;
        const real rainq = raining ? d.rain_rates[P.rain_cells ? P.rain[L] : 0] : RC(0);
        real infil;
        if (rainq > RC(0)) {
            real rt = P.rain_time[L] + dt;
            P.rain_time[L] = rt;
            // without Horton classes every f0, fc and k is zero (checked by the planner)
            real f0 = P.horton ? P.f0[L] : RC(0), fc = P.horton ? P.fc[L] : RC(0);
            real diff = f0 - fc;
            const real old = P.infil[L];
            infil = diff == RC(0) ? fc + RC(0) : fc + diff * exp_real(-(P.horton ? P.k[L] : RC(0)) * rt / RC(3600.0));
            if (__float_as_uint(infil) != __float_as_uint(old)) P.infil[L] = infil;
        } else {
            infil = P.infil[L];
        }
        real ql = RC(0) + sh_qv[ry - 1][rx - 1] * P.len_v, qr = RC(0) + sh_qv[ry - 1][rx] * P.len_v;
        real qb = RC(0) + sh_qh[ry - 1][rx - 1] * P.len_h, qt = RC(0) + sh_qh[ry][rx - 1] * P.len_h;
        real tq = ql - qr + qb - qt + ssq;
        real ea = P.area;
        real rain_depth = rainq * dt;
        real flux = tq * dt;
        real increment = (flux == RC(0) ? flux : flux / ea) + rain_depth;
        real previous = sh_h[ry][rx];
        real raw_depth = previous + increment;
        real removed = rmin(infil * dt, rmax(raw_depth, RC(0)));
        raw_depth -= removed;
        real floor_v = rmax(-raw_depth, RC(0));
        real level[5] = {RC(0), RC(0), RC(0), RC(0), RC(0)};
        real depth;
        if (kind == 0) {
            real target = rmax(d.level_values[bi] - sh_z[ry][rx], RC(0));
            level[0] = (target - previous) * ea;
            level[1] = -(ql - qr + qb - qt) * dt;
            level[2] = -pipe * dt;
            level[3] = -rain_depth * ea;
            level[4] = removed * ea;
            depth = target;
        } else {
            depth = rmax(raw_depth, RC(0));
        }
        h_out[L] = depth;
        real h = rmax(depth, RC(0.01));
        real u = RC(0), v = RC(0);
        if (depth >= d.min_h) {
            u = (ql + qr) / P.height / h * RC(0.5);
            v = (qb + qt) / P.width / h * RC(0.5);
        }
        real s2 = u * u + v * v;
        real speed = s2 == RC(0) ? RC(0) : sqrt(s2);
        if (speed > P.max_speed[L]) P.max_speed[L] = speed;
        if (depth > P.max_depth[L]) {
            P.max_depth[L] = depth;
            P.peak_hi[L] = c->step_end[0];
            P.peak_lo[L] = c->step_end[1];
        }
        wet = depth >= d.min_h ? 1u : 0u;
        // budget terms of this cell by global id: 0 removed, 1 / 2 bed clamp
        // off / on level cells, 3 pipe (none), 4 + 5 b + k level, 4 + 5 B + b discharge
        uint32_t mask = 0;
        float *terms = P.terms;
        const size_t e = (size_t)m.e_num;
        const real removed_v = removed * ea, floor_a = floor_v * ea;
        if (removed_v != RC(0)) { terms[0 * e + g] = removed_v; mask |= 1u; }
        if (floor_a != RC(0)) {
            const int t = kind == 0 ? 2 : 1;
            terms[t * e + g] = floor_a;
            mask |= 1u << t;
        }
        if (kind == 0)
            for (int q5 = 0; q5 < 5; ++q5)
                if (level[q5] != RC(0)) {
                    const int t = 4 + 5 * bi + q5;
                    terms[t * e + g] = level[q5];
                    mask |= 1u << t;
                }
        if (kind == 1 && t_discharge != RC(0)) {
            const int t = 4 + 5 * B + bi;
            terms[t * e + g] = t_discharge;
            mask |= 1u << t;
        }
        if (mask) atomicOr(&P.touched[g >> 8], mask);
    }
    // the tile's own faces: west and south of each cell
    if (sh_live[ry][rx - 1] || sh_live[ry][rx]) qv_out[L] = sh_qv[ry - 1][rx - 1];
    if (sh_live[ry - 1][rx] || sh_live[ry][rx]) qh_out[L] = sh_qh[ry - 1][rx - 1];
    const unsigned wet_warp = __popc(__ballot_sync(0xffffffffu, wet));
    if ((tid & 31) == 0 && wet_warp) atomicAdd(&sh_cnt[2], wet_warp);
    __syncthreads();
    if (tid == 0) {
        if (sh_cnt[0]) {
            atomicAdd(&c->limited_cells, sh_cnt[0]);
            atomicMin(&c->min_scale_bits, sh_minbits);
        }
        if (sh_cnt[1]) atomicAdd(&c->limited_faces, sh_cnt[1]);
        if (sh_cnt[2]) atomicAdd(&c->wet, sh_cnt[2]);
    }
}

// prepare_step (solver_compact.py:364-382) with the state in lattice order.
__device__ void lattice_prepare(const Dev &d, Ctl *c)
{
    const nhf_mesh &m = d.m;
    const LatticePlan &P = d.lat;
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
        const int si = c->cfl_arg;
        const int el = m.topology[3 * si + 1], eh = m.topology[3 * si + 2];
        const real *h = P.h[c->parity];
        const real de = el ? __ldcg(h + P.glat[el]) : m.depth[0];
        const real dh = eh ? __ldcg(h + P.glat[eh]) : m.depth[0];
        real fd = RC(0), q = m.q[0];
        if (si) {
            fd = cfl_face_depth(m.bed[el], de, m.bed[eh], dh);
            const int gs = P.gside[si];
            q = __ldcg(((gs & 1) ? P.qh[c->parity] : P.qv[c->parity]) + (gs >> 1));
        }
        c->limit_value[0] = c->ndt;
        c->limit_value[1] = de; c->limit_value[2] = dh;
        c->limit_value[3] = fd;
        c->limit_value[4] = q / rmax(fd, RC(1e-30));
        c->limit_ids[0] = si; c->limit_ids[1] = el; c->limit_ids[2] = eh;
    }
}

// Budget blocks the step touched (the canonical 256-cell tree), then the CFL
// candidate of the new state over the interior sides; the last block commits
// the step and prepares the next.
__global__ void __launch_bounds__(256) k_lattice_cfl(const __grid_constant__ Dev d)
{
    __shared__ double sh_tree[256];
    __shared__ unsigned long long sh_min[8];
    __shared__ bool last;
    const LatticePlan &P = d.lat;
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    const int active = c->active;
    const int tid = threadIdx.x;
    if (active) {
        const size_t e = (size_t)m.e_num;
        const int T = d.terms;
        for (int b = blockIdx.x; b < d.blocks; b += gridDim.x) {
            const uint32_t mask = P.touched[b];
            if (!mask) continue;
            const int g = b * 256 + tid;
            for (uint32_t rest = mask; rest; rest &= rest - 1) {
                const int t = __ffs(rest) - 1;
                float v = 0.0f;
                if (g < m.e_num) {
                    v = P.terms[t * e + g];
                    if (v != 0.0f) P.terms[t * e + g] = 0.0f;
                }
                const double sum = block_tree((double)v, sh_tree);
                if (tid == 0) acc_add(d.acc_sum + (size_t)b * T + t, d.acc_comp + (size_t)b * T + t, sum);
            }
            if (tid == 0) P.touched[b] = 0u;
        }
    }
    unsigned long long best = kCflEmpty;
    if (active) {
        const int p = c->parity ^ 1;  // the state the step just wrote
        const real *h = P.h[p], *qv = P.qv[p], *qh = P.qh[p];
        const int nx = P.nx, ny = P.ny, lx = P.lx;
        const long long n = (long long)(nx + 1) * (ny + 1);
        for (long long idx = (long long)blockIdx.x * 256 + tid; idx < n; idx += (long long)gridDim.x * 256) {
            const int x = (int)(idx % (nx + 1)), y = (int)(idx / (nx + 1));
            const size_t L = (size_t)(y + 2) * lx + (x + 2);
            const bool here = P.live[L];
            if (!here) continue;
            if (P.live[L - 1]) {  // west side
                const real fd = cfl_face_depth(P.z[L - 1], h[L - 1], P.z[L], h[L]);
                const real cfl = cfl_value(d.afa, d.g, P.len_v, qv[L], fd);
                const uint32_t bits = __float_as_uint(cfl);
                if (bits <= (uint32_t)(best >> 32)) {
                    const unsigned long long key = ((unsigned long long)bits << 32) | (unsigned)P.side_v[L];
                    best = key < best ? key : best;
                }
            }
            if (P.live[L - lx]) {  // south side
                const real fd = cfl_face_depth(P.z[L - lx], h[L - lx], P.z[L], h[L]);
                const real cfl = cfl_value(d.afa, d.g, P.len_h, qh[L], fd);
                const uint32_t bits = __float_as_uint(cfl);
                if (bits <= (uint32_t)(best >> 32)) {
                    const unsigned long long key = ((unsigned long long)bits << 32) | (unsigned)P.side_h[L];
                    best = key < best ? key : best;
                }
            }
        }
    }
    best = warp_min_u64(best);
    if ((tid & 31) == 0) sh_min[tid >> 5] = best;
    __syncthreads();
    if (tid == 0) {
        unsigned long long bmin = kCflEmpty;
        for (int w = 0; w < 8; ++w) bmin = sh_min[w] < bmin ? sh_min[w] : bmin;
        if (bmin != kCflEmpty) atomicMin(&c->cfl_packed, bmin);
        __threadfence();
        const unsigned ticket = atomicAdd(&c->done_blocks, 1u);
        last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (!last || tid != 0) return;
    __threadfence();
    const unsigned long long packed = atomicExch(&c->cfl_packed, kCflEmpty);
    c->done_blocks = 0;
    if (active) {
        if (packed == kCflEmpty) {
            c->ndt = __uint_as_float(0x7f800000u);
            c->cfl_arg = 0;
        } else {
            c->ndt = __uint_as_float((uint32_t)(packed >> 32));
            c->cfl_arg = (int32_t)(packed & 0xffffffffu);
        }
        c->parity ^= 1;
    }
    finish_step(c);
    if (c->slot < d.batch_size) lattice_prepare(d, c);
}

// Static lattice arrays from the caller's mesh (once).
__global__ void k_lattice_setup(const __grid_constant__ Dev d)
{
    const LatticePlan &P = d.lat;
    const nhf_mesh &m = d.m;
    const size_t n = (size_t)P.lx * P.ly;
    for (size_t L = (size_t)blockIdx.x * blockDim.x + threadIdx.x; L < n; L += (size_t)gridDim.x * blockDim.x) {
        const int g = P.cell[L];
        P.bi[L] = (int16_t)(g ? m.boundary_id[g] : -1);
        if (P.rain_cells) P.rain[L] = g ? m.rain_index[g] : 0;
        if (P.horton) {
            P.f0[L] = g ? m.f0[g] : RC(0);
            P.fc[L] = g ? m.fc[g] : RC(0);
            P.k[L] = g ? m.k[g] : RC(0);
        }
        const int sv = P.side_v[L], sh = P.side_h[L];
        P.nv[L] = sv ? m.side_n[sv] : RC(0);
        P.nh[L] = sh ? m.side_n[sh] : RC(0);
    }
}

// Batch start: the caller's state into lattice order (buffer 0).
__global__ void k_lattice_gather(const __grid_constant__ Dev d)
{
    const LatticePlan &P = d.lat;
    const nhf_mesh &m = d.m;
    const size_t n = (size_t)P.lx * P.ly;
    for (size_t L = (size_t)blockIdx.x * blockDim.x + threadIdx.x; L < n; L += (size_t)gridDim.x * blockDim.x) {
        const int g = P.cell[L];
        P.h[0][L] = m.depth[g];  // holes and the border hold the sentinel's values
        if (!g) P.h[1][L] = m.depth[0];
        P.z[L] = m.bed[g];
        if (g) {
            P.rain_time[L] = m.rain_time[g];
            P.infil[L] = m.infiltration[g];
            P.max_depth[L] = m.max_depth[g];
            P.max_speed[L] = m.max_speed[g];
            P.peak_hi[L] = m.peak_hi[g];
            P.peak_lo[L] = m.peak_lo[g];
        }
        const int sv = P.side_v[L], sh = P.side_h[L];
        P.qv[0][L] = sv ? m.q[sv] : RC(0);
        P.qh[0][L] = sh ? m.q[sh] : RC(0);
    }
}

// Batch end: the lattice state back into the caller's arrays.
__global__ void k_lattice_scatter(const __grid_constant__ Dev d)
{
    __shared__ bool last;
    const LatticePlan &P = d.lat;
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    const int p = c->parity;
    const size_t n = (size_t)P.lx * P.ly;
    for (size_t L = (size_t)blockIdx.x * blockDim.x + threadIdx.x; L < n; L += (size_t)gridDim.x * blockDim.x) {
        const int g = P.cell[L];
        if (g) {
            m.depth[g] = P.h[p][L];
            m.rain_time[g] = P.rain_time[L];
            m.infiltration[g] = P.infil[L];
            m.max_depth[g] = P.max_depth[L];
            m.max_speed[g] = P.max_speed[L];
            m.peak_hi[g] = P.peak_hi[L];
            m.peak_lo[g] = P.peak_lo[L];
        }
        const int sv = P.side_v[L], sh = P.side_h[L];
        if (sv) m.q[sv] = P.qv[p][L];
        if (sh) m.q[sh] = P.qh[p][L];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned ticket = atomicAdd(&c->done_blocks, 1u);
        last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        c->done_blocks = 0;
        c->parity = 0;
    }
}

int stream_grid(size_t n)
{
    size_t g = (n + 255) / 256;
    return (int)std::min<size_t>(std::max<size_t>(g, 1), 148 * 16);
}

}  // namespace

// ------------------------------------------------------------------ planner

int lattice_build(const Dev &d, cudaStream_t st, LatticeBuild *out, char *why, size_t why_len)
{
    const nhf_mesh &m = d.m;
    auto no = [&](const char *msg) { snprintf(why, why_len, "%s", msg); return 1; };
    const int e = m.e_num, s = m.s_num;
    if (e < 1 + 1024) return no("fewer than 1024 cells");
    if (!d.theta_one) return no("theta < 1");
    if (m.hang_cells > 0) return no("hanging edges");
    if (d.terms > 32) return no("more than four boundaries");
    if (m.isl_len != 4 * (e - 1)) return no("not one side per face");
    std::vector<float> x(e), y(e), w(e), hg(e), area(e), len(s);
    std::vector<int32_t> topo((size_t)s * 3), fptr((size_t)e * 4), fcnt((size_t)e * 4), isl(m.isl_len);
    if (cudaMemcpyAsync(x.data(), m.x, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(y.data(), m.y, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(w.data(), m.width, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(hg.data(), m.height, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(area.data(), m.area, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(len.data(), m.length, 4 * (size_t)s, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(topo.data(), m.topology, 12 * (size_t)s, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(fptr.data(), m.face_ptr, 16 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(fcnt.data(), m.face_count, 16 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(isl.data(), m.isl_data, 4 * (size_t)m.isl_len, cudaMemcpyDeviceToHost, st) ||
        cudaStreamSynchronize(st))
        return no("copy of the mesh tables failed");
    const float W = w[1], H = hg[1], A = area[1];
    float x0 = x[1], y0 = y[1];
    for (int c = 1; c < e; ++c) {
        if (w[c] != W || hg[c] != H || area[c] != A) return no("cell sizes differ");
        x0 = std::min(x0, x[c]);
        y0 = std::min(y0, y[c]);
        for (int dd = 0; dd < 4; ++dd)
            if (fcnt[4 * c + dd] != 1) return no("a face without exactly one side");
    }
    if (!(W > 0.0f) || !(H > 0.0f)) return no("empty cells");
    std::vector<int32_t> ci(e), cj(e);
    int nx = 0, ny = 0;
    for (int c = 1; c < e; ++c) {
        const double fi = ((double)x[c] - x0) / W, fj = ((double)y[c] - y0) / H;
        const long long i = llround(fi), j = llround(fj);
        if (std::fabs(fi - i) > 1e-3 || std::fabs(fj - j) > 1e-3 || i > (1 << 20) || j > (1 << 20))
            return no("cell centres off a lattice");
        ci[c] = (int)i; cj[c] = (int)j;
        nx = std::max(nx, (int)i + 1);
        ny = std::max(ny, (int)j + 1);
    }
    if ((double)nx * ny > 1.5 * (e - 1)) return no("lattice mostly empty");
    LatticePlan P{};
    P.nx = nx; P.ny = ny;
    P.tiles_x = (nx + 1 + kTX - 1) / kTX;  // the tiles cover columns 0..nx and rows 0..ny
    P.tiles_y = (ny + 1 + kTY - 1) / kTY;
    P.lx = P.tiles_x * kTX + 4;
    P.ly = P.tiles_y * kTY + 4;
    const size_t nl = (size_t)P.lx * P.ly;
    if (nl >= ((size_t)1 << 30)) return no("lattice too large");
    auto at = [&](int i, int j) { return (size_t)(j + 2) * P.lx + (i + 2); };
    std::vector<int32_t> cell(nl, 0), side_v(nl, 0), side_h(nl, 0), glat(e, 0), gside(s, 0);
    std::vector<uint8_t> live(nl, 0);
    for (int c = 1; c < e; ++c) {
        const size_t L = at(ci[c], cj[c]);
        if (cell[L]) return no("two cells at one lattice point");
        cell[L] = c; live[L] = 1; glat[c] = (int32_t)L;
    }
    auto cell_at = [&](int i, int j) -> int {
        if (i < 0 || j < 0 || i >= nx || j >= ny) return 0;
        return cell[at(i, j)];
    };
    // every face's side joins the lattice neighbours (west/east: orientation
    // 2, lower = west; south/north: orientation 1, lower = south)
    bool have_v = false, have_h = false;
    float sdc_v = 0.0f, sdc_h = 0.0f, len_v = 0.0f, len_h = 0.0f;
    std::vector<int> seen(s, 0);
    for (int c = 1; c < e; ++c) {
        const int i = ci[c], j = cj[c];
        const int nb[4] = {cell_at(i - 1, j), cell_at(i + 1, j), cell_at(i, j - 1), cell_at(i, j + 1)};
        for (int dd = 0; dd < 4; ++dd) {
            const int p = fptr[4 * c + dd];
            if (p < 0 || p >= m.isl_len) return no("a face pointer outside the side list");
            const int sid = isl[p];
            if (sid < 1 || sid >= s) return no("a face lists an invalid side");
            const int so = topo[3 * sid], lo = topo[3 * sid + 1], hi = topo[3 * sid + 2];
            const bool vertical = dd < 2;
            const int want_lo = (dd == 0 || dd == 2) ? nb[dd] : c, want_hi = (dd == 0 || dd == 2) ? c : nb[dd];
            if (so != (vertical ? 2 : 1) || lo != want_lo || hi != want_hi) return no("sides off the lattice");
            // the lattice side is the west / south face of its higher cell
            // (or of the lattice point east / north of its lower cell)
            const size_t L = (dd == 0 || dd == 2) ? at(i, j) : (dd == 1 ? at(i + 1, j) : at(i, j + 1));
            std::vector<int32_t> &map = vertical ? side_v : side_h;
            if (map[L] && map[L] != sid) return no("two sides at one lattice face");
            map[L] = sid;
            gside[sid] = (int32_t)((L << 1) | (vertical ? 0u : 1u));
            seen[sid] = 1;
            const float l = len[sid];
            if (vertical) {
                if (have_v && l != len_v) return no("side lengths differ");
                len_v = l;
            } else {
                if (have_h && l != len_h) return no("side lengths differ");
                len_h = l;
            }
            if (lo && hi) {  // interior: centre distance as k_initialize computes it
                const float dist = vertical ? std::max(std::fabs(x[hi] - x[lo]), 0.01f)
                                           : std::max(std::fabs(y[hi] - y[lo]), 0.01f);
                float &ref = vertical ? sdc_v : sdc_h;
                bool &have = vertical ? have_v : have_h;
                if (have && dist != ref) return no("centre distances differ");
                ref = dist;
                have = true;
            }
        }
    }
    for (int sid = 1; sid < s; ++sid)
        if (!seen[sid]) return no("a side no face lists");
    if (!have_v || !have_h) return no("no interior side in one direction");
    P.sdc_v = sdc_v; P.sdc_h = sdc_h; P.len_v = len_v; P.len_h = len_h;
    P.area = A; P.width = W; P.height = H;
    // rain pixels and Horton parameters per lattice cell only when they vary
    std::vector<int32_t> rain(e);
    std::vector<float> f0(e), fc(e), kk(e);
    if (cudaMemcpyAsync(rain.data(), m.rain_index, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(f0.data(), m.f0, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(fc.data(), m.fc, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(kk.data(), m.k, 4 * (size_t)e, cudaMemcpyDeviceToHost, st) || cudaStreamSynchronize(st))
        return no("copy of the cell parameters failed");
    P.rain_cells = 0;
    P.horton = 0;
    // resident blocks per SM of the step kernel (a tuning knob, default 2)
    const char *occ = getenv("NHF_LATTICE_BLOCKS");
    P.blocks_per_sm = (occ && atoi(occ) == 3) ? 3 : 2;
    for (int c = 1; c < e; ++c) {
        if (rain[c] != 0) P.rain_cells = 1;
        if (f0[c] != 0.0f || fc[c] != 0.0f || kk[c] != 0.0f) P.horton = 1;
    }
    // device memory: maps, state copies, static arrays, budget scratch
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    const size_t o_cell = take(4 * nl), o_sv = take(4 * nl), o_sh = take(4 * nl), o_live = take(nl);
    const size_t o_glat = take(4 * (size_t)e), o_gside = take(4 * (size_t)s);
    size_t o_h[2], o_qv[2], o_qh[2];
    for (int k = 0; k < 2; ++k) { o_h[k] = take(4 * nl); o_qv[k] = take(4 * nl); o_qh[k] = take(4 * nl); }
    const size_t o_z = take(4 * nl), o_nv = take(4 * nl), o_nh = take(4 * nl), o_bi = take(2 * nl);
    const size_t o_rain = P.rain_cells ? take(4 * nl) : 0;
    const size_t o_rt = take(4 * nl), o_inf = take(4 * nl), o_md = take(4 * nl), o_ms = take(4 * nl);
    const size_t o_ph = take(4 * nl), o_pl = take(4 * nl);
    size_t o_f0 = 0, o_fc = 0, o_k = 0;
    if (P.horton) { o_f0 = take(4 * nl); o_fc = take(4 * nl); o_k = take(4 * nl); }
    const size_t o_terms = take(4 * (size_t)d.terms * e), o_touch = take(4 * (size_t)d.blocks);
    char *mem = nullptr;
    if (cudaMalloc((void **)&mem, off)) { cudaGetLastError(); return no("no device memory for the lattice"); }
    out->device_memory = mem;
    if (cudaMemsetAsync(mem, 0, off, st) ||
        cudaMemcpyAsync(mem + o_cell, cell.data(), 4 * nl, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(mem + o_sv, side_v.data(), 4 * nl, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(mem + o_sh, side_h.data(), 4 * nl, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(mem + o_live, live.data(), nl, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(mem + o_glat, glat.data(), 4 * (size_t)e, cudaMemcpyHostToDevice, st) ||
        cudaMemcpyAsync(mem + o_gside, gside.data(), 4 * (size_t)s, cudaMemcpyHostToDevice, st) ||
        cudaStreamSynchronize(st))
        return no("upload of the lattice maps failed");
    P.cell = (const int32_t *)(mem + o_cell);
    P.side_v = (const int32_t *)(mem + o_sv);
    P.side_h = (const int32_t *)(mem + o_sh);
    P.live = (const uint8_t *)(mem + o_live);
    P.glat = (const int32_t *)(mem + o_glat);
    P.gside = (const int32_t *)(mem + o_gside);
    for (int k = 0; k < 2; ++k) {
        P.h[k] = (real *)(mem + o_h[k]);
        P.qv[k] = (real *)(mem + o_qv[k]);
        P.qh[k] = (real *)(mem + o_qh[k]);
    }
    P.z = (real *)(mem + o_z); P.nv = (real *)(mem + o_nv); P.nh = (real *)(mem + o_nh);
    P.bi = (int16_t *)(mem + o_bi);
    P.rain = P.rain_cells ? (int32_t *)(mem + o_rain) : nullptr;
    P.rain_time = (real *)(mem + o_rt); P.infil = (real *)(mem + o_inf);
    P.max_depth = (real *)(mem + o_md); P.max_speed = (real *)(mem + o_ms);
    P.peak_hi = (uint32_t *)(mem + o_ph); P.peak_lo = (uint32_t *)(mem + o_pl);
    if (P.horton) { P.f0 = (real *)(mem + o_f0); P.fc = (real *)(mem + o_fc); P.k = (real *)(mem + o_k); }
    P.terms = (float *)(mem + o_terms);
    P.touched = (uint32_t *)(mem + o_touch);
    Dev dd = d;
    dd.lat = P;
    k_lattice_setup<<<stream_grid(nl), 256, 0, st>>>(dd);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(st)) return no("lattice setup failed");
    out->plan = P;
    return 0;
}

void lattice_enqueue_batch_start(const Dev &d, cudaStream_t s)
{
    k_lattice_gather<<<stream_grid((size_t)d.lat.lx * d.lat.ly), 256, 0, s>>>(d);
}

void lattice_enqueue_step(const Dev &d, cudaStream_t s)
{
    if (d.lat.blocks_per_sm == 3) k_lattice_step<3><<<dim3(d.lat.tiles_x, d.lat.tiles_y), kNT, 0, s>>>(d);
    else k_lattice_step<2><<<dim3(d.lat.tiles_x, d.lat.tiles_y), kNT, 0, s>>>(d);
    int grid = std::max(1, std::min(148 * 8, (int)(((long long)(d.lat.nx + 1) * (d.lat.ny + 1) + 255) / 256)));
    k_lattice_cfl<<<grid, 256, 0, s>>>(d);
}

void lattice_enqueue_batch_end(const Dev &d, cudaStream_t s)
{
    k_lattice_scatter<<<stream_grid((size_t)d.lat.lx * d.lat.ly), 256, 0, s>>>(d);
    tiled_enqueue_velocity(d, s);
}

}  // namespace nhf
