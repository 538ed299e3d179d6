// Lattice form of the fused step, for meshes that are uniform grids.
//
// A uniform NE/NS mesh (one cell size, one side length per orientation,
// one side per face) is a 2-D lattice whatever its numbering. The planner
// below recognises it from the mesh tables and numbers it into a padded
// lattice: a border of holes (2 columns west, 2 rows south) and padding up
// to whole strips of 28 columns and chunks of rows (3 rows above the last
// chunk). During a batch the library keeps its own lattice-ordered copies
// of the state (depth and side discharges double-buffered, rain time,
// infiltration, extrema), gathered from the caller's arrays at the batch
// start and scattered back at its end. Inside the batch every neighbour is
// found by arithmetic: no index tables, rows of 32 cells per warp,
// coalesced loads.
//
// One step is two launches. k_lattice_march: each warp marches up a strip
// of the lattice with the rows it needs in registers and does, row by row,
// what the reference's passes do (solver_compact.py:439-641): momentum q*,
// donor factors, final discharges, sources and depth update, extrema,
// budget terms and the CFL candidates of the sides inside its strip and
// chunk; it writes its counters, its CFL minimum and its edge columns to
// per-warp records. k_lattice_close: those records, the CFL candidates of
// the sides on strip and chunk edges, the canonical 256-cell budget trees
// of the blocks the step touched, and in its last block the commit of the
// step and the prepare of the next. Each quantity is computed in the
// reference's operation order with the same expressions as the tiled and
// multi-pass steps, so the three forms and the CPU restatement agree bit
// for bit.
//
// Budget terms are sums over the reference's 256-cell blocks of global ids
// (ei // 256), which a lattice strip does not follow: the march writes each
// nonzero per-cell term into a scratch array by global id and marks its
// block; the close pass reduces the marked blocks with the canonical tree
// and clears them.
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

constexpr int kLanes = 32;                        // a warp marches a strip of 32 lattice columns
constexpr int kOut = 28;                          // and owns the 28 of lanes 2..29
constexpr int kWarps = 8, kNT = kLanes * kWarps;  // a block: up to 8 strips side by side
constexpr int kWest = 2;                          // border columns west of cell column 0

// Momentum (solver_compact.py:439-486) of one side from the cells either
// side of it (a: lower, b: higher) and the side's discharge xq and Manning
// n; the same expressions as the tiled step's P1.
__device__ __forceinline__ real lattice_momentum(const Dev &d, real dt, real za, real ha, real zb, real hb,
                                                 bool live_a, bool live_b, real xq, real n,
                                                 const int32_t *side_ids, size_t L, real sdc)
{
    real hl = za + ha, hr = zb + hb;
    real xwh = rmax(hl, hr) - rmax(rmax(za, zb), kDh);
    real new_q = RC(0);
    if (!(xwh < d.min_h)) {
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

// Donor factor (solver_compact.py:491-514) of the cell at lattice index L
// (boundary id bi) from its depth and the q* of its west, east, south and
// north faces; sets ``limited`` when the outflow had to be scaled.
__device__ __forceinline__ real lattice_donor(const Dev &d, const LatticePlan &P, size_t L, int bi, real h, real dt,
                                              int raining, real qw, real qe, real qs, real qn, bool &limited)
{
    const nhf_mesh &m = d.m;
    int kind = -1;
    real discharge = RC(0);
    if (bi >= 0) {
        kind = m.kind[bi];
        if (kind == 1) discharge = d.values[bi] * m.weight[__ldg(P.cell + L)];
    }
    const real rainq = raining ? d.rain_rates[P.rain_cells ? __ldg(P.rain + L) : 0] : RC(0);
    real pipe = RC(0);
    real positive = (rmax(pipe, RC(0)) + rmax(discharge, RC(0))) * dt;
    real area = P.area;
    real available = h * area + positive + rainq * dt * area;
    real outgoing = (rmax(-pipe, RC(0)) + rmax(-discharge, RC(0))) * dt;
    const real face[4] = {qw * P.len_v, qe * P.len_v, qs * P.len_h, qn * P.len_h};
#pragma unroll
    for (int dd = 0; dd < 4; ++dd) {
        real signed_q = face[dd];
        if (dd == 0 || dd == 2) signed_q = -signed_q;
        outgoing += rmax(signed_q, RC(0)) * dt;
    }
    real sc = RC(1);
    limited = false;
    if (outgoing > available && kind != 0) {
        sc = available / outgoing;
        limited = true;
    }
    return sc;
}

// The per-cell inputs of a depth update, loaded a row ahead of their use.
struct LatticeCell {
    int g, bi;
    real rain_time, infil, max_speed, max_depth;
};

// Sources and depth update (solver_compact.py:525-610) of the cell at
// lattice index L from its old depth, its donor factor and the final
// discharges of its four faces; writes the cell's rain time, infiltration,
// extrema and budget terms and returns the new depth.
__device__ __forceinline__ real lattice_update(const Dev &d, const LatticePlan &P, size_t L, real dt, int raining,
                                               real previous, real z, real sc, real fw, real fe, real fs, real fn,
                                               const LatticeCell &k, const uint32_t *step_end)
{
    const nhf_mesh &m = d.m;
    const int g = k.g, bi = k.bi;
    const int B = m.b_num;
    const int kind = bi >= 0 ? m.kind[bi] : -1;
    real pq = RC(0);
    real pipe = rmax(pq, RC(0)) + rmin(pq, RC(0)) * sc;
    real discharge = RC(0), t_discharge = RC(0);
    if (kind == 1) {
        real requested = d.values[bi] * m.weight[g];
        discharge = rmax(requested, RC(0)) + rmin(requested, RC(0)) * sc;
        t_discharge = discharge * dt;
    }
    real ssq = pipe + discharge;
    const real rainq = raining ? d.rain_rates[P.rain_cells ? __ldg(P.rain + L) : 0] : RC(0);
    real infil;
    if (rainq > RC(0)) {
        real rt = k.rain_time + dt;
        P.rain_time[L] = rt;
        // without Horton classes every f0, fc and k is zero (checked by the planner)
        real f0 = P.horton ? P.f0[L] : RC(0), fc = P.horton ? P.fc[L] : RC(0);
        real diff = f0 - fc;
        infil = diff == RC(0) ? fc + RC(0) : fc + diff * exp_real(-(P.horton ? P.k[L] : RC(0)) * rt / RC(3600.0));
        if (__float_as_uint(infil) != __float_as_uint(k.infil)) P.infil[L] = infil;
    } else {
        infil = k.infil;
    }
    real ql = RC(0) + fw * P.len_v, qr = RC(0) + fe * P.len_v;
    real qb = RC(0) + fs * P.len_h, qt = RC(0) + fn * P.len_h;
    real tq = ql - qr + qb - qt + ssq;
    real ea = P.area;
    real rain_depth = rainq * dt;
    real flux = tq * dt;
    real increment = (flux == RC(0) ? flux : flux / ea) + rain_depth;
    real raw_depth = previous + increment;
    real removed = rmin(infil * dt, rmax(raw_depth, RC(0)));
    raw_depth -= removed;
    real floor_v = rmax(-raw_depth, RC(0));
    real depth = kind == 0 ? rmax(d.level_values[bi] - z, RC(0)) : rmax(raw_depth, RC(0));
    real h = rmax(depth, RC(0.01));
    real u = RC(0), v = RC(0);
    if (depth >= d.min_h) {
        u = (ql + qr) / P.height / h * RC(0.5);
        v = (qb + qt) / P.width / h * RC(0.5);
    }
    real s2 = u * u + v * v;
    real speed = s2 == RC(0) ? RC(0) : sqrt(s2);
    if (speed > k.max_speed) P.max_speed[L] = speed;
    if (depth > k.max_depth) {
        P.max_depth[L] = depth;
        P.peak_hi[L] = __ldg(step_end);  // the clock words are not written during the march
        P.peak_lo[L] = __ldg(step_end + 1);
    }
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
    if (kind == 0) {
        const real level[5] = {(depth - previous) * ea, -(ql - qr + qb - qt) * dt, -pipe * dt, -rain_depth * ea,
                               removed * ea};
        for (int q5 = 0; q5 < 5; ++q5)
            if (level[q5] != RC(0)) {
                const int t = 4 + 5 * bi + q5;
                terms[t * e + g] = level[q5];
                mask |= 1u << t;
            }
    }
    if (kind == 1 && t_discharge != RC(0)) {
        const int t = 4 + 5 * B + bi;
        terms[t * e + g] = t_discharge;
        mask |= 1u << t;
    }
    if (mask) atomicOr(&P.touched[g >> 8], mask);
    return depth;
}

// CFL candidate (solver_compact.py:617-641) of one interior side, folded
// into the running minimum key (dt bits << 32 | side id); the side id is
// read only for a candidate at or below the minimum.
__device__ __forceinline__ void lattice_cfl(const Dev &d, real len, real q, real za, real ha, real zb, real hb,
                                            const int32_t *side_ids, size_t L, unsigned long long &best)
{
    const real fd = cfl_face_depth(za, ha, zb, hb);
    const uint32_t bits = __float_as_uint(cfl_value(d.afa, d.g, len, q, fd));
    if (bits <= (uint32_t)(best >> 32)) {
        const unsigned long long key = ((unsigned long long)bits << 32) | (unsigned)__ldg(side_ids + L);
        best = key < best ? key : best;
    }
}

// prepare_step (solver_compact.py:364-382) with the state in lattice order.
__device__ __noinline__ void lattice_prepare(const Dev &d, Ctl *c)
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
// One step of the lattice form (solver_compact.py:439-641) but the CFL of
// the sides on strip and chunk edges, which k_lattice_close takes.
//
// A warp owns a strip of 32 lattice columns and P.rows rows and marches up
// it one row per iteration, the rows it needs held in registers and the
// west/east neighbours taken by shuffles. Iteration y forms q* of the south
// faces of row y + 2 and the west faces of row y + 1 (439-486), the donor
// factors of row y + 1 (491-514), the final discharge of the south faces
// of row y + 1 and the west faces of row y (516-522), the update of row y
// (525-610) and the CFL candidates (617-641) of row y's west and south
// sides whose cells this warp updated; and it loads what iteration y + 1
// will need (row y + 3 and the side discharges and Manning n first, the
// update inputs of row y + 1 after the update), so the loads of a row are
// in flight while the row before it is computed. Lanes 2..29 own the
// strip's 28 columns; lanes 0, 1, 30 and 31 are the halo the donor factors
// need. The first three iterations, below the chunk's rows, only fill the
// registers. No shared memory and no block barrier: each warp writes its
// counters and CFL minimum for the close pass and leaves.
template <int kMinBlocks>
__global__ void __launch_bounds__(kNT, kMinBlocks) k_lattice_march(const __grid_constant__ Dev d)
{
    constexpr unsigned kAll = 0xffffffffu;
    const LatticePlan &P = d.lat;
    Ctl *c = d.ctl;
    if (!c->active) return;
    const int lane = threadIdx.x & 31, warps = blockDim.x >> 5;
    const int strip = blockIdx.x * warps + (threadIdx.x >> 5);
    if (strip >= P.strips) return;
    // limited cells, limited faces and wet cells of this lane, 10 bits each
    // (at most 2 x 256 rows), and the smallest donor factor's bits
    uint32_t counts = 0, min_bits = __float_as_uint(1.0f);
    unsigned long long best = kCflEmpty;
    {
        const real dt = c->dt;
        const int raining = c->raining;
        const int parity = c->parity;
        // the second buffer of depth, west and south discharge lies
        // P.buffer_stride elements after the first: one offset selects the
        // state a step reads (rd) and the one it writes (wr), the bases stay
        // kernel parameters
        const int rd = parity ? P.buffer_stride : 0, wr = P.buffer_stride - rd;
        const int lx = P.lx;  // lattice indices fit 30 bits (checked by the planner)
        const int x = strip * kOut + lane;  // lattice column of this lane
        const bool own = lane >= 2 && lane < 2 + kOut;
        const int y0 = 2 + blockIdx.y * P.rows, y1 = y0 + P.rows;  // the rows this warp updates
        // iteration y holds row y (h0 z0 l0), row y + 1 (h1 z1 l1), row y + 2
        // (h2 z2 l2), the inputs of the south side of row y + 2 (xs ns), of
        // the west side of row y + 1 (xw nw), the boundary id of row y + 1
        // (b1) and the update inputs of row y (k0); it loads row y + 3 and
        // the side inputs first, the update inputs of row y + 1 last
        int L1 = (y0 - 2) * lx + x;
        int L2 = L1 + lx;
        real h1 = __ldg(P.h[0] + rd + L1), z1 = __ldg(P.z + L1);
        bool l1 = __ldg(P.live + L1);
        real h2 = __ldg(P.h[0] + rd + L2), z2 = __ldg(P.z + L2);
        bool l2 = __ldg(P.live + L2);
        real xs = __ldg(P.qh[0] + rd + L2), ns = __ldg(P.nh + L2);
        real xw = __ldg(P.qv[0] + rd + L1), nw = __ldg(P.nv + L1);
        int b1 = __ldg(P.bi + L1);
        LatticeCell k0{0, -1, RC(0), RC(0), RC(0), RC(0)};
        real h0 = RC(0), z0 = RC(0), hm = RC(0), zm = RC(0);
        bool l0 = false, lm = false;
        real qs1 = RC(0), qw0 = RC(0), d0 = RC(0), fs0 = RC(0);  // q* south y+1, q* west y, donor y, final south y
        for (int y = y0 - 3; y < y1; ++y) {
            const int L0 = L1 - lx, L3 = L2 + lx;
            // what iteration y + 1 needs
            const real h3 = __ldg(P.h[0] + rd + L3), z3 = __ldg(P.z + L3);
            const bool l3 = __ldg(P.live + L3);
            const real xs3 = __ldg(P.qh[0] + rd + L3), ns3 = __ldg(P.nh + L3);
            const real xw2 = __ldg(P.qv[0] + rd + L2), nw2 = __ldg(P.nv + L2);
            const int b2 = __ldg(P.bi + L2);
            // q* of the south side of row y + 2 and of the west side of row y + 1
            real qs2 = RC(0);
            if (l1 || l2) qs2 = lattice_momentum(d, dt, z1, h1, z2, h2, l1, l2, xs, ns, P.side_h, L2, P.sdc_h);
            const real hw = __shfl_up_sync(kAll, h1, 1), zw = __shfl_up_sync(kAll, z1, 1);
            const bool lw = __shfl_up_sync(kAll, (int)l1, 1) != 0;
            real qw1 = RC(0);
            if (lane > 0 && (lw || l1)) qw1 = lattice_momentum(d, dt, zw, hw, z1, h1, lw, l1, xw, nw, P.side_v, L1, P.sdc_v);
            const real qe1 = __shfl_down_sync(kAll, qw1, 1);
            const bool out1 = own && y + 1 >= y0 && y + 1 < y1, out0 = own && y >= y0;
            // donor factor of row y + 1 (holes: the sentinel's factor 0)
            real d1 = RC(0);
            if (l1) {
                bool limited;
                d1 = lattice_donor(d, P, L1, b1, h1, dt, raining, qw1, qe1, qs1, qs2, limited);
                if (limited && out1) {
                    counts += 1u;
                    const uint32_t bits = __float_as_uint(d1);
                    min_bits = bits < min_bits ? bits : min_bits;
                }
            }
            // final discharge of the south side of row y + 1 and the west side of row y
            const real ss = qs1 >= RC(0) ? d0 : d1;
            const real fs1 = qs1 * ss;
            if (out1 && qs1 != RC(0) && ss < RC(1)) counts += 1u << 10;
            const real dwest = __shfl_up_sync(kAll, d0, 1);
            const real sw = qw0 >= RC(0) ? dwest : d0;
            const real fw0 = qw0 * sw;
            if (out0 && qw0 != RC(0) && sw < RC(1)) counts += 1u << 10;
            const real fe0 = __shfl_down_sync(kAll, fw0, 1);
            // update of row y
            real hn = h0;
            if (out0 && l0) {
                hn = lattice_update(d, P, L0, dt, raining, h0, z0, d0, fw0, fe0, fs0, fs1, k0, c->step_end);
                P.h[0][wr + L0] = hn;
                if (hn >= d.min_h) counts += 1u << 20;
            }
            const real hnw = __shfl_up_sync(kAll, hn, 1), zw0 = __shfl_up_sync(kAll, z0, 1);
            const bool lw0 = __shfl_up_sync(kAll, (int)l0, 1) != 0;
            if (out0) {
                if (l0 || lw0) P.qv[0][wr + L0] = fw0;
                if (l0 || lm) P.qh[0][wr + L0] = fs0;
                // the strip's edge cells for the close pass: the first column
                // (new depth, bed, discharge of its west side, liveness) and
                // the last (new depth, -1 for a hole, and bed)
                const size_t e_at = (size_t)strip * P.chunks * P.rows + (y - 2);
                if (lane == 2) P.edge_first[e_at] = make_float4(hn, z0, fw0, l0 ? 1.0f : 0.0f);
                if (lane == 1 + kOut) P.edge_last[e_at] = make_float2(l0 ? hn : -1.0f, z0);
                // interior sides both of whose cells this warp updated
                if (l0 && lw0 && lane > 2) lattice_cfl(d, P.len_v, fw0, zw0, hnw, z0, hn, P.side_v, L0, best);
                if (l0 && lm && y > y0) lattice_cfl(d, P.len_h, fs0, zm, hm, z0, hn, P.side_h, L0, best);
            }
            // the update inputs of row y + 1, half an iteration ahead of their use
            k0 = LatticeCell{0, b1, RC(0), RC(0), RC(0), RC(0)};
            if (own && l1 && y + 1 >= y0 && y + 1 < y1) {
                k0.g = __ldg(P.cell + L1);
                k0.rain_time = P.rain_time[L1];
                k0.infil = P.infil[L1];
                k0.max_speed = P.max_speed[L1];
                k0.max_depth = P.max_depth[L1];
            }
            hm = hn; zm = z0; lm = l0;
            h0 = h1; z0 = z1; l0 = l1;
            h1 = h2; z1 = z2; l1 = l2;
            h2 = h3; z2 = z3; l2 = l3;
            xs = xs3; ns = ns3; xw = xw2; nw = nw2;
            b1 = b2;
            qs1 = qs2; qw0 = qw1; d0 = d1; fs0 = fs1;
            L1 += lx; L2 += lx;
        }
    }
    // counters and the CFL candidate of the warp, for the close pass: no
    // block barrier, so a warp leaves as soon as its strip is done
    const uint32_t n_lim = __reduce_add_sync(kAll, counts & 1023u);
    const uint32_t n_faces = __reduce_add_sync(kAll, (counts >> 10) & 1023u);
    const uint32_t n_wet = __reduce_add_sync(kAll, counts >> 20);
    min_bits = __reduce_min_sync(kAll, min_bits);
    best = warp_min_u64(best);
    if (lane == 0) {
        const size_t w = (size_t)blockIdx.y * P.strips + strip, W = (size_t)P.strips * P.chunks;
        P.part[w] = n_lim;
        P.part[W + w] = n_faces;
        P.part[2 * W + w] = n_wet;
        P.part[3 * W + w] = min_bits;
        P.part_cfl[w] = best;
    }
}
// After the march: the budget blocks the step touched (the canonical
// 256-cell tree of each term a block holds, device_budget.py:28-84, added
// into the compensated partials; scratch and marks cleared), the CFL
// candidates (solver_compact.py:617-641) of the sides on strip and chunk
// edges, whose two cells two different warps updated, and in the last block
// to finish the commit of the step and the prepare of the next.
__global__ void __launch_bounds__(256, 6) k_lattice_close(const __grid_constant__ Dev d)
{
    __shared__ double sh_tree[256];
    __shared__ uint32_t sh_mask[256];
    __shared__ unsigned long long sh_min[8];
    __shared__ uint32_t sh_cnt[8][4];
    __shared__ bool last;
    const LatticePlan &P = d.lat;
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    const int tid = threadIdx.x;
    const size_t e = (size_t)m.e_num;
    const int T = d.terms;
    // an even share of the marks per block (at most 256 per round, one per
    // thread); the block then takes the marked budget blocks one by one
    const int per = min(256, (d.blocks + (int)gridDim.x - 1) / (int)gridDim.x);
    for (int base = blockIdx.x * per; base < d.blocks; base += gridDim.x * per) {
        const uint32_t mine = (tid < per && base + tid < d.blocks) ? P.touched[base + tid] : 0u;
        sh_mask[tid] = mine;
        if (!__syncthreads_or(mine != 0u)) continue;
        for (int j = 0; j < per; ++j) {
            const uint32_t mask = sh_mask[j];
            if (!mask) continue;
            const int b = base + j, g = b * 256 + tid;
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
        __syncthreads();  // sh_mask is rewritten next round
    }
    const int active = c->active;
    unsigned long long best = kCflEmpty;
    uint32_t lim = 0, faces = 0, wet = 0, mb = __float_as_uint(1.0f);
    if (active) {
        // the march's per-warp counters and CFL minima
        const int W = P.strips * P.chunks;
        for (int w = blockIdx.x * 256 + tid; w < W; w += gridDim.x * 256) {
            lim += P.part[w];
            faces += P.part[W + w];
            wet += P.part[2 * W + w];
            mb = P.part[3 * W + w] < mb ? P.part[3 * W + w] : mb;
            best = P.part_cfl[w] < best ? P.part_cfl[w] : best;
        }
        const int p = c->parity ^ 1;  // the state the march just wrote
        const real *h = P.h[p], *qh = P.qh[p];
        const size_t lx = (size_t)P.lx;
        // counts below 2^31: the planner keeps the lattice under 2^30 points
        const int rows = P.chunks * P.rows, cols = P.strips * kOut;
        const int n_west = P.strips * rows, n = n_west + P.chunks * cols;
        for (int i = blockIdx.x * 256 + tid; i < n; i += gridDim.x * 256) {
            if (i < n_west) {  // west side of the first column of a strip, from the march's edge records
                const int s = i / rows, y = i % rows;
                if (s == 0) continue;  // west of strip 0: the border
                const float4 r = P.edge_first[i];
                const float2 l = P.edge_last[i - rows];
                if (r.w != 0.0f && l.x >= 0.0f) {
                    const size_t L = (size_t)(y + 2) * lx + (size_t)(s * kOut + 2);
                    lattice_cfl(d, P.len_v, r.z, l.y, l.x, r.y, r.x, P.side_v, L, best);
                }
            } else {  // south side of the first row of a chunk
                const int k = i - n_west, ch = k / cols, x = 2 + k % cols;
                const size_t L = (size_t)(2 + ch * P.rows) * lx + (size_t)x;
                if (P.live[L] && P.live[L - lx])
                    lattice_cfl(d, P.len_h, qh[L], P.z[L - lx], h[L - lx], P.z[L], h[L], P.side_h, L, best);
            }
        }
    }
    best = warp_min_u64(best);
    lim = __reduce_add_sync(0xffffffffu, lim);
    faces = __reduce_add_sync(0xffffffffu, faces);
    wet = __reduce_add_sync(0xffffffffu, wet);
    mb = __reduce_min_sync(0xffffffffu, mb);
    if ((tid & 31) == 0) {
        sh_min[tid >> 5] = best;
        sh_cnt[tid >> 5][0] = lim; sh_cnt[tid >> 5][1] = faces; sh_cnt[tid >> 5][2] = wet; sh_cnt[tid >> 5][3] = mb;
    }
    __syncthreads();
    if (tid == 0) {
        unsigned long long bmin = kCflEmpty;
        uint32_t l = 0, f = 0, wt = 0, m2 = __float_as_uint(1.0f);
        for (int w = 0; w < 8; ++w) {
            bmin = sh_min[w] < bmin ? sh_min[w] : bmin;
            l += sh_cnt[w][0]; f += sh_cnt[w][1]; wt += sh_cnt[w][2];
            m2 = sh_cnt[w][3] < m2 ? sh_cnt[w][3] : m2;
        }
        if (bmin != kCflEmpty) atomicMin(&c->cfl_packed, bmin);
        if (l) {
            atomicAdd(&c->limited_cells, l);
            atomicMin(&c->min_scale_bits, m2);
        }
        if (f) atomicAdd(&c->limited_faces, f);
        if (wt) atomicAdd(&c->wet, wt);
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

// Rows per chunk, warps per block and resident warps per SM of the march.
// A warp marches its rows after three rows of warm-up; chunks of 16 rows
// measured fastest on the 4096 x 4096 grid (the many short strips keep
// every SM busy to the end of a step), fewer rows when that would leave
// fewer than two waves of blocks. NHF_LATTICE_ROWS, NHF_LATTICE_WARPS
// (warps per block, 1..8) and NHF_LATTICE_BLOCKS (2, 3 or 4: 512, 768 or
// 1024 resident threads per SM, the register budget) override the choice.
static void lattice_shape(LatticePlan *P)
{
    // warps leave independently (no block barrier): small blocks free their
    // slots as soon as their strips are done
    const char *bw = getenv("NHF_LATTICE_WARPS");
    const int warps = (bw && atoi(bw) >= 1 && atoi(bw) <= kWarps) ? atoi(bw) : 2;
    const int per_row = (P->strips + warps - 1) / warps;  // blocks across the strips
    P->block_warps = (P->strips + per_row - 1) / per_row;  // <= warps, as even as the strips allow
    const char *occ = getenv("NHF_LATTICE_BLOCKS");
    const int want = occ ? atoi(occ) : 0;
    P->min_blocks = (want >= 2 && want <= 4) ? want : 4;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }
    const long long waves2 = 2LL * sms * P->min_blocks * kWarps / P->block_warps;
    const int need = P->ny + 1;
    int rows = 16;
    while (rows > 4 && (long long)((need + rows - 1) / rows) * per_row < waves2) rows /= 2;
    const char *env = getenv("NHF_LATTICE_ROWS");
    if (env && atoi(env) >= 1 && atoi(env) <= 256) rows = atoi(env);  // a lane's counters hold 10 bits
    P->rows = rows;
    P->chunks = (need + rows - 1) / rows;
}

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
    // strips of 28 columns cover cell columns 0..nx (column nx: the east
    // sides), chunks of P.rows rows cover cell rows 0..ny
    P.strips = (nx + 1 + kOut - 1) / kOut;
    lattice_shape(&P);
    P.lx = P.strips * kOut + kWest + 2;
    P.ly = P.chunks * P.rows + 5;  // 2 rows below, 3 above: the march loads a row ahead
    const size_t nl = (size_t)P.lx * P.ly;
    if (nl >= ((size_t)1 << 30)) return no("lattice too large");
    auto at = [&](int i, int j) { return (size_t)(j + 2) * P.lx + (i + kWest); };
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
    const size_t n_warps = (size_t)P.strips * P.chunks;
    const size_t o_part = take(16 * n_warps), o_pcfl = take(8 * n_warps);
    const size_t n_edge = (size_t)P.strips * P.chunks * P.rows;
    const size_t o_efirst = take(16 * n_edge), o_elast = take(8 * n_edge);
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
    // the three pairs are allocated as h0 qv0 qh0 h1 qv1 qh1 of equal size
    P.buffer_stride = (int32_t)(P.h[1] - P.h[0]);
    if (P.qv[1] - P.qv[0] != P.buffer_stride || P.qh[1] - P.qh[0] != P.buffer_stride)
        return no("lattice buffers not evenly spaced");
    P.z = (real *)(mem + o_z); P.nv = (real *)(mem + o_nv); P.nh = (real *)(mem + o_nh);
    P.bi = (int16_t *)(mem + o_bi);
    P.rain = P.rain_cells ? (int32_t *)(mem + o_rain) : nullptr;
    P.rain_time = (real *)(mem + o_rt); P.infil = (real *)(mem + o_inf);
    P.max_depth = (real *)(mem + o_md); P.max_speed = (real *)(mem + o_ms);
    P.peak_hi = (uint32_t *)(mem + o_ph); P.peak_lo = (uint32_t *)(mem + o_pl);
    if (P.horton) { P.f0 = (real *)(mem + o_f0); P.fc = (real *)(mem + o_fc); P.k = (real *)(mem + o_k); }
    P.terms = (float *)(mem + o_terms);
    P.touched = (uint32_t *)(mem + o_touch);
    P.part = (uint32_t *)(mem + o_part);
    P.part_cfl = (unsigned long long *)(mem + o_pcfl);
    P.edge_first = (float4 *)(mem + o_efirst);
    P.edge_last = (float2 *)(mem + o_elast);
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
    const LatticePlan &P = d.lat;
    const int per_block = (P.strips + P.block_warps - 1) / P.block_warps;
    const dim3 grid(per_block, P.chunks), block(32 * P.block_warps);
    if (P.min_blocks == 2) k_lattice_march<2><<<grid, block, 0, s>>>(d);
    else if (P.min_blocks == 3) k_lattice_march<3><<<grid, block, 0, s>>>(d);
    else k_lattice_march<4><<<grid, block, 0, s>>>(d);
    const long long edges = (long long)P.strips * P.chunks * (P.rows + kOut);
    const long long work = std::max<long long>(edges / 256, d.blocks / 8);
    k_lattice_close<<<(int)std::max<long long>(1, std::min<long long>(148 * 8, work)), 256, 0, s>>>(d);
}

void lattice_enqueue_batch_end(const Dev &d, cudaStream_t s)
{
    k_lattice_scatter<<<stream_grid((size_t)d.lat.lx * d.lat.ly), 256, 0, s>>>(d);
    tiled_enqueue_velocity(d, s);
}

}  // namespace nhf
