// Fused local-inertial step: one kernel launch per time step (plus, on large
// meshes, a separate CFL pass).
//
// Cells are split into tiles of T consecutive reference indices (T = 1024,
// 512 or 256; a tile covers T/256 whole budget blocks). A block owns one
// tile and stages in shared memory the tile (ring 0) and the rings of
// neighbours (graph distance 1..3) that one step of the reference's passes
// (solver_compact.py:439-613) and its CFL (617-641) reach:
//   ring <= 3  water level and bed           -> momentum q* of faces(ring <= 2)
//   ring <= 2  donor factor from those q*    -> final q of faces(ring <= 1)
//   ring <= 1  depth update from final q     -> CFL of the sides the tile owns
// That is the fused-CFL form. On meshes of several waves of tiles the plan
// drops ring 3 and the ring-1 depth recompute, and the CFL candidate of the
// next step is a separate grid-wide pass on the new state (k_cfl_tiled): the
// halo work saved outweighs one more launch per step (TilePlan::split).
// Every quantity is computed with the reference's operation order, so a cell
// that several tiles recompute gets the same bits everywhere; each output
// (depth, side q, extrema, budget block) has exactly one writer, its owner
// tile. depth, q and rain_time are double-buffered so that halo reads never
// see a neighbour's update of the same step. The last block to finish commits
// the clock and writes the trace row and (fused-CFL form) prepares the next
// step; in the split form the CFL pass's last block prepares it. A batch is
// one or two launches per step in one CUDA graph.
//
// The host planner below builds, per tile, the ring lists, the local side
// list and a local face CSR, all relative to the tile's first cell and side.
// Tiles whose relative tables coincide (regular grids numbered tile by tile)
// share one pattern, so the index tables stay in L2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "nhf_common.cuh"
#include "nhf_math.cuh"

namespace nhf {
namespace {

constexpr int kMaxSharedBytes = 108 * 1024;
// Resident blocks per SM the register budget is sized for: 5 x 256 threads
// (48 registers) for 256-cell tiles, 2 x 512 threads (64) for larger ones.
template <int NT>
constexpr int kMinBlocks = NT == 256 ? 5 : 2;
// The ensemble step reads its descriptor from shared memory and needs more
// registers: 4 x 256 or 2 x 512 threads (64 registers).
template <int NT>
constexpr int kEnsembleMinBlocks = NT == 256 ? 4 : 2;
constexpr uint8_t kOwned = 1, kFinal = 2;

// 4-byte asynchronous global -> shared copy (no register round trip); a
// thread waits for all of its copies with cp_async_wait_all.
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// ----------------------------------------------------------------- kernels

template <int CPT>
struct CellTerms {
    float removed[CPT], floor_v[CPT], level[CPT][5], discharge[CPT];
    int bi[CPT], kind[CPT];
};

struct Tile {
    int n_ext, n_r0, n_r01, n_don, n_sides, n_owned, n_qf, r0off, n_faces;
    int cbase, sbase;
    const int32_t *ext;
    const int32_t *srel;
    const uint32_t *lohi;
    const uint32_t *fdesc;
    const uint16_t *fidx;
};

// Face flux sums of one local cell (solver_compact.py:548-557) in the
// reference's CSR order.
__device__ __forceinline__ void face_sums(const Tile &tl, const float *sh_q, const float *sh_len, int slot,
                                          float fl[4])
{
    uint32_t fd = tl.fdesc[slot];
    int k = (int)(fd & 0xffffu);
    uint32_t counts = fd >> 16;
    for (int dd = 0; dd < 4; ++dd) {
        int cnt = (int)((counts >> (4 * dd)) & 15u);
        float face_flux = 0.0f;
        for (int j = 0; j < cnt; ++j) {
            int ls = tl.fidx[k++];
            face_flux += sh_q[ls] * sh_len[ls];
        }
        fl[dd] = face_flux;
    }
}

// The canonical 256-slot pairwise tree (stride 128 .. 1) run on every
// 256-thread half of the block at once; the sums land in threads 0, 256, ...
template <int NT>
__device__ __forceinline__ double tree_halves(double v, double *sh)
{
    const int tid = threadIdx.x;
    const int lane256 = tid & 255;
    sh[tid] = v;
    __syncthreads();
    for (int stride = 128; stride >= 32; stride >>= 1) {
        if (lane256 < stride) sh[tid] += sh[tid + stride];
        __syncthreads();
    }
    double r = 0.0;
    if (lane256 < 32) {
        r = sh[tid];
        for (int stride = 16; stride >= 1; stride >>= 1) r += __shfl_down_sync(0xffffffffu, r, stride);
    }
    __syncthreads();
    return r;
}

__device__ __forceinline__ float term_value(int t, int B, float removed, float floor_v, const float *level,
                                            float discharge, int bi, int kind)
{
    if (t == 0) return removed;
    if (t == 1) return kind == 0 ? 0.0f : floor_v;
    if (t == 2) return kind == 0 ? floor_v : 0.0f;
    if (t == 3) return 0.0f;  // pipe exchange: no coupling
    if (t < 4 + 5 * B) {
        const int b = (t - 4) / 5, q = (t - 4) % 5;
        if (b != bi || kind != 0) return 0.0f;
        // selected without a dynamic index, so the terms stay in registers
        return q == 0 ? level[0] : q == 1 ? level[1] : q == 2 ? level[2] : q == 3 ? level[3] : level[4];
    }
    return (t - 4 - 5 * B == bi) ? discharge : 0.0f;
}

// One fused step of tile t of the mesh described by d (n_tiles tiles).
// kHang: 0 no hanging edges, 1 hanging edges, 2 decided by d at run time.
// kGate (256-cell tiles, separate CFL pass): the gate controller's source
// terms of pond and gate cells (core/gate.py:151-193) from the depth update,
// reduced per 256-cell block into gd's partials.
template <bool kThetaOne, int kHang, int NT, int CPT, bool kGate = false>
__device__ __forceinline__ void step_tile(const Dev &d, const int t_index, const unsigned n_tiles,
                                          const GateDev *gd = nullptr)
{
    static_assert(!kGate || (NT == 256 && CPT == 1), "gate terms need one 256-cell budget block per tile");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ unsigned long long sh_min[NT / 32];
    __shared__ uint32_t sh_cnt[3];
    __shared__ uint32_t sh_minbits;
    __shared__ uint32_t sh_mask[CPT][NT / 256];
    __shared__ int sh_last;
    Ctl *c = d.ctl;
    const nhf_mesh &m = d.m;
    const int tid = threadIdx.x;

    if (tid == 0) { sh_cnt[0] = sh_cnt[1] = sh_cnt[2] = 0u; sh_minbits = __float_as_uint(1.0f); }
    if (tid < CPT * (NT / 256)) (&sh_mask[0][0])[tid] = 0u;
    const int active = c->active;
    if (!active) {
        // No physics this slot: the last block advances the slot and prepares the next.
        __syncthreads();
        if (tid == 0) {
            __threadfence();
            unsigned ticket = atomicAdd(&c->done_blocks, 1u);
            if (ticket == n_tiles - 1) {
                c->done_blocks = 0;
                finish_step(c);
                if (!d.plan.split && c->slot < d.batch_size)
                    prepare_step(d, c, cur_depth(d, c->parity), cur_q(d, c->parity));
            }
        }
        return;
    }
    const int parity = c->parity;
    const float dt = c->dt;
    const int raining = c->raining;
    const float *depth_in = parity ? d.depth_b : m.depth;
    float *depth_out = parity ? m.depth : d.depth_b;
    const float *q_in = parity ? d.q_b : m.q;
    float *q_out = parity ? m.q : d.q_b;
    const float *rt_in = parity ? d.rain_time_b : m.rain_time;
    float *rt_out = parity ? m.rain_time : d.rain_time_b;

    const TilePlan &P = d.plan;
    const bool hanging = kHang == 1 || (kHang == 2 && m.hang_cells > 0);
    Tile tl;
    {
        const int4 *head = P.tile_head + 4 * t_index;
        const int4 h0 = head[0], h1 = head[1], h2 = head[2], h3 = head[3];
        tl.n_ext = h0.x; tl.n_r0 = h0.y; tl.n_r01 = h0.z; tl.n_don = h0.w;
        tl.n_sides = h1.x; tl.n_owned = h1.y; tl.n_qf = h1.z; tl.r0off = h1.w;
        tl.n_faces = h2.x;
        tl.cbase = h2.y;
        tl.sbase = h2.z;
        tl.ext = P.ext_rel + h2.w;
        tl.srel = P.side_rel + h3.x;
        tl.lohi = P.side_lohi + h3.x;
        tl.fdesc = P.face_desc + h3.y;
        tl.fidx = P.face_idx + h3.z;
    }
    const int E = P.max_ext;
    // The first six arrays are dead once the depth update is done; the
    // budget reduction then reuses their 24 * E bytes.
    float *sh_h = reinterpret_cast<float *>(smem_raw);
    float *sh_rq = sh_h + E;     // rain rate of the cell (0 when not raining)
    float *sh_area = sh_rq + E;
    int *sh_g = reinterpret_cast<int *>(sh_area + E);
    int *sh_bi = sh_g + E;       // boundary id, -1 for none
    uint32_t *sh_fdesc = reinterpret_cast<uint32_t *>(sh_bi + E);
    float *sh_z = reinterpret_cast<float *>(sh_fdesc + E);
    float *sh_s = sh_z + E;      // donor factor, then the new depth
    float *sh_q = sh_s + E;      // q*, then final q
    float *sh_len = sh_q + P.max_sides;
    int32_t *sh_srel = reinterpret_cast<int32_t *>(sh_len + P.max_sides);
    uint32_t *sh_lohi = reinterpret_cast<uint32_t *>(sh_srel + P.max_sides);
    uint16_t *sh_fidx = reinterpret_cast<uint16_t *>(sh_lohi + P.max_sides);

    // P0: stage the tile in two asynchronous phases. (a) The pattern's index
    // tables (contiguous in global memory; the ring list goes to sh_g for now).
    for (int i = tid; i < tl.n_ext; i += NT) cp_async4(sh_g + i, tl.ext + i);
    for (int i = tid; i < tl.n_sides; i += NT) {
        cp_async4(sh_srel + i, tl.srel + i);
        cp_async4(sh_lohi + i, tl.lohi + i);
    }
    for (int i = tid; i <= tl.n_don; i += NT) cp_async4(sh_fdesc + i, tl.fdesc + i);
    for (int i = tid; i < (tl.n_faces + 1) >> 1; i += NT)  // patterns keep an even length
        cp_async4(reinterpret_cast<uint32_t *>(sh_fidx) + i, reinterpret_cast<const uint32_t *>(tl.fidx) + i);
    cp_async_wait_all();
    __syncthreads();
    // (b) Gathers: depth and bed of the tile and its rings, the per-cell
    // inputs of the donor rings (the rain pixel index parks in sh_rq), and q and
    // length of every local side.
    for (int i = tid; i < tl.n_ext; i += NT) {
        const int g = i ? tl.cbase + sh_g[i] : 0;
        sh_g[i] = g;
        if (i) cp_async4(sh_h + i, depth_in + g);
        else sh_h[0] = m.depth[0];
        cp_async4(sh_z + i, m.bed + g);
        if (i >= 1 && i <= tl.n_don) {
            cp_async4(sh_area + i, m.area + g);
            cp_async4(sh_bi + i, m.boundary_id + g);
            cp_async4(sh_rq + i, m.rain_index + g);
        }
    }
    for (int j = tid; j < tl.n_sides; j += NT) {
        const int gid = tl.sbase + sh_srel[j];
        cp_async4(sh_q + j, q_in + gid);
        cp_async4(sh_len + j, m.length + gid);
    }
    tl.srel = sh_srel;
    tl.lohi = sh_lohi;
    tl.fdesc = sh_fdesc;
    tl.fidx = sh_fidx;
    if (tid == 0) sh_s[0] = 0.0f;  // donor_scale of the exterior sentinel (the outer ring is never a donor)
    cp_async_wait_all();
    __syncthreads();

    // P1: momentum (solver_compact.py:439-486) for every local side. A side
    // whose flow height is below min_h gets q = +0 whatever its other inputs
    // (select then * bf), so their loads and arithmetic are skipped.
    for (int j = tid; j < tl.n_sides; j += NT) {
        const int gid = tl.sbase + tl.srel[j];
        const uint32_t lh = tl.lohi[j];
        const int a = (int)(lh & 0xffffu), b = (int)(lh >> 16);
        float zl = sh_z[a], zh = sh_z[b];
        float hl = zl + sh_h[a], hr = zh + sh_h[b];
        float xwh = maxf(hl, hr) - maxf(maxf(zl, zh), kDh);
        float new_q = 0.0f;
        if (!(xwh < d.min_h)) {
            float xq = sh_q[j];
            const float2 sdn = d.sdn[gid];
            float dx = sdn.x;
            float n = sdn.y;
            // exterior sides (exactly one neighbour, the sentinel slot 0) are closed
            // (sbf, build_boundary_fdb in domain.py:472-479; checked by the planner)
            float bf = (a == 0) != (b == 0) ? 0.0f : 1.0f;
            float difference = hr - hl;
            if (hanging) {
                int index = m.edge_index[gid];
                if (index >= 0 && sh_h[a] > d.min_h && sh_h[b] > d.min_h) {
                    int axis = m.topology[3 * gid] == 2 ? 1 : 0;
                    float o0 = m.offsets[2 * index], o1 = m.offsets[2 * index + 1];
                    if (o0 != 0.0f) difference -= d.gradients[2 * m.slots[2 * index] + axis] * o0;
                    if (o1 != 0.0f) difference += d.gradients[2 * m.slots[2 * index + 1] + axis] * o1;
                }
            }
            float xdq = (d.neg_g * difference / dx) * maxf(xwh, 0.0f) * dt;
            float ratio = 0.0f;
            if (xq != 0.0f) ratio = xq / pow_f32(maxf(xwh, 0.00001f), d.seven_thirds);
            float xf = 1.0f + d.g * dt * (n * n) * fabsf(ratio);
            float nb;
            if (kThetaOne) {
                nb = 0.0f + 0.0f;
            } else {
                int so = m.topology[3 * gid];
                int dl = so == 2 ? 0 : 2, dr = so == 2 ? 1 : 3;
                int ga = sh_g[a], gb = sh_g[b];
                nb = boundary_neighbor_sum(xq, d.face_qn[4 * ga + dl], d.face_qn[4 * gb + dr],
                                           m.open_face[4 * ga + dl], m.open_face[4 * gb + dr]);
            }
            new_q = (d.sita * xq + d.half_rest * nb + xdq) / xf;
            new_q *= bf;
        }
        sh_q[j] = new_q;
    }
    __syncthreads();

    // P2: donor factor (solver_compact.py:491-514) for the donor rings.
    {
        uint32_t my_limited = 0;
        uint32_t my_min = __float_as_uint(1.0f);
        for (int i = 1 + tid; i <= tl.n_don; i += NT) {
            const int bi = sh_bi[i];
            int kind = -1;
            float discharge = 0.0f;
            if (bi >= 0) {
                kind = m.kind[bi];
                if (kind == 1) discharge = d.values[bi] * m.weight[sh_g[i]];
            }
            // rain rate from the staged pixel index, kept for the depth update
            const float rainq = raining ? d.rain_rates[__float_as_int(sh_rq[i])] : 0.0f;
            sh_rq[i] = rainq;
            float pipe = 0.0f;
            float positive = (maxf(pipe, 0.0f) + maxf(discharge, 0.0f)) * dt;
            float area = sh_area[i];
            float available = sh_h[i] * area + positive + rainq * dt * area;
            float outgoing = (maxf(-pipe, 0.0f) + maxf(-discharge, 0.0f)) * dt;
            uint32_t fd = tl.fdesc[i];
            int k = (int)(fd & 0xffffu);
            uint32_t counts = fd >> 16;
            for (int dd = 0; dd < 4; ++dd) {
                int cntd = (int)((counts >> (4 * dd)) & 15u);
                for (int jj = 0; jj < cntd; ++jj) {
                    int ls = tl.fidx[k++];
                    float signed_q = sh_q[ls] * sh_len[ls];
                    if (dd == 0 || dd == 2) signed_q = -signed_q;
                    outgoing += maxf(signed_q, 0.0f) * dt;
                }
            }
            float sc = 1.0f;
            if (outgoing > available && kind != 0) {
                sc = available / outgoing;
                if (i <= tl.n_r0) {
                    my_limited += 1;
                    uint32_t bits = __float_as_uint(sc);
                    my_min = bits < my_min ? bits : my_min;
                }
            }
            sh_s[i] = sc;
        }
        if (my_limited) {
            atomicAdd(&sh_cnt[0], my_limited);
            atomicMin(&sh_minbits, my_min);
        }
    }
    __syncthreads();

    // P3: final discharge of the final faces (rings 0..1, ring 0 in the split form)
    // (solver_compact.py:516-522).
    {
        uint32_t my_faces = 0;
        for (int j = tid; j < tl.n_qf; j += NT) {
            const uint32_t lh = tl.lohi[j];
            const int a = (int)(lh & 0xffffu), b = (int)(lh >> 16);
            float q = sh_q[j];
            int donor = q >= 0.0f ? a : b;
            float sc = sh_s[donor];
            if (j < tl.n_owned && q != 0.0f && sc < 1.0f) my_faces += 1;
            sh_q[j] = q * sc;
        }
        if (my_faces) atomicAdd(&sh_cnt[1], my_faces);
    }
    __syncthreads();

    // P4: sources and depth update (solver_compact.py:525-610). Ring 0 cells
    // are mapped to threads as tile offset o = tid + NT * k, so each budget
    // block of the tile sits on one 256-thread half in thread order.
    CellTerms<CPT> terms;
    uint32_t my_wet = 0;
    int g_off = -1;  // kGate: first source term of this pond or gate cell, -1 elsewhere
    float g_v[6] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    const int T = d.terms;
    const int B = m.b_num;
    const uint32_t step_hi = c->step_end[0], step_lo = c->step_end[1];
    // P4a: issue every per-cell load of this thread's ring-0 cells before any
    // store, so the loads overlap.
    int in_g[CPT], in_slot[CPT], in_kind[CPT];
    float in_w[CPT], in_rt[CPT], in_f0[CPT], in_fc[CPT], in_k[CPT], in_inf[CPT], in_hgt[CPT], in_wid[CPT],
        in_ms[CPT], in_md[CPT];
#pragma unroll
    for (int kk = 0; kk < CPT; ++kk) {
        const int o = tid + NT * kk;
        const int slot = o - tl.r0off + 1;
        in_slot[kk] = (o < tl.r0off || slot > tl.n_r0) ? -1 : slot;
        in_g[kk] = tl.cbase + o;
        in_kind[kk] = -1;
        in_w[kk] = in_rt[kk] = in_f0[kk] = in_fc[kk] = in_k[kk] = 0.0f;
        in_inf[kk] = in_hgt[kk] = in_wid[kk] = in_ms[kk] = in_md[kk] = 0.0f;
        if (in_slot[kk] < 0) continue;
        const int g = in_g[kk];
        const int bi = sh_bi[slot];
        if (bi >= 0) { in_kind[kk] = m.kind[bi]; in_w[kk] = m.weight[g]; }
        if (sh_rq[slot] > 0.0f) { in_rt[kk] = rt_in[g]; in_f0[kk] = m.f0[g]; in_fc[kk] = m.fc[g]; in_k[kk] = m.k[g]; }
        in_inf[kk] = m.infiltration[g];
        in_hgt[kk] = m.height[g];
        in_wid[kk] = m.width[g];
        in_ms[kk] = m.max_speed[g];
        in_md[kk] = m.max_depth[g];
    }
    // P4b: the update itself.
#pragma unroll
    for (int kk = 0; kk < CPT; ++kk) {
        terms.removed[kk] = 0.0f; terms.floor_v[kk] = 0.0f; terms.discharge[kk] = 0.0f;
        for (int q5 = 0; q5 < 5; ++q5) terms.level[kk][q5] = 0.0f;
        terms.bi[kk] = -1; terms.kind[kk] = -1;
        const int slot = in_slot[kk];
        if (slot < 0) continue;
        const int g = in_g[kk];
        const int bi = sh_bi[slot];
        const int kind = in_kind[kk];
        terms.bi[kk] = bi; terms.kind[kk] = kind;
        float sc = sh_s[slot];
        float pq = 0.0f;
        float pipe = maxf(pq, 0.0f) + minf(pq, 0.0f) * sc;
        float discharge = 0.0f;
        if (kind == 1) {
            float requested = d.values[bi] * in_w[kk];
            discharge = maxf(requested, 0.0f) + minf(requested, 0.0f) * sc;
            terms.discharge[kk] = discharge * dt;
        }
        float ssq = pipe + discharge;
        float rainq = sh_rq[slot];
        float infil;
        if (rainq > 0.0f) {
            float rt = in_rt[kk] + dt;
            rt_out[g] = rt;
            float f0 = in_f0[kk], fc = in_fc[kk];
            float diff = f0 - fc;
            infil = diff == 0.0f ? fc + 0.0f : fc + diff * exp_f32(-in_k[kk] * rt / 3600.0f);
            if (__float_as_uint(infil) != __float_as_uint(in_inf[kk])) m.infiltration[g] = infil;
        } else {
            infil = in_inf[kk];
        }
        float fl[4];
        face_sums(tl, sh_q, sh_len, slot, fl);
        float ql = fl[0], qr = fl[1], qb = fl[2], qt = fl[3];
        float tq = ql - qr + qb - qt + ssq;
        float ea = sh_area[slot];
        float rain_depth = rainq * dt;
        float flux = tq * dt;
        // flux / ea for flux = +-0 is flux itself: skip the division
        float increment = (flux == 0.0f ? flux : flux / ea) + rain_depth;
        float previous = sh_h[slot];
        float raw_depth = previous + increment;
        float removed = minf(infil * dt, maxf(raw_depth, 0.0f));
        raw_depth -= removed;
        float floor_v = maxf(-raw_depth, 0.0f);
        terms.removed[kk] = removed * ea;
        terms.floor_v[kk] = floor_v * ea;
        float depth;
        if (kind == 0) {
            float target = maxf(d.level_values[bi] - sh_z[slot], 0.0f);
            terms.level[kk][0] = (target - previous) * ea;
            terms.level[kk][1] = -(ql - qr + qb - qt) * dt;
            terms.level[kk][2] = -pipe * dt;
            terms.level[kk][3] = -rain_depth * ea;
            terms.level[kk][4] = removed * ea;
            depth = target;
        } else {
            depth = maxf(raw_depth, 0.0f);
        }
        depth_out[g] = depth;
        sh_s[slot] = depth;
        float h = maxf(depth, 0.01f);
        float u = 0.0f, v = 0.0f;
        if (depth >= d.min_h) {
            // x / 2 and x * 0.5 are the same correctly rounded value
            u = (ql + qr) / in_hgt[kk] / h * 0.5f;
            v = (qb + qt) / in_wid[kk] / h * 0.5f;
        }
        float s2 = u * u + v * v;
        float speed = s2 == 0.0f ? 0.0f : sqrtf(s2);
        if (speed > in_ms[kk]) m.max_speed[g] = speed;
        if (depth > in_md[kk]) {
            m.max_depth[g] = depth;
            m.peak_hi[g] = step_hi; m.peak_lo[g] = step_lo;
        }
        my_wet += depth >= d.min_h ? 1u : 0u;
        if (kGate) {
            // record_cell, measure_inventory and the rounding term
            // (solver_compact.py:595-604; gate.py:151-193)
            const int cg = gd->cell_gate[g];
            g_off = gd->pond[g] == 1 ? 4 * gd->count + 2 : (cg >= 0 ? 4 * gd->count + 8 + 6 * cg : -1);
            if (g_off >= 0) {
                float applied_floor = floor_v, level_exchange = 0.0f;
                if (kind == 0) {
                    applied_floor = 0.0f;
                    level_exchange = (depth - previous) * ea - (ql - qr + qb - qt) * dt - pipe * dt
                                     - rain_depth * ea + removed * ea;
                }
                g_v[0] = rain_depth * ea;
                g_v[1] = removed * ea;
                g_v[2] = applied_floor * ea;
                g_v[3] = pipe * dt;
                g_v[4] = (ssq - pipe) * dt + level_exchange;
                const float rounding = (depth - previous) - increment + removed - applied_floor;
                g_v[5] = rounding * ea - level_exchange;
            }
        }
        if (T <= 32) {
            uint32_t mask = 0;
            if (terms.removed[kk] != 0.0f) mask |= 1u;
            if (terms.floor_v[kk] != 0.0f) mask |= kind == 0 ? 4u : 2u;
            if (kind == 0)
                for (int q5 = 0; q5 < 5; ++q5)
                    if (terms.level[kk][q5] != 0.0f) mask |= 1u << (4 + 5 * bi + q5);
            if (kind == 1 && terms.discharge[kk] != 0.0f) mask |= 1u << (4 + 5 * B + bi);
            if (mask) atomicOr(&sh_mask[kk][tid >> 8], mask);
        }
    }
    // ring 1 (fused-CFL form): the new depth only, for the CFL of owned sides
    for (int i = tl.n_r0 + 1 + tid; i <= tl.n_r01; i += NT) {
        const int g = sh_g[i];
        const int bi = sh_bi[i];
        const int kind = bi >= 0 ? m.kind[bi] : -1;
        float sc = sh_s[i];
        float pq = 0.0f;
        float pipe = maxf(pq, 0.0f) + minf(pq, 0.0f) * sc;
        float discharge = 0.0f;
        if (kind == 1) {
            float requested = d.values[bi] * m.weight[g];
            discharge = maxf(requested, 0.0f) + minf(requested, 0.0f) * sc;
        }
        float ssq = pipe + discharge;
        float rainq = sh_rq[i];
        float infil;
        if (rainq > 0.0f) {
            float rt = rt_in[g] + dt;
            float f0 = m.f0[g], fc = m.fc[g];
            float diff = f0 - fc;
            infil = diff == 0.0f ? fc + 0.0f : fc + diff * exp_f32(-m.k[g] * rt / 3600.0f);
        } else {
            infil = m.infiltration[g];
        }
        float fl[4];
        face_sums(tl, sh_q, sh_len, i, fl);
        float tq = fl[0] - fl[1] + fl[2] - fl[3] + ssq;
        float ea = sh_area[i];
        float rain_depth = rainq * dt;
        float flux = tq * dt;
        float increment = (flux == 0.0f ? flux : flux / ea) + rain_depth;
        float raw_depth = sh_h[i] + increment;
        float removed = minf(infil * dt, maxf(raw_depth, 0.0f));
        raw_depth -= removed;
        float depth = kind == 0 ? maxf(d.level_values[bi] - sh_z[i], 0.0f) : maxf(raw_depth, 0.0f);
        sh_s[i] = depth;
    }
    __syncthreads();

    // Budget partials: one writer per (budget block, term), the canonical
    // pairwise tree of the 256 cells of a block (stride 128 .. 1). Terms
    // whose values some cell of the tile holds are staged together in the
    // dead shared arrays; one warp then reduces one (block, term): lane l
    // forms ((v[l] + v[l+128]) + (v[l+64] + v[l+192])) + ((v[l+32] + v[l+160])
    // + (v[l+96] + v[l+224])), which are the tree's strides 128, 64 and 32,
    // and a shuffle tree does strides 16 .. 1.
    if (T <= 32) {
        double *buf = reinterpret_cast<double *>(smem_raw);
        const int cap = (24 * E) / (NT * 8);  // >= 1: the planner pads E
        const int lane_b = tid & 31, warp_b = tid >> 5;
#pragma unroll
        for (int kk = 0; kk < CPT; ++kk) {
            const int blk0 = (tl.cbase >> 8) + kk * (NT / 256);
            uint32_t any = 0;
            for (int hh = 0; hh < NT / 256; ++hh) any |= sh_mask[kk][hh];
            while (any) {
                uint32_t chunk = 0;
                int n = 0;
                for (uint32_t rest = any; rest && n < cap; rest &= rest - 1, ++n) chunk |= rest & (0u - rest);
                any &= ~chunk;
                int j = 0;
                for (uint32_t rest = chunk; rest; rest &= rest - 1, ++j) {
                    const int t = __ffs(rest) - 1;
                    buf[j * NT + tid] = (double)term_value(t, B, terms.removed[kk], terms.floor_v[kk], terms.level[kk],
                                                           terms.discharge[kk], terms.bi[kk], terms.kind[kk]);
                }
                __syncthreads();
                const int halves = NT / 256;
                for (int item = warp_b; item < halves * n; item += NT / 32) {
                    const int h = item % halves, jj = item / halves;
                    const double *v = buf + jj * NT + h * 256;
                    double r = ((v[lane_b] + v[lane_b + 128]) + (v[lane_b + 64] + v[lane_b + 192])) +
                               ((v[lane_b + 32] + v[lane_b + 160]) + (v[lane_b + 96] + v[lane_b + 224]));
                    for (int stride = 16; stride >= 1; stride >>= 1) r += __shfl_down_sync(0xffffffffu, r, stride);
                    if (lane_b == 0) {
                        uint32_t rest = chunk;
                        for (int q = 0; q < jj; ++q) rest &= rest - 1;
                        const int t = __ffs(rest) - 1;
                        const int blk = blk0 + h;
                        if (blk < d.blocks && ((sh_mask[kk][h] >> t) & 1u))
                            acc_add(d.acc_sum + (size_t)blk * T + t, d.acc_comp + (size_t)blk * T + t, r);
                    }
                }
                // the staging area is reused only by a further chunk; after the
                // last one the other warps go on while these finish
                if (any || kk + 1 < CPT) __syncthreads();
            }
        }
    }
    // More than 32 terms (over five boundaries): one term at a time, skipped
    // when no cell of the tile holds it.
    if (T > 32) {
#pragma unroll
        for (int kk = 0; kk < CPT; ++kk) {
            const int blk0 = (tl.cbase >> 8) + kk * (NT / 256);
            for (int t = 0; t < T; ++t) {
                float val = term_value(t, B, terms.removed[kk], terms.floor_v[kk], terms.level[kk],
                                       terms.discharge[kk], terms.bi[kk], terms.kind[kk]);
                if (!__syncthreads_or(val != 0.0f)) continue;
                // the tree's NT doubles live in the dead shared arrays (24 * E >= 8 * NT)
                double sum = tree_halves<NT>((double)val, reinterpret_cast<double *>(smem_raw));
                const int blk = blk0 + (tid >> 8);
                if ((tid & 255) == 0 && blk < d.blocks && sum != 0.0)
                    acc_add(d.acc_sum + (size_t)blk * T + t, d.acc_comp + (size_t)blk * T + t, sum);
            }
        }
    }

    if (kGate) {
        // gate source terms: the pond group, then gate by gate, six terms
        // each, the canonical 256-cell tree in the dead shared arrays
        double *buf = reinterpret_cast<double *>(smem_raw);
        const int blk = tl.cbase >> 8;
        for (int grp = -1; grp < gd->count; ++grp) {
            const int off = grp < 0 ? 4 * gd->count + 2 : 4 * gd->count + 8 + 6 * grp;
            if (!__syncthreads_or(g_off == off)) continue;
#pragma unroll
            for (int k = 0; k < 6; ++k) {
                const float val = g_off == off ? g_v[k] : 0.0f;
                if (!__syncthreads_or(val != 0.0f)) continue;
                const double sum = tree_halves<NT>((double)val, buf);
                if (tid == 0) {
                    const size_t idx = (size_t)blk * gd->terms + off + k;
                    acc_add(gd->acc_sum + idx, gd->acc_comp + idx, sum);
                }
            }
        }
    }

    // P5: owned sides: final q out; in the fused-CFL form also the CFL of the
    // owned sides with the new depths (the split form's CFL pass follows).
    const bool split = P.split != 0;
    unsigned long long best = kCflEmpty;
    // A side at the 0.01 m face-depth floor with q = 0 has the CFL value
    // afa * L / sqrt(g * 0.01); it is reused while L repeats.
    float dry_len = -1.0f, dry_cfl = 0.0f;
    for (int j = tid; j < tl.n_owned; j += NT) {
        const int gid = tl.sbase + tl.srel[j];
        float qv = sh_q[j];
        q_out[gid] = qv;
        if (split) continue;
        const uint32_t lh = tl.lohi[j];
        const int a = (int)(lh & 0xffffu), b = (int)(lh >> 16);
        if (a != 0 && b != 0) {
            float zl = sh_z[a], zh = sh_z[b];
            float head = maxf(zl + sh_s[a], zh + sh_s[b]);
            float h = maxf(head - maxf(maxf(zl, zh), kDh), 0.01f);
            float cfl;
            if (h == 0.01f && qv == 0.0f) {
                if (sh_len[j] != dry_len) {
                    dry_len = sh_len[j];
                    dry_cfl = d.afa * dry_len / (sqrtf(d.g * h) + fabsf(qv) / h);
                }
                cfl = dry_cfl;
            } else {
                cfl = d.afa * sh_len[j] / (sqrtf(d.g * h) + fabsf(qv) / h);
            }
            unsigned long long key = ((unsigned long long)__float_as_uint(cfl) << 32) | (unsigned)gid;
            best = key < best ? key : best;
        }
    }
    if (!split) {
        best = warp_min_u64(best);
        if ((tid & 31) == 0) sh_min[tid >> 5] = best;
    }
    if (my_wet) atomicAdd(&sh_cnt[2], my_wet);
    __syncthreads();
    if (tid == 0) {
        if (!split) {
            unsigned long long bmin = kCflEmpty;
            for (int w = 0; w < NT / 32; ++w) bmin = sh_min[w] < bmin ? sh_min[w] : bmin;
            if (bmin != kCflEmpty) atomicMin(&c->cfl_packed, bmin);
        }
        if (sh_cnt[0]) {
            atomicAdd(&c->limited_cells, sh_cnt[0]);
            atomicMin(&c->min_scale_bits, sh_minbits);
        }
        if (sh_cnt[1]) atomicAdd(&c->limited_faces, sh_cnt[1]);
        if (sh_cnt[2]) atomicAdd(&c->wet, sh_cnt[2]);
        __threadfence();
        unsigned ticket = atomicAdd(&c->done_blocks, 1u);
        sh_last = ticket == n_tiles - 1;
    }
    __syncthreads();
    if (!sh_last || tid != 0) return;
    // Last block: (fused-CFL form: the CFL result,) trace row, clock commit,
    // the new state becomes current (and the next step is prepared).
    __threadfence();
    c->done_blocks = 0;
    if (!split) {
        unsigned long long packed = atomicExch(&c->cfl_packed, kCflEmpty);
        if (packed == kCflEmpty) {
            c->ndt = __uint_as_float(0x7f800000u);
            c->cfl_arg = 0;
        } else {
            c->ndt = __uint_as_float((uint32_t)(packed >> 32));
            c->cfl_arg = (int32_t)(packed & 0xffffffffu);
        }
    }
    finish_step(c);
    c->parity = parity ^ 1;
    if (!split && c->slot < d.batch_size) prepare_step(d, c, depth_out, q_out);
}

// CFL pass (solver_compact.py:617-641) over sides [first, end) with stride,
// on the current (just updated) state; each block adds its minimum packed
// key (cfl bits, side id) and the last of `blocks` blocks sets ndt /
// cfl_arg (the lowest side id attains the minimum) and prepares the next
// step (solver_compact.py:364-382).
__device__ __forceinline__ void cfl_pass(const Dev &d, int first, int end, int stride, unsigned blocks,
                                         const GateDev *gd = nullptr)
{
    __shared__ unsigned long long sh[32];
    __shared__ bool last;
    __shared__ int prepared;
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    const int active = c->active;
    const float *depth = cur_depth(d, c->parity);
    const float *q = cur_q(d, c->parity);
    unsigned long long best = kCflEmpty;
    if (active) {
        for (int si = first + (int)threadIdx.x; si < end; si += stride) {
            const int el = m.topology[3 * si + 1], eh = m.topology[3 * si + 2];
            if (el != 0 && eh != 0) {
                const float zl = m.bed[el], zh = m.bed[eh];
                const float head = maxf(zl + depth[el], zh + depth[eh]);
                const float h = maxf(head - maxf(maxf(zl, zh), kDh), 0.01f);
                const float cfl = d.afa * m.length[si] / (sqrtf(d.g * h) + fabsf(q[si]) / h);
                const unsigned long long key = ((unsigned long long)__float_as_uint(cfl) << 32) | (unsigned)si;
                best = key < best ? key : best;
            }
        }
    }
    best = warp_min_u64(best);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = best;
    __syncthreads();
    if (warp == 0) {
        best = lane < (int)(blockDim.x >> 5) ? sh[lane] : kCflEmpty;
        best = warp_min_u64(best);
        if (lane == 0) {
            if (best != kCflEmpty) atomicMin(&c->cfl_packed, best);
            __threadfence();
            const unsigned ticket = atomicAdd(&c->done_blocks, 1u);
            last = ticket == blocks - 1;
        }
    }
    __syncthreads();
    if (!last) return;
    if (threadIdx.x == 0) {
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
        }
        prepared = c->slot < d.batch_size;
        if (prepared) prepare_step(d, c, depth, q);
    }
    if (!gd) return;
    // gate runs: the next step's check_gates (trigger check and beds at its
    // start) by this block, once that step is prepared in this batch
    __syncthreads();
    if (!prepared || !c->active) return;
    const uint32_t hi = c->now[0], lo = c->now[1];
    gate_check(d, *gd, hi, lo);
    __syncthreads();
    gate_move_beds(d, *gd, hi, lo);
}

template <bool kThetaOne, bool kHanging, int NT, int CPT>
__global__ void __launch_bounds__(NT, kMinBlocks<NT>) k_step_tiled(const __grid_constant__ Dev d)
{
    step_tile<kThetaOne, kHanging ? 1 : 0, NT, CPT>(d, blockIdx.x, gridDim.x);
}

// The fused step with the gate controller's source terms (256-cell tiles,
// split plans); the controller's bed motion and exchange volumes are
// separate passes around it.
template <bool kThetaOne, bool kHanging>
__global__ void __launch_bounds__(256, 4) k_step_tiled_gate(const __grid_constant__ Dev d,
                                                            const __grid_constant__ GateDev g)
{
    step_tile<kThetaOne, kHanging ? 1 : 0, 256, 1, true>(d, blockIdx.x, gridDim.x, &g);
}

// CFL pass of one mesh after its fused step (grid-stride over the sides);
// split plans only.
__global__ void __launch_bounds__(256) k_cfl_tiled(const __grid_constant__ Dev d)
{
    if (!d.plan.split) return;
    cfl_pass(d, 1 + (int)(blockIdx.x * blockDim.x), d.m.s_num, (int)(gridDim.x * blockDim.x), gridDim.x);
}

// CFL pass of a gate run (split plan): also the next step's check_gates.
__global__ void __launch_bounds__(256) k_cfl_tiled_gate(const __grid_constant__ Dev d, const __grid_constant__ GateDev g)
{
    cfl_pass(d, 1 + (int)(blockIdx.x * blockDim.x), d.m.s_num, (int)(gridDim.x * blockDim.x), gridDim.x, &g);
}

// Ensemble step: one launch advances every member mesh by one of its own
// time steps. items[i] = (member, tile); the grid is persistent (a block
// takes items blockIdx.x, + gridDim.x, ...) or one block per item. The
// member's descriptor is staged in shared memory once per change of member.
template <bool kThetaOne, int NT, int CPT>
__global__ void __launch_bounds__(NT, kEnsembleMinBlocks<NT>)
    k_step_ensemble(const Dev *__restrict__ devs, const int2 *__restrict__ items, int n_items)
{
    for (int it = blockIdx.x; it < n_items; it += gridDim.x) {
        const int2 w = items[it];
        // the member's descriptor is read in place through the read-only
        // data path (it does not change during the launch)
        const Dev &md = devs[w.x];
        __syncthreads();  // the previous item's shared arrays are dead
        step_tile<kThetaOne, 2, NT, CPT>(md, w.y, (unsigned)md.plan.n_tiles);
    }
}

// Batch start: the rain-time second buffer equals the caller's buffer (cells
// that do not rain during the batch are never rewritten).
__global__ void k_batch_start(Dev d)
{
    const nhf_mesh &m = d.m;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.e_num; i += gridDim.x * blockDim.x)
        d.rain_time_b[i] = m.rain_time[i];
}

// Batch end: bring the current state back into the caller's buffers.
__global__ void k_batch_end(Dev d)
{
    const nhf_mesh &m = d.m;
    Ctl *c = d.ctl;
    __shared__ int last;
    if (c->parity) {
        const int stride = gridDim.x * blockDim.x;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.e_num; i += stride) {
            m.depth[i] = d.depth_b[i];
            m.rain_time[i] = d.rain_time_b[i];
        }
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < m.s_num; i += stride) m.q[i] = d.q_b[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        unsigned ticket = atomicAdd(&c->done_blocks, 1u);
        last = ticket == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        c->done_blocks = 0;
        c->parity = 0;
    }
}

// u, v of the current state (the velocity function, solver_compact.py:355-362).
__device__ __forceinline__ void velocity_cell(const Dev &d, int ei)
{
    const nhf_mesh &m = d.m;
    {
        float fl[4];
        for (int dd = 0; dd < 4; ++dd) {
            float total = 0.0f;
            int p = m.face_ptr[4 * ei + dd], cnt = m.face_count[4 * ei + dd];
            for (int j = 0; j < cnt; ++j) {
                int si = m.isl_data[p + j];
                total += m.q[si] * m.length[si];
            }
            fl[dd] = total;
        }
        float depth = m.depth[ei];
        float h = maxf(depth, 0.01f);
        float u = 0.0f, v = 0.0f;
        if (depth >= d.min_h) {
            u = (fl[0] + fl[1]) / m.height[ei] / h / 2.0f;
            v = (fl[2] + fl[3]) / m.width[ei] / h / 2.0f;
        }
        m.u[ei] = u;
        m.v[ei] = v;
    }
}

__global__ void k_velocity(const __grid_constant__ Dev d)
{
    for (int ei = 1 + blockIdx.x * blockDim.x + threadIdx.x; ei < d.m.e_num; ei += gridDim.x * blockDim.x)
        velocity_cell(d, ei);
}

// --------------------------------------------------------------- planner

struct Pattern {
    std::vector<int32_t> counts;  // 8
    std::vector<int32_t> ext;
    std::vector<int32_t> srel;
    std::vector<uint32_t> lohi;
    std::vector<uint32_t> fdesc;
    std::vector<uint16_t> fidx;
};

uint64_t fnv(uint64_t h, const void *p, size_t n)
{
    const unsigned char *b = (const unsigned char *)p;
    for (size_t i = 0; i < n; ++i) { h ^= b[i]; h *= 1099511628211ULL; }
    return h;
}

uint64_t pattern_hash(const Pattern &p)
{
    uint64_t h = 1469598103934665603ULL;
    h = fnv(h, p.counts.data(), p.counts.size() * 4);
    h = fnv(h, p.ext.data(), p.ext.size() * 4);
    h = fnv(h, p.srel.data(), p.srel.size() * 4);
    h = fnv(h, p.lohi.data(), p.lohi.size() * 4);
    h = fnv(h, p.fdesc.data(), p.fdesc.size() * 4);
    h = fnv(h, p.fidx.data(), p.fidx.size() * 2);
    return h;
}

bool same(const Pattern &a, const Pattern &b)
{
    return a.counts == b.counts && a.ext == b.ext && a.srel == b.srel && a.lohi == b.lohi && a.fdesc == b.fdesc &&
           a.fidx == b.fidx;
}

struct HostMesh {
    int e, s;
    std::vector<int32_t> topo, fptr, fcnt, isl;
    std::vector<uint8_t> sbf;
};

int copy_back(const nhf_mesh &m, cudaStream_t st, HostMesh &hm)
{
    hm.e = m.e_num; hm.s = m.s_num;
    hm.topo.resize((size_t)m.s_num * 3);
    hm.fptr.resize((size_t)m.e_num * 4);
    hm.fcnt.resize((size_t)m.e_num * 4);
    hm.isl.resize((size_t)(m.isl_len > 0 ? m.isl_len : 1));
    hm.sbf.resize((size_t)m.s_num);
    if (cudaMemcpyAsync(hm.topo.data(), m.topology, hm.topo.size() * 4, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(hm.sbf.data(), m.sbf, hm.sbf.size(), cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(hm.fptr.data(), m.face_ptr, hm.fptr.size() * 4, cudaMemcpyDeviceToHost, st) ||
        cudaMemcpyAsync(hm.fcnt.data(), m.face_count, hm.fcnt.size() * 4, cudaMemcpyDeviceToHost, st) ||
        (m.isl_len > 0 && cudaMemcpyAsync(hm.isl.data(), m.isl_data, (size_t)m.isl_len * 4, cudaMemcpyDeviceToHost, st)) ||
        cudaStreamSynchronize(st))
        return 1;
    return 0;
}

// Sides listed by each cell must be exactly the sides naming that cell as a
// neighbour; every side must be listed by its owner (lower, else higher).
bool consistent(const HostMesh &hm, std::string &why)
{
    std::vector<int> listed(hm.s, 0);
    for (int c = 1; c < hm.e; ++c)
        for (int dd = 0; dd < 4; ++dd) {
            int p = hm.fptr[4 * c + dd], n = hm.fcnt[4 * c + dd];
            if (n < 0 || n > 15) { why = "a face has more than 15 sides"; return false; }
            for (int j = 0; j < n; ++j) {
                int sid = hm.isl[p + j];
                if (sid < 1 || sid >= hm.s) { why = "face lists an invalid side"; return false; }
                int lo = hm.topo[3 * sid + 1], hi = hm.topo[3 * sid + 2];
                if (lo != c && hi != c) { why = "face lists a side that does not touch the cell"; return false; }
                listed[sid] += 1;
            }
        }
    for (int sid = 1; sid < hm.s; ++sid) {
        int lo = hm.topo[3 * sid + 1], hi = hm.topo[3 * sid + 2];
        int expect = (lo != 0) + (hi != 0);
        if (expect == 0 || listed[sid] != expect || lo == hi) { why = "a side is not listed by exactly its cells"; return false; }
        // the fused step derives the closed-edge flag from the topology
        if (hm.sbf[sid] != ((lo == 0) != (hi == 0) ? 1 : 0)) { why = "sbf differs from the exterior-side rule"; return false; }
    }
    return true;
}

int plan_tiles(const HostMesh &hm, int T, std::vector<Pattern> &patterns, std::vector<int32_t> &tile_pattern,
               std::vector<int32_t> &tile_cbase, std::vector<int32_t> &tile_sbase, int &max_ext, int &max_sides,
               int &max_faces, int rings, std::string &why)
{
    const int e = hm.e, s = hm.s;
    // cell adjacency through interior sides
    std::vector<int> deg(e + 1, 0);
    for (int sid = 1; sid < s; ++sid) {
        int lo = hm.topo[3 * sid + 1], hi = hm.topo[3 * sid + 2];
        if (lo && hi) { deg[lo]++; deg[hi]++; }
    }
    std::vector<int> aptr(e + 1, 0);
    for (int c = 0; c < e; ++c) aptr[c + 1] = aptr[c] + deg[c];
    std::vector<int> adj(aptr[e]);
    std::vector<int> fill(aptr.begin(), aptr.end() - 1);
    for (int sid = 1; sid < s; ++sid) {
        int lo = hm.topo[3 * sid + 1], hi = hm.topo[3 * sid + 2];
        if (lo && hi) { adj[fill[lo]++] = hi; adj[fill[hi]++] = lo; }
    }
    const int n_tiles = (e + T - 1) / T;
    std::vector<int> stamp(e, -1), ring(e, 0), slot(e, 0);
    std::vector<int> sstamp(s, -1), sloc(s, 0);
    std::vector<uint8_t> sflag(s, 0);
    std::unordered_map<uint64_t, std::vector<int>> index;
    patterns.clear();
    tile_pattern.assign(n_tiles, 0);
    tile_cbase.assign(n_tiles, 0);
    tile_sbase.assign(n_tiles, 0);
    max_ext = max_sides = max_faces = 0;
    std::vector<int> ext, sides;
    for (int t = 0; t < n_tiles; ++t) {
        const int cbase = t * T;
        const int r0_first = std::max(cbase, 1), r0_end = std::min(cbase + T, e);
        ext.clear();
        ext.push_back(0);
        stamp[0] = t; ring[0] = -1; slot[0] = 0;
        for (int g = r0_first; g < r0_end; ++g) { stamp[g] = t; ring[g] = 0; slot[g] = (int)ext.size(); ext.push_back(g); }
        int ring_begin[5];
        ring_begin[0] = 1;
        for (int r = 1; r <= rings; ++r) {
            ring_begin[r] = (int)ext.size();
            for (int i = ring_begin[r - 1]; i < ring_begin[r]; ++i) {
                int cc = ext[i];
                for (int k = aptr[cc]; k < aptr[cc + 1]; ++k) {
                    int nb = adj[k];
                    if (stamp[nb] != t) { stamp[nb] = t; ring[nb] = r; ext.push_back(nb); }
                }
            }
            std::sort(ext.begin() + ring_begin[r], ext.end());
            for (int i = ring_begin[r]; i < (int)ext.size(); ++i) slot[ext[i]] = i;
        }
        ring_begin[rings + 1] = (int)ext.size();
        // donor rings: 0..rings-1; the final q reaches faces of rings
        // 0..rings-2 (ring 1 too in the fused-CFL form, for its new depth)
        const int n_r0 = ring_begin[1] - 1, n_don = ring_begin[rings] - 1;
        const int n_r01 = rings == 3 ? ring_begin[2] - 1 : n_r0;
        const int final_ring = rings - 2;
        // local sides: faces of the donor rings (their momentum feeds the
        // donor factors)
        sides.clear();
        for (int i = 1; i <= n_don; ++i) {
            int cc = ext[i];
            for (int dd = 0; dd < 4; ++dd) {
                int p = hm.fptr[4 * cc + dd], n = hm.fcnt[4 * cc + dd];
                for (int j = 0; j < n; ++j) {
                    int sid = hm.isl[p + j];
                    if (sstamp[sid] != t) { sstamp[sid] = t; sflag[sid] = 0; sides.push_back(sid); }
                    if (ring[cc] <= final_ring) sflag[sid] |= kFinal;
                }
            }
        }
        for (int sid : sides) {
            int lo = hm.topo[3 * sid + 1], hi = hm.topo[3 * sid + 2];
            if ((lo && stamp[lo] != t) || (hi && stamp[hi] != t)) { why = "side endpoint outside the staged rings"; return 1; }
            int owner = lo ? lo : hi;
            if (owner && ring[owner] == 0 && stamp[owner] == t) sflag[sid] |= kOwned;
        }
        auto rank = [&](int sid) { return (sflag[sid] & kOwned) ? 0 : ((sflag[sid] & kFinal) ? 1 : 2); };
        std::sort(sides.begin(), sides.end(), [&](int x, int y) {
            int rx = rank(x), ry = rank(y);
            return rx != ry ? rx < ry : x < y;
        });
        int n_owned = 0, n_qf = 0;
        for (int i = 0; i < (int)sides.size(); ++i) {
            sloc[sides[i]] = i;
            n_owned += (sflag[sides[i]] & kOwned) ? 1 : 0;
            n_qf += (sflag[sides[i]] & (kOwned | kFinal)) ? 1 : 0;
        }
        if ((int)ext.size() > 65535 || (int)sides.size() > 65535) { why = "tile halo too large"; return 1; }
        int sbase = sides.empty() ? 0 : *std::min_element(sides.begin(), sides.end());
        Pattern p;
        p.counts = {(int)ext.size(), n_r0, n_r01, n_don, (int)sides.size(), n_owned, n_qf, r0_first - cbase,
                    0, 0, 0, 0};
        p.ext.resize(ext.size());
        p.ext[0] = 0;
        for (size_t i = 1; i < ext.size(); ++i) p.ext[i] = ext[i] - cbase;
        p.srel.resize(sides.size());
        p.lohi.resize(sides.size());
        for (size_t i = 0; i < sides.size(); ++i) {
            int sid = sides[i];
            p.srel[i] = sid - sbase;
            int lo = hm.topo[3 * sid + 1], hi = hm.topo[3 * sid + 2];
            p.lohi[i] = (uint32_t)slot[lo] | ((uint32_t)slot[hi] << 16);
        }
        p.fdesc.assign(n_don + 1, 0u);
        for (int i = 1; i <= n_don; ++i) {
            int cc = ext[i];
            if (p.fidx.size() > 65535) { why = "tile face table too large"; return 1; }
            uint32_t counts = 0;
            uint32_t start = (uint32_t)p.fidx.size();
            for (int dd = 0; dd < 4; ++dd) {
                int pp = hm.fptr[4 * cc + dd], n = hm.fcnt[4 * cc + dd];
                counts |= (uint32_t)n << (4 * dd);
                for (int j = 0; j < n; ++j) p.fidx.push_back((uint16_t)sloc[hm.isl[pp + j]]);
            }
            p.fdesc[i] = start | (counts << 16);
        }
        if (p.fidx.size() > 65535) { why = "tile face table too large"; return 1; }
        p.counts[8] = (int)p.fidx.size();
        max_faces = std::max(max_faces, (int)p.fidx.size());
        max_ext = std::max(max_ext, (int)ext.size());
        max_sides = std::max(max_sides, (int)sides.size());
        uint64_t hsh = pattern_hash(p);
        int found = -1;
        auto it = index.find(hsh);
        if (it != index.end())
            for (int cand : it->second)
                if (same(patterns[cand], p)) { found = cand; break; }
        if (found < 0) {
            found = (int)patterns.size();
            patterns.push_back(std::move(p));
            index[hsh].push_back(found);
        }
        tile_pattern[t] = found;
        tile_cbase[t] = cbase;
        tile_sbase[t] = sbase;
    }
    return 0;
}

// The attribute only permits dynamic shared memory up to a size; it is set
// to the planner's limit once, so that building one mesh never lowers it
// below what an already captured graph of another mesh launches with.
template <typename K>
void set_smem(K kernel, size_t bytes)
{
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(bytes > (size_t)kMaxSharedBytes ? bytes : (size_t)kMaxSharedBytes));
}

template <int NT, int CPT>
void set_smem_all(size_t bytes)
{
    set_smem(k_step_tiled<true, false, NT, CPT>, bytes);
    set_smem(k_step_tiled<false, false, NT, CPT>, bytes);
    set_smem(k_step_tiled<true, true, NT, CPT>, bytes);
    set_smem(k_step_tiled<false, true, NT, CPT>, bytes);
    set_smem(k_step_ensemble<true, NT, CPT>, bytes);
    set_smem(k_step_ensemble<false, NT, CPT>, bytes);
    if (NT == 256 && CPT == 1) {
        set_smem(k_step_tiled_gate<true, false>, bytes);
        set_smem(k_step_tiled_gate<false, false>, bytes);
        set_smem(k_step_tiled_gate<true, true>, bytes);
        set_smem(k_step_tiled_gate<false, true>, bytes);
    }
}

template <int NT, int CPT>
void launch_step(const Dev &d, size_t smem, cudaStream_t s)
{
    const int grid = d.plan.n_tiles;
    const bool hanging = d.m.hang_cells > 0;
    if (d.theta_one) {
        if (hanging) k_step_tiled<true, true, NT, CPT><<<grid, NT, smem, s>>>(d);
        else k_step_tiled<true, false, NT, CPT><<<grid, NT, smem, s>>>(d);
    } else {
        if (hanging) k_step_tiled<false, true, NT, CPT><<<grid, NT, smem, s>>>(d);
        else k_step_tiled<false, false, NT, CPT><<<grid, NT, smem, s>>>(d);
    }
}

}  // namespace

// Tangential gradients for the tiled form (reads the current-parity depth).
namespace {
__device__ __forceinline__ void pressure_slot(const Dev &d, int slot)
{
    const nhf_mesh &m = d.m;
    const float *depth = cur_depth(d, d.ctl->parity);
    int cell = m.hcells[slot];
    for (int axis = 0; axis < 2; ++axis) {
        if (m.axes[2 * slot + axis] != 1) continue;
        float value = 0.0f;
        if (depth[cell] > d.min_h) {
            float dv[2], xv[2];
            int ok[2];
            for (int side_of = 0; side_of < 2; ++side_of) {
                int direction = axis == 1 ? 2 + side_of : side_of;
                float val = 0.0f, distance = 0.0f, total = 0.0f;
                int usable = 1;
                float eta = m.bed[cell] + depth[cell];
                int start = m.face_ptr[4 * cell + direction], count = m.face_count[4 * cell + direction];
                for (int j = 0; j < count; ++j) {
                    int side = m.isl_data[start + j];
                    int other = m.topology[3 * side + 1] + m.topology[3 * side + 2] - cell;
                    if (other == 0 || depth[other] <= d.min_h) {
                        usable = 0;
                    } else {
                        float weight = m.length[side];
                        val += weight * ((m.bed[other] + depth[other]) - eta);
                        float delta = axis == 1 ? m.y[other] - m.y[cell] : m.x[other] - m.x[cell];
                        distance += weight * delta;
                        total += weight;
                    }
                }
                if (total > 0.0f) { val /= total; distance /= total; }
                else usable = 0;
                dv[side_of] = val; xv[side_of] = distance; ok[side_of] = usable;
            }
            if (ok[0] && ok[1]) value = (dv[1] - dv[0]) / (xv[1] - xv[0]);
            else if (ok[0]) value = dv[0] / xv[0];
            else if (ok[1]) value = dv[1] / xv[1];
        }
        d.gradients[2 * slot + axis] = value;
    }
}

__global__ void k_pressure_tiled(const __grid_constant__ Dev d)
{
    if (!d.ctl->active) return;
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot < d.m.hang_cells) pressure_slot(d, slot);
}

// length-weighted face discharge for theta < 1 (solver_compact.py:118-132)
__device__ __forceinline__ void face_qn_cell(const Dev &d, int ei)
{
    const nhf_mesh &m = d.m;
    const float *q = cur_q(d, d.ctl->parity);
    for (int dd = 0; dd < 4; ++dd) {
        int start = m.face_ptr[4 * ei + dd], count = m.face_count[4 * ei + dd];
        float result = 0.0f;
        if (count == 1) {
            result = q[m.isl_data[start]];
        } else if (count > 1) {
            float total = 0.0f, width = 0.0f;
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

__global__ void k_face_qn_tiled(const __grid_constant__ Dev d)
{
    if (!d.ctl->active) return;
    int ei = blockIdx.x * blockDim.x + threadIdx.x;
    if (ei < d.m.e_num) face_qn_cell(d, ei);
}

// ------------------------------------------------------- ensemble kernels

// clock.begin for every member (clock.py:75-92) and the preparation of its
// first step; words[4 * member] = next_hi, next_lo, origin_hi, origin_lo.
__global__ void k_ens_begin(const Dev *devs, const uint32_t *words)
{
    const Dev &d = devs[blockIdx.x];
    Ctl *c = d.ctl;
    const int t = threadIdx.x;
    const uint32_t *w = words + 4 * blockIdx.x;
    if (t == 0) {
        c->next[0] = w[0]; c->next[1] = w[1];
        c->origin[0] = w[2]; c->origin[1] = w[3];
        c->slot = 0;
    }
    for (int i = t; i < NHF_MAX_BATCH * NHF_TRACE_COLS; i += blockDim.x) c->trace[i] = 0u;
    __syncthreads();
    if (t == 0) prepare_step(d, c, d.m.depth, d.m.q);
}

__global__ void k_ens_batch_start(const Dev *devs, const int2 *items)
{
    const int2 w = items[blockIdx.x];
    const Dev &d = devs[w.x];
    const int end = min(d.m.e_num, (w.y + 1) * kEnsChunk);
    for (int i = w.y * kEnsChunk + threadIdx.x; i < end; i += blockDim.x) d.rain_time_b[i] = d.m.rain_time[i];
}

__global__ void k_ens_pressure(const Dev *devs, const int2 *items)
{
    const int2 w = items[blockIdx.x];
    const Dev &d = devs[w.x];
    if (!d.ctl->active) return;
    const int end = min(d.m.hang_cells, (w.y + 1) * kEnsChunk);
    for (int i = w.y * kEnsChunk + threadIdx.x; i < end; i += blockDim.x) pressure_slot(d, i);
}

__global__ void k_ens_face_qn(const Dev *devs, const int2 *items)
{
    const int2 w = items[blockIdx.x];
    const Dev &d = devs[w.x];
    if (!d.ctl->active) return;
    const int end = min(d.m.e_num, (w.y + 1) * kEnsChunk);
    for (int i = w.y * kEnsChunk + threadIdx.x; i < end; i += blockDim.x) face_qn_cell(d, i);
}

// CFL pass of every member: items are (member, chunk of kEnsChunk sides);
// a member's last chunk block prepares that member's next step. Members with
// a fused-CFL plan did both in their step and are skipped.
__global__ void __launch_bounds__(256) k_ens_cfl(const Dev *devs, const int2 *items)
{
    const int2 w = items[blockIdx.x];
    const Dev &d = devs[w.x];
    if (!d.plan.split) return;
    const int n = d.m.e_num > d.m.s_num ? d.m.e_num : d.m.s_num;
    const unsigned chunks = (unsigned)((n + kEnsChunk - 1) / kEnsChunk);
    const int first = max(1, w.y * kEnsChunk), end = min(d.m.s_num, (w.y + 1) * kEnsChunk);
    cfl_pass(d, first, end, (int)blockDim.x, chunks);
}

// Batch end, part 1: the current state back into the caller's buffers.
__global__ void k_ens_copy_back(const Dev *devs, const int2 *items)
{
    const int2 w = items[blockIdx.x];
    const Dev &d = devs[w.x];
    if (!d.ctl->parity) return;
    const int first = w.y * kEnsChunk;
    const int end_e = min(d.m.e_num, first + kEnsChunk), end_s = min(d.m.s_num, first + kEnsChunk);
    for (int i = first + threadIdx.x; i < end_e; i += blockDim.x) {
        d.m.depth[i] = d.depth_b[i];
        d.m.rain_time[i] = d.rain_time_b[i];
    }
    for (int i = first + threadIdx.x; i < end_s; i += blockDim.x) d.m.q[i] = d.q_b[i];
}

// Batch end, part 2: u, v from the caller's buffers.
__global__ void k_ens_velocity(const Dev *devs, const int2 *items)
{
    const int2 w = items[blockIdx.x];
    const Dev &d = devs[w.x];
    const int end = min(d.m.e_num, (w.y + 1) * kEnsChunk);
    for (int i = max(1, w.y * kEnsChunk) + threadIdx.x; i < end; i += blockDim.x) velocity_cell(d, i);
}

// Batch end, part 3: every member's trace rows into one buffer; the state
// now lives in the caller's buffers again.
__global__ void k_ens_finish(const Dev *devs, uint32_t *trace, int batch)
{
    const Dev &d = devs[blockIdx.x];
    Ctl *c = d.ctl;
    uint32_t *out = trace + (size_t)blockIdx.x * batch * NHF_TRACE_COLS;
    for (int i = threadIdx.x; i < batch * NHF_TRACE_COLS; i += blockDim.x) out[i] = c->trace[i];
    if (threadIdx.x == 0) c->parity = 0;
}
}  // namespace

int tiled_build(const nhf_mesh &m, cudaStream_t s, TiledBuild *out, char *why, size_t why_len, int tile_request,
                int cfl_mode)
{
    std::string reason;
    auto bad = [&](const std::string &r) {
        snprintf(why, why_len, "%s", r.c_str());
        return 1;
    };
    if (m.e_num < 2) return bad("mesh has no cells");
    HostMesh hm;
    if (copy_back(m, s, hm)) return bad("copying the mesh tables to the host failed");
    if (!consistent(hm, reason)) return bad(reason);
    std::vector<Pattern> patterns;
    std::vector<int32_t> tp, tc, ts;
    int max_ext = 0, max_sides = 0, max_faces = 0, tile = 0;
    size_t smem = 0;
    // Small meshes take small tiles so that every SM gets work.
    // Multi-resolution meshes (irregular halos, more work per cell) run best
    // with 256-cell tiles and five blocks per SM; on uniform meshes large
    // tiles amortise the halo.
    std::vector<int> sizes = {1024, 512, 256};
    if (m.e_num < 148 * 2 * 1024 || m.hang_cells > 0) sizes = {256, 512, 1024};
    else if (m.e_num < 148 * 4 * 1024) sizes = {512, 256};
    if (tile_request) {
        if (tile_request != 256 && tile_request != 512 && tile_request != 1024)
            return bad("tile size must be 256, 512 or 1024");
        sizes = {tile_request};
    }
    bool split = false;
    for (int T : sizes) {
        // The separate CFL pass pays one launch per step for less halo work
        // (no ring 3, no ring-1 depth recompute): worth it from two waves of
        // resident blocks on.
        const int resident = 148 * (T == 256 ? kMinBlocks<256> : kMinBlocks<512>);
        const int n_tiles = (m.e_num + T - 1) / T;
        split = cfl_mode == 2 || (cfl_mode == 0 && n_tiles >= 2 * resident);
        if (plan_tiles(hm, T, patterns, tp, tc, ts, max_ext, max_sides, max_faces, split ? 2 : 3, reason))
            return bad(reason);
        // The budget reduction stages one term of every thread (NT doubles)
        // in the 24 * max_ext bytes of shared arrays that are dead after the
        // depth update; meshes smaller than a tile need the padding.
        const int nt = T == 256 ? 256 : 512;
        if (24 * max_ext < 8 * nt) max_ext = (8 * nt + 23) / 24;
        smem = (size_t)max_ext * 32 + (size_t)max_sides * 16 + (size_t)max_faces * 2 + 16;
        if (smem <= (size_t)kMaxSharedBytes) { tile = T; break; }
    }
    if (!tile) return bad("tile halos exceed shared memory (cell numbering is not spatially coherent)");
    // flatten patterns
    std::vector<int32_t> counts, offsets, ext, srel;
    std::vector<uint32_t> lohi, fdesc;
    std::vector<uint16_t> fidx;
    for (const Pattern &p : patterns) {
        counts.insert(counts.end(), p.counts.begin(), p.counts.end());
        offsets.push_back((int32_t)ext.size());
        offsets.push_back((int32_t)srel.size());
        offsets.push_back((int32_t)fdesc.size());
        offsets.push_back((int32_t)fidx.size());
        ext.insert(ext.end(), p.ext.begin(), p.ext.end());
        srel.insert(srel.end(), p.srel.begin(), p.srel.end());
        lohi.insert(lohi.end(), p.lohi.begin(), p.lohi.end());
        fdesc.insert(fdesc.end(), p.fdesc.begin(), p.fdesc.end());
        fidx.insert(fidx.end(), p.fidx.begin(), p.fidx.end());
        if (fidx.size() & 1) fidx.push_back(0);  // the kernel copies face indices in pairs
    }
    if (fidx.empty()) { fidx.push_back(0); fidx.push_back(0); }
    // per-tile header: the pattern's counts and offsets with the tile's bases
    std::vector<int32_t> head((size_t)tp.size() * 16, 0);
    for (size_t t = 0; t < tp.size(); ++t) {
        const int32_t *cnt = counts.data() + 12 * (size_t)tp[t];
        const int32_t *off = offsets.data() + 4 * (size_t)tp[t];
        int32_t *h = head.data() + 16 * t;
        for (int k = 0; k < 9; ++k) h[k] = cnt[k];
        h[9] = tc[t]; h[10] = ts[t];
        h[11] = off[0]; h[12] = off[1]; h[13] = off[2]; h[14] = off[3];
    }
    if (srel.empty()) { srel.push_back(0); lohi.push_back(0); }
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    size_t o_ext = take(ext.size() * 4);
    size_t o_srel = take(srel.size() * 4), o_lohi = take(lohi.size() * 4), o_fd = take(fdesc.size() * 4);
    size_t o_fi = take(fidx.size() * 2);
    size_t o_hd = take(head.size() * 4);
    void *mem = nullptr;
    if (cudaMalloc(&mem, off) != cudaSuccess) return bad("allocating the tile plan failed");
    char *b = (char *)mem;
    auto up = [&](size_t o, const void *src, size_t n) {
        return cudaMemcpyAsync(b + o, src, n, cudaMemcpyHostToDevice, s) == cudaSuccess;
    };
    bool ok = up(o_ext, ext.data(), ext.size() * 4) &&
              up(o_srel, srel.data(), srel.size() * 4) && up(o_lohi, lohi.data(), lohi.size() * 4) &&
              up(o_fd, fdesc.data(), fdesc.size() * 4) && up(o_fi, fidx.data(), fidx.size() * 2) &&
              up(o_hd, head.data(), head.size() * 4) &&
              cudaStreamSynchronize(s) == cudaSuccess;
    if (!ok) { cudaFree(mem); return bad("uploading the tile plan failed"); }
    TilePlan &P = out->plan;
    P.n_tiles = (int32_t)tp.size();
    P.tile = tile;
    P.max_ext = max_ext;
    P.max_sides = max_sides;
    P.cells_per_thread = tile == 1024 ? 2 : 1;
    P.split = split ? 1 : 0;
    P.tile_head = (const int4 *)(b + o_hd);
    P.ext_rel = (const int32_t *)(b + o_ext);
    P.side_rel = (const int32_t *)(b + o_srel);
    P.side_lohi = (const uint32_t *)(b + o_lohi);
    P.face_desc = (const uint32_t *)(b + o_fd);
    P.face_idx = (const uint16_t *)(b + o_fi);
    out->device_memory = mem;
    out->shared_bytes = smem;
    out->patterns = (int)patterns.size();
    if (tile == 1024) set_smem_all<512, 2>(smem);
    else if (tile == 512) set_smem_all<512, 1>(smem);
    else set_smem_all<256, 1>(smem);
    return 0;
}

void tiled_enqueue_step(const Dev &d, const TiledBuild &b, cudaStream_t s, const GateDev *gate)
{
    const nhf_mesh &m = d.m;
    if (m.hang_cells > 0) k_pressure_tiled<<<(m.hang_cells + 255) / 256, 256, 0, s>>>(d);
    if (!d.theta_one) k_face_qn_tiled<<<(m.e_num + 255) / 256, 256, 0, s>>>(d);
    if (gate) {  // 256-cell tiles, split plan (checked when the controller is attached)
        const int grid = d.plan.n_tiles;
        const size_t smem = b.shared_bytes;
        const bool hanging = m.hang_cells > 0;
        if (d.theta_one) {
            if (hanging) k_step_tiled_gate<true, true><<<grid, 256, smem, s>>>(d, *gate);
            else k_step_tiled_gate<true, false><<<grid, 256, smem, s>>>(d, *gate);
        } else {
            if (hanging) k_step_tiled_gate<false, true><<<grid, 256, smem, s>>>(d, *gate);
            else k_step_tiled_gate<false, false><<<grid, 256, smem, s>>>(d, *gate);
        }
        return;  // the caller adds the controller's passes, then the CFL pass
    }
    switch (d.plan.tile) {
    case 1024: launch_step<512, 2>(d, b.shared_bytes, s); break;
    case 512: launch_step<512, 1>(d, b.shared_bytes, s); break;
    default: launch_step<256, 1>(d, b.shared_bytes, s); break;
    }
    tiled_enqueue_cfl(d, b, s);
}

void tiled_enqueue_cfl(const Dev &d, const TiledBuild &b, cudaStream_t s, const GateDev *gate)
{
    if (b.plan.split) {
        int gc = (d.m.s_num + 255) / 256;
        if (gc > 148 * 8) gc = 148 * 8;
        if (gate) k_cfl_tiled_gate<<<gc, 256, 0, s>>>(d, *gate);
        else k_cfl_tiled<<<gc, 256, 0, s>>>(d);
    }
}

void tiled_enqueue_batch_start(const Dev &d, cudaStream_t s)
{
    int grid = (d.m.e_num + 255) / 256;
    if (grid > 148 * 16) grid = 148 * 16;
    k_batch_start<<<grid, 256, 0, s>>>(d);
}

template <int NT, int CPT>
int ensemble_occupancy(int theta_one, size_t smem)
{
    int n = 0;
    if (theta_one) cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step_ensemble<true, NT, CPT>, NT, smem);
    else cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_step_ensemble<false, NT, CPT>, NT, smem);
    return n;
}

int ensemble_blocks_per_sm(int tile, int theta_one, size_t smem)
{
    switch (tile) {
    case 1024: set_smem_all<512, 2>(smem); return ensemble_occupancy<512, 2>(theta_one, smem);
    case 512: set_smem_all<512, 1>(smem); return ensemble_occupancy<512, 1>(theta_one, smem);
    default: set_smem_all<256, 1>(smem); return ensemble_occupancy<256, 1>(theta_one, smem);
    }
}

void ensemble_enqueue_begin(const EnsembleLaunch &e, cudaStream_t s)
{
    k_ens_begin<<<e.members, 256, 0, s>>>(e.devs, e.words);
}

void ensemble_enqueue_batch_start(const EnsembleLaunch &e, cudaStream_t s)
{
    if (e.n_cell) k_ens_batch_start<<<e.n_cell, 256, 0, s>>>(e.devs, e.cell_items);
}

template <int NT, int CPT>
void ensemble_launch(const EnsembleLaunch &e, cudaStream_t s)
{
    if (e.theta_one) k_step_ensemble<true, NT, CPT><<<e.grid, NT, e.smem, s>>>(e.devs, e.step_items, e.n_step);
    else k_step_ensemble<false, NT, CPT><<<e.grid, NT, e.smem, s>>>(e.devs, e.step_items, e.n_step);
}

void ensemble_enqueue_step(const EnsembleLaunch &e, cudaStream_t s)
{
    if (e.n_hang) k_ens_pressure<<<e.n_hang, 256, 0, s>>>(e.devs, e.hang_items);
    if (!e.theta_one && e.n_qn) k_ens_face_qn<<<e.n_qn, 256, 0, s>>>(e.devs, e.qn_items);
    switch (e.tile) {
    case 1024: ensemble_launch<512, 2>(e, s); break;
    case 512: ensemble_launch<512, 1>(e, s); break;
    default: ensemble_launch<256, 1>(e, s); break;
    }
    k_ens_cfl<<<e.n_cell, 256, 0, s>>>(e.devs, e.cell_items);
}

void ensemble_enqueue_batch_end(const EnsembleLaunch &e, cudaStream_t s)
{
    if (e.n_cell) {
        k_ens_copy_back<<<e.n_cell, 256, 0, s>>>(e.devs, e.cell_items);
        k_ens_velocity<<<e.n_cell, 256, 0, s>>>(e.devs, e.cell_items);
    }
    k_ens_finish<<<e.members, 256, 0, s>>>(e.devs, e.trace, e.batch);
}

void tiled_enqueue_velocity(const Dev &d, cudaStream_t s)
{
    int grid = (d.m.e_num + 255) / 256;
    if (grid > 148 * 16) grid = 148 * 16;
    k_velocity<<<grid, 256, 0, s>>>(d);
}

void tiled_enqueue_batch_end(const Dev &d, cudaStream_t s)
{
    int n = d.m.e_num > d.m.s_num ? d.m.e_num : d.m.s_num;
    int grid = (n + 255) / 256;
    if (grid > 148 * 16) grid = 148 * 16;
    k_batch_end<<<grid, 256, 0, s>>>(d);
    k_velocity<<<grid, 256, 0, s>>>(d);
}

}  // namespace nhf
