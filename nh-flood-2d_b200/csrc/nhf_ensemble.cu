// Ensemble form of the C ABI: many member meshes advance together, each with
// its own clock, dt (its own CFL candidate), limiter statistics, budget
// partials and extrema, exactly as a single-mesh batch does
// (solver_compact.py:918-985 per member). Two schedules:
//  - one ensemble graph (members on the fused tiled step with one tile size
//    and batch size): the members' begin words in, for every slot one
//    pre-pass launch per hanging/theta need and ONE fused step launch over
//    the tiles of all members, the batch epilogue, every member's trace out;
//  - member graphs (grid_blocks = -2): every member runs its own batch graph
//    (its own step form, tile size and CFL placement) on its own stream, all
//    of them launched together, so that small members fill the GPU beside
//    large ones while each keeps the single-mesh kernels.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "nhf_common.cuh"
#include "nhf_handle.cuh"

using namespace nhf;

struct nhf_ensemble {
    std::vector<nhf_handle *> members;
    std::vector<cudaStream_t> streams;  // distinct caller streams of the ensemble and its members
    cudaStream_t user = nullptr, s = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    EnsembleLaunch launch{};
    void *device_memory = nullptr;
    uint32_t *h_words = nullptr;  // pinned [members][4]
    uint32_t *h_trace = nullptr;  // pinned [members][batch][NHF_TRACE_COLS]
    cudaGraph_t graph_def = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool in_flight = false;
    bool member_graphs = false;             // grid_blocks = -2
    std::vector<cudaEvent_t> member_done;   // member-graph schedule: one per member
    std::string err;
};

namespace {

std::string g_ens_create_error;

int efail(nhf_ensemble *e, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (e) e->err = buf; else g_ens_create_error = buf;
    return code;
}

#define ECK(e, call)                                                                        \
    do {                                                                                    \
        cudaError_t e_ = (call);                                                            \
        if (e_ != cudaSuccess)                                                              \
            return efail((e), NHF_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_));   \
    } while (0)

int build_graph(nhf_ensemble *e)
{
    const EnsembleLaunch &L = e->launch;
    ECK(e, cudaStreamBeginCapture(e->s, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync((void *)L.words, e->h_words, sizeof(uint32_t) * 4 * L.members, cudaMemcpyHostToDevice, e->s);
    ensemble_enqueue_begin(L, e->s);
    ensemble_enqueue_batch_start(L, e->s);
    for (int i = 0; i < L.batch; ++i) ensemble_enqueue_step(L, e->s);
    ensemble_enqueue_batch_end(L, e->s);
    cudaMemcpyAsync(e->h_trace, L.trace, sizeof(uint32_t) * NHF_TRACE_COLS * L.batch * L.members,
                    cudaMemcpyDeviceToHost, e->s);
    cudaGraph_t g = nullptr;
    cudaError_t err = cudaStreamEndCapture(e->s, &g);
    if (err != cudaSuccess) return efail(e, NHF_ECUDA, "ensemble graph capture failed: %s", cudaGetErrorString(err));
    err = cudaGraphInstantiate(&e->graph, g, 0);
    if (err != cudaSuccess) {
        cudaGraphDestroy(g);
        return efail(e, NHF_ECUDA, "ensemble graph instantiate failed: %s", cudaGetErrorString(err));
    }
    e->graph_def = g;
    return NHF_OK;
}

void append_chunks(std::vector<int2> &items, int member, int count)
{
    for (int c = 0; c * kEnsChunk < count; ++c) items.push_back(make_int2(member, c));
}

// The member-graph schedule: members may differ in step form and tile size,
// not in batch size; their batch graphs are built here.
int create_member_graphs(nhf_handle *const *members, int32_t n, void *stream, nhf_ensemble **out)
{
    const nhf_handle *h0 = members[0];
    for (int i = 0; i < n; ++i) {
        const nhf_handle *h = members[i];
        if (!h) return efail(nullptr, NHF_EINVAL, "member %d is null", i);
        if (h->p.batch_size != h0->p.batch_size) return efail(nullptr, NHF_EINVAL, "member %d has another batch size", i);
        for (int j = 0; j < i; ++j)
            if (members[j] == h) return efail(nullptr, NHF_EINVAL, "member %d is listed twice", i);
    }
    nhf_ensemble *e = new nhf_ensemble();
    e->member_graphs = true;
    e->members.assign(members, members + n);
    e->user = (cudaStream_t)stream;
    e->streams.push_back(e->user);
    for (int i = 0; i < n; ++i) {
        bool seen = false;
        for (cudaStream_t st : e->streams) seen = seen || st == members[i]->user;
        if (!seen) e->streams.push_back(members[i]->user);
    }
    int rc = NHF_OK;
    auto bad = [&](int code, const char *what, cudaError_t err) {
        rc = efail(nullptr, code, "%s failed: %s", what, cudaGetErrorString(err));
        nhf_ensemble_destroy(e);
        return rc;
    };
    cudaError_t err;
    if ((err = cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking)) != cudaSuccess) return bad(NHF_ECUDA, "cudaStreamCreateWithFlags", err);
    if ((err = cudaEventCreateWithFlags(&e->ev_in, cudaEventDisableTiming)) != cudaSuccess) return bad(NHF_ECUDA, "cudaEventCreateWithFlags", err);
    if ((err = cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming)) != cudaSuccess) return bad(NHF_ECUDA, "cudaEventCreateWithFlags", err);
    e->member_done.assign(n, nullptr);
    int tiles = 0;
    for (int i = 0; i < n; ++i) {
        if ((err = cudaEventCreateWithFlags(&e->member_done[i], cudaEventDisableTiming)) != cudaSuccess)
            return bad(NHF_ECUDA, "cudaEventCreateWithFlags", err);
        int mrc = member_graph_prepare(members[i]);
        if (mrc) {
            rc = efail(nullptr, mrc, "member %d: %s", i, members[i]->err.c_str());
            nhf_ensemble_destroy(e);
            return rc;
        }
        tiles += members[i]->tiled ? members[i]->tb.plan.n_tiles : 0;
    }
    EnsembleLaunch &L = e->launch;
    L.members = n;
    L.batch = h0->p.batch_size;
    L.tile = 0;     // per member
    L.grid = -2;
    L.n_step = tiles;
    *out = e;
    return NHF_OK;
}

}  // namespace

extern "C" {

const char *nhf_ensemble_last_error(const nhf_ensemble *e) { return e ? e->err.c_str() : g_ens_create_error.c_str(); }

int nhf_ensemble_destroy(nhf_ensemble *e)
{
    if (!e) return NHF_OK;
    if (e->s) cudaStreamSynchronize(e->s);
    if (e->graph) cudaGraphExecDestroy(e->graph);
    if (e->graph_def) cudaGraphDestroy(e->graph_def);
    if (e->device_memory) cudaFree(e->device_memory);
    if (e->h_words) cudaFreeHost(e->h_words);
    if (e->h_trace) cudaFreeHost(e->h_trace);
    if (e->ev_in) cudaEventDestroy(e->ev_in);
    if (e->ev_out) cudaEventDestroy(e->ev_out);
    for (cudaEvent_t ev : e->member_done) cudaEventDestroy(ev);
    if (e->s) cudaStreamDestroy(e->s);
    delete e;
    return NHF_OK;
}

int nhf_ensemble_create(nhf_handle *const *members, int32_t n, int32_t grid_blocks, void *stream,
                        nhf_ensemble **out)
{
    if (!members || n < 1 || !out) return efail(nullptr, NHF_EINVAL, "null argument or no members");
    *out = nullptr;
    const nhf_handle *h0 = members[0];
    if (!h0) return efail(nullptr, NHF_EINVAL, "member 0 is null");
    if (grid_blocks < -2) return efail(nullptr, NHF_EINVAL, "grid_blocks must be -2, -1, 0 or positive");
    if (grid_blocks == -2) return create_member_graphs(members, n, stream, out);
    const int tile = h0->tb.plan.tile;
    for (int i = 0; i < n; ++i) {
        const nhf_handle *h = members[i];
        if (!h) return efail(nullptr, NHF_EINVAL, "member %d is null", i);
        if (!h->tiled) return efail(nullptr, NHF_EINVAL, "member %d is not on the fused tiled step (%s)", i, h->path.c_str());
        // the one-launch step has no gate passes: a gated member runs its own
        // batch graph in the member-graph schedule
        if (h->gate_on)
            return efail(nullptr, NHF_EINVAL, "member %d has a gate controller; use the member-graph schedule", i);
        if (h->tb.plan.tile != tile) return efail(nullptr, NHF_EINVAL, "member %d has tile %d, member 0 has %d", i, h->tb.plan.tile, tile);
        if (h->p.batch_size != h0->p.batch_size) return efail(nullptr, NHF_EINVAL, "member %d has another batch size", i);
        if (h->dev.theta_one != h0->dev.theta_one) return efail(nullptr, NHF_EINVAL, "members mix theta = 1 and theta < 1");
        for (int j = 0; j < i; ++j)
            if (members[j] == h) return efail(nullptr, NHF_EINVAL, "member %d is listed twice", i);
    }
    nhf_ensemble *e = new nhf_ensemble();
    e->members.assign(members, members + n);
    e->user = (cudaStream_t)stream;
    e->streams.push_back(e->user);
    for (int i = 0; i < n; ++i) {
        bool seen = false;
        for (cudaStream_t st : e->streams) seen = seen || st == members[i]->user;
        if (!seen) e->streams.push_back(members[i]->user);
    }
    int rc;
#define ECKC(call)                                                                                  \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) {                                                                    \
            rc = efail(nullptr, NHF_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_));         \
            nhf_ensemble_destroy(e);                                                                \
            return rc;                                                                              \
        }                                                                                           \
    } while (0)
    ECKC(cudaStreamCreateWithFlags(&e->s, cudaStreamNonBlocking));
    ECKC(cudaEventCreateWithFlags(&e->ev_in, cudaEventDisableTiming));
    ECKC(cudaEventCreateWithFlags(&e->ev_out, cudaEventDisableTiming));
    // work lists: tiles of all members, then chunks for the side passes
    std::vector<int2> steps, hang, qn, cells;
    size_t smem = 0;
    for (int i = 0; i < n; ++i) {
        const nhf_handle *h = members[i];
        for (int t = 0; t < h->tb.plan.n_tiles; ++t) steps.push_back(make_int2(i, t));
        if (h->m.hang_cells > 0) append_chunks(hang, i, h->m.hang_cells);
        if (!h->dev.theta_one) append_chunks(qn, i, h->m.e_num);
        append_chunks(cells, i, h->m.e_num > h->m.s_num ? h->m.e_num : h->m.s_num);
        smem = h->tb.shared_bytes > smem ? h->tb.shared_bytes : smem;
    }
    std::vector<Dev> devs(n);
    for (int i = 0; i < n; ++i) devs[i] = members[i]->dev;
    const int batch = h0->p.batch_size;
    size_t off = 0;
    auto take = [&](size_t bytes) { size_t o = off; off += (bytes + 255) & ~size_t(255); return o; };
    size_t o_dev = take(sizeof(Dev) * n), o_st = take(sizeof(int2) * steps.size()),
           o_hg = take(sizeof(int2) * (hang.size() + 1)), o_qn = take(sizeof(int2) * (qn.size() + 1)),
           o_ce = take(sizeof(int2) * cells.size()), o_w = take(sizeof(uint32_t) * 4 * n),
           o_tr = take(sizeof(uint32_t) * NHF_TRACE_COLS * batch * (size_t)n);
    ECKC(cudaMalloc(&e->device_memory, off));
    char *b = (char *)e->device_memory;
    ECKC(cudaMemcpyAsync(b + o_dev, devs.data(), sizeof(Dev) * n, cudaMemcpyHostToDevice, e->s));
    ECKC(cudaMemcpyAsync(b + o_st, steps.data(), sizeof(int2) * steps.size(), cudaMemcpyHostToDevice, e->s));
    if (!hang.empty()) ECKC(cudaMemcpyAsync(b + o_hg, hang.data(), sizeof(int2) * hang.size(), cudaMemcpyHostToDevice, e->s));
    if (!qn.empty()) ECKC(cudaMemcpyAsync(b + o_qn, qn.data(), sizeof(int2) * qn.size(), cudaMemcpyHostToDevice, e->s));
    ECKC(cudaMemcpyAsync(b + o_ce, cells.data(), sizeof(int2) * cells.size(), cudaMemcpyHostToDevice, e->s));
    ECKC(cudaMallocHost(&e->h_words, sizeof(uint32_t) * 4 * n));
    ECKC(cudaMallocHost(&e->h_trace, sizeof(uint32_t) * NHF_TRACE_COLS * batch * (size_t)n));
    ECKC(cudaStreamSynchronize(e->s));
    EnsembleLaunch &L = e->launch;
    L.devs = (const Dev *)(b + o_dev);
    L.members = n;
    L.batch = batch;
    L.tile = tile;
    L.theta_one = h0->dev.theta_one;
    L.smem = smem;
    L.step_items = (const int2 *)(b + o_st); L.n_step = (int)steps.size();
    L.hang_items = (const int2 *)(b + o_hg); L.n_hang = (int)hang.size();
    L.qn_items = (const int2 *)(b + o_qn); L.n_qn = (int)qn.size();
    L.cell_items = (const int2 *)(b + o_ce); L.n_cell = (int)cells.size();
    L.words = (const uint32_t *)(b + o_w);
    L.trace = (uint32_t *)(b + o_tr);
    // grid: 0 = persistent (resident blocks per SM x SMs), -1 = a block per tile
    int per_sm = ensemble_blocks_per_sm(tile, L.theta_one, smem);
    int sms = 0, dev = 0;
    ECKC(cudaGetDevice(&dev));
    ECKC(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    if (per_sm < 1) {
        rc = efail(nullptr, NHF_ECUDA, "the ensemble step kernel does not fit an SM (tile %d, %zu B shared)", tile, smem);
        nhf_ensemble_destroy(e);
        return rc;
    }
    int grid = grid_blocks > 0 ? grid_blocks : grid_blocks < 0 ? L.n_step : per_sm * sms;
    if (grid > L.n_step) grid = L.n_step;
    L.grid = grid;
#undef ECKC
    *out = e;
    return NHF_OK;
}

int nhf_ensemble_info(const nhf_ensemble *e, int32_t info[6])
{
    if (!e || !info) return NHF_EINVAL;
    const EnsembleLaunch &L = e->launch;
    info[0] = L.members; info[1] = L.tile; info[2] = L.grid; info[3] = L.n_step; info[4] = L.batch;
    info[5] = (int32_t)L.smem;
    return NHF_OK;
}

void *nhf_ensemble_stream(const nhf_ensemble *e) { return e ? (void *)e->s : nullptr; }

int nhf_ensemble_run_batch_async(nhf_ensemble *e, const uint32_t *targets, const uint32_t *origins)
{
    if (!e || !targets || !origins) return NHF_EINVAL;
    // the pinned words of the previous batch may still be in use
    if (e->in_flight) ECK(e, cudaStreamSynchronize(e->s));
    const int n = e->launch.members;
    if (e->member_graphs) {
        // after all work queued on the caller streams, every member's own
        // batch graph on its own stream; the ensemble stream joins them
        for (cudaStream_t st : e->streams) {
            ECK(e, cudaEventRecord(e->ev_in, st));
            ECK(e, cudaStreamWaitEvent(e->s, e->ev_in, 0));
        }
        ECK(e, cudaEventRecord(e->ev_in, e->s));
        for (int i = 0; i < n; ++i) {
            int rc = member_graph_launch(e->members[i], targets + 2 * i, origins + 2 * i, e->ev_in, e->member_done[i]);
            if (rc) return efail(e, rc, "member %d: %s", i, e->members[i]->err.c_str());
        }
        for (int i = 0; i < n; ++i) ECK(e, cudaStreamWaitEvent(e->s, e->member_done[i], 0));
        e->in_flight = true;
        ECK(e, cudaGetLastError());
        ECK(e, cudaEventRecord(e->ev_out, e->s));
        for (cudaStream_t st : e->streams) ECK(e, cudaStreamWaitEvent(st, e->ev_out, 0));
        return NHF_OK;
    }
    for (int i = 0; i < n; ++i)
        if (e->members[i]->gate_on)
            return efail(e, NHF_ESTATE, "member %d has a gate controller attached after the one-launch ensemble was made", i);
    for (int i = 0; i < n; ++i) {
        e->h_words[4 * i] = targets[2 * i];
        e->h_words[4 * i + 1] = targets[2 * i + 1];
        e->h_words[4 * i + 2] = origins[2 * i];
        e->h_words[4 * i + 3] = origins[2 * i + 1];
    }
    // after all work queued on the caller streams of the ensemble and of its members
    for (cudaStream_t st : e->streams) {
        ECK(e, cudaEventRecord(e->ev_in, st));
        ECK(e, cudaStreamWaitEvent(e->s, e->ev_in, 0));
    }
    if (!e->graph) { int rc = build_graph(e); if (rc) return rc; }
    ECK(e, cudaGraphLaunch(e->graph, e->s));
    e->in_flight = true;
    ECK(e, cudaGetLastError());
    ECK(e, cudaEventRecord(e->ev_out, e->s));
    for (cudaStream_t st : e->streams) ECK(e, cudaStreamWaitEvent(st, e->ev_out, 0));
    return NHF_OK;
}

int nhf_ensemble_read_trace(nhf_ensemble *e, uint32_t *trace)
{
    if (!e || !trace) return NHF_EINVAL;
    ECK(e, cudaStreamSynchronize(e->s));
    e->in_flight = false;
    if (e->member_graphs) {
        const size_t rows = (size_t)NHF_TRACE_COLS * e->launch.batch;
        for (int i = 0; i < e->launch.members; ++i)
            memcpy(trace + rows * i, e->members[i]->h_trace, sizeof(uint32_t) * rows);
        return NHF_OK;
    }
    memcpy(trace, e->h_trace, sizeof(uint32_t) * NHF_TRACE_COLS * e->launch.batch * (size_t)e->launch.members);
    return NHF_OK;
}

int nhf_ensemble_run_batch(nhf_ensemble *e, const uint32_t *targets, const uint32_t *origins, uint32_t *trace)
{
    int rc = nhf_ensemble_run_batch_async(e, targets, origins);
    if (rc) return rc;
    return nhf_ensemble_read_trace(e, trace);
}

}  // extern "C"
