// The handle behind the C ABI (one mesh, its scratch, streams and graph).
// Shared by the single-mesh entry points and the ensemble form.
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "nhf_common.cuh"

struct nhf_handle {
    nhf_mesh m{};
    nhf_params p{};
    nhf::Dev dev{};
    cudaStream_t user = nullptr, s = nullptr;
    cudaEvent_t ev_in = nullptr, ev_out = nullptr;
    nhf::Ctl *ctl = nullptr;
    void *scratch = nullptr;
    uint32_t *h_begin = nullptr;  // pinned {next, origin}
    uint32_t *d_begin = nullptr;
    uint32_t *h_trace = nullptr;  // pinned
    nhf::real *h_small = nullptr; // pinned staging for forcing / scalars
    double *h_acc = nullptr;      // pinned budget staging
    int32_t *d_ids = nullptr;
    nhf::real *d_samples = nullptr;
    int ids_cap = 0;
    cudaGraph_t graph_def = nullptr;
    cudaGraphExec_t graph = nullptr;
    cudaGraphNode_t begin_node = nullptr;
    cudaKernelNodeParams begin_params{};
    nhf::TiledBuild tb{};
    nhf::LatticeBuild lb{};
    bool lattice = false;
    nhf::GateDev gate{};
    bool gate_on = false;
    void *gate_mem = nullptr;   // gate budget partials
    double *h_gacc = nullptr;   // pinned staging of the gate partials
    bool tiled = false;
    std::string path = "multipass";
    std::string err;
};

namespace nhf {
// The ensemble's member-graph schedule (nhf_step.cu): build a member's batch
// graph, and launch it on the member's stream after `start`, recording `done`.
int member_graph_prepare(nhf_handle *h);
int member_graph_launch(nhf_handle *h, const uint32_t target[2], const uint32_t origin[2], cudaEvent_t start,
                        cudaEvent_t done);
}  // namespace nhf
