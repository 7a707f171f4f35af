// set.hpp -- host-side state of a lulesh_set (one GPU, one stream).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "host_setup.hpp"
#include "kernels.cuh"
#include "lulesh_b200.h"
#include "lulesh_dev.h"

// Node blocks last to first: the nodal kernel follows the force kernel,
// whose last-written corner forces are the ones still in L2 (measured on
// B200 at -s 100: nodal 53.7 -> 48.9 us, the same results).
#ifndef LULESH_NODAL_REVERSE
#define LULESH_NODAL_REVERSE 1
#endif

// The EOS of a subdomain set's fused cycle, and of a part of a multi-GPU
// problem, reads a comm face's neighbour element in the neighbouring
// subdomain or its proxy (k_eos<..., SUB>): the value k_monoq_ghost would
// copy into this subdomain's ghost face (CommMonoQ semantics,
// lulesh-comms-gpu.cu:1665-1806).  1 copies the ghost faces and reads them.
#ifndef LULESH_FUSED_MONOQ_GHOST
#define LULESH_FUSED_MONOQ_GHOST 0
#endif

// 0 launches every cycle kernel with plain stream order
#ifndef LULESH_PDL
#define LULESH_PDL 1
#endif

struct lulesh_set {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int flags = 0;
    lulesh::Params P{};
    int tp = 1;  // subdomains per axis of each job (1 for batches)
    // one unstructured domain read from this lmesh file (empty: -s meshes)
    std::string mesh_path;
    bool unstructured = false;
    // FNV-1a of an unstructured mesh's sizes, connectivity and coordinates
    // (identifies the mesh in checkpoints; 0 for -s meshes)
    unsigned long long mesh_hash = 0;
    int ndom = 0, njobs = 0;

    // per-domain metadata kept on the host
    std::vector<lulesh::DomDev> hdoms;
    std::vector<int> dom_rank;         // rank of each domain inside its job
    std::vector<int> dom_job;          // job of each domain
    std::vector<int> job_origin;       // domain holding the job's origin
    std::vector<lulesh_job> jobs;
    std::vector<size_t> corner_list_len;

    // block shapes and block-table order (lulesh_set_tuning): elements per
    // block of the FP64 element kernels, nodes per block of the nodal
    // kernel, 0 = domains in creation order / 1 = largest domain first
    int eb = lulesh::kElemBlock, nb = lulesh::kNodeBlock, order = 0;

    // device tables (elem_blocks is the base of one allocation holding all)
    lulesh::DomDev *ddoms = nullptr;
    lulesh::TimeCtl *dtc = nullptr;
    lulesh::TimeCtl *htc_pinned = nullptr;  // pinned mirror for readback
    int2 *elem_blocks = nullptr, *node_blocks = nullptr, *ghost_blocks = nullptr;
    int n_elem_blocks = 0, n_node_blocks = 0, n_ghost_blocks = 0;
    // subdomain sets: blocks over the max-side node faces (PosVel sync)
    int2 *sync_blocks = nullptr;
    int n_sync_blocks = 0;

    // mixed precision corner buffers
    lulesh::CornerF32 *dcorner32 = nullptr;

    // L2 access-policy window set on `stream` (single domains)
    bool l2_window = false;
    // launch the cycle kernels with programmatic dependent launch
    bool pdl = LULESH_PDL != 0;

    // the arena; subdomain sets start it with the node region (every
    // domain's x..zd, node_region_bytes), single domains carve in place
    void *arena = nullptr;
    size_t arena_bytes = 0;
    size_t node_region_bytes = 0;

    // captured cycle, and a graph of graph_cycles consecutive cycles
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_ready = false;
    int graph_cycles = 1;
    cudaGraph_t graph_k = nullptr;
    cudaGraphExec_t exec_k = nullptr;
    bool graph_k_ready = false;
    // whole-run graph: a WHILE conditional node around one cycle
    // (rungraph.cu); run_ctl[0] counts cycles, run_ctl[1] is the cap
    cudaGraph_t graph_run = nullptr;
    cudaGraphExec_t exec_run = nullptr;
    unsigned long long *run_ctl = nullptr;

    // one part of a problem split over several GPUs (lulesh_create_part):
    // the local domains hold ranks [first_rank, first_rank + ndom); proxies
    // of the remote neighbours follow them in the device domain table
    // (index ndom + k), with their arrays in proxy_arena
    int nparts = 1, part = 0, first_rank = 0;
    std::vector<lulesh::DomDev> hproxies;
    std::vector<int> proxy_rank;
    void *proxy_arena = nullptr;
    bool mass_pending = false;  // nodal mass waits for the MASS exchange
    // pointer tables of the halo pack (send) and unpack (recv) kernels, per
    // (kind, peer part)
    struct HaloTable {
        double **ptrs = nullptr;
        long long n = 0;
    };
    std::vector<int> peers;
    std::vector<HaloTable> halo_send, halo_recv;  // [kind * peers.size() + peer slot]
    // direct transport: this part's mailbox (every message it receives, at
    // the offsets of mailbox_layout, then one arrival flag per message) and
    // the mailboxes of its peers (mapped through CUDA IPC, or device
    // pointers of parts in the same process)
    void *mailbox = nullptr;
    size_t mailbox_bytes = 0;
    std::vector<void *> peer_mailbox;  // by peer slot
    std::vector<bool> peer_mailbox_ipc;

    // staged comm state: receive-buffer capacity per domain (doubles)
    long com_buf_doubles = 0;
    int max_plane = 0, max_edge = 0;
    int posted_msg = 0, posted_fields = 0, posted_do_recv = 1, posted_plane_only = 0;

    lulesh::SetArgs args(const int2 *blocks) const
    {
        lulesh::SetArgs a;
        a.doms = ddoms;
        a.tcs = dtc;
        a.blocks = blocks;
        a.materialize = (flags & LULESH_FLAG_MATERIALIZE) ? 1 : 0;
        a.pdl = pdl ? 1 : 0;
        return a;
    }
};

namespace lulesh {
void set_error(const std::string &msg);
int cuda_status(cudaError_t e, const char *what);
// enqueue one cycle (no graph)
int enqueue_cycle(lulesh_set *s);
// the FP64 force phase of every domain of the set
void launch_force_fp64(lulesh_set *s, cudaStream_t st);
// staged comm path of one cycle (comm.cu)
int enqueue_cycle_staged(lulesh_set *s);
// free the comm message tables of a set (comm.cu)
void comm_release(const lulesh_set *s);
// allocate the staged cycle's message tables ahead of graph capture
int comm_prepare(lulesh_set *s);
// (re)build the block tables from s->eb, s->nb, s->order
int build_tables(lulesh_set *s);
// release the captured cycle graphs (rebuilt at the next step)
void drop_graph(lulesh_set *s);
// read every job's time state back and return the first job's non-OK
// status (LULESH_OK when all are fine); synchronises the stream
int run_status(lulesh_set *s);
// prepare what enqueue_cycle needs before a capture (staged comm tables)
int prepare_capture(lulesh_set *s);
// nodal mass of every subdomain over the whole problem (setup.cu): each node
// adds volume/8 of the elements touching it in ascending global element
// index, reading neighbouring subdomains (or their proxies) through nbr
int nodal_mass_on_device(lulesh_set *s);
// a part of a multi-GPU problem: the proxies and halo tables (part.cu)
int part_build(lulesh_set *s);
void part_release(lulesh_set *s);
}  // namespace lulesh
