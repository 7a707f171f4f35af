// part.cu -- one GPU's part of a LULESH problem split over several GPUs.
//
// The reference runs one MPI rank per GPU and moves halos between them with
// one of its comm backends (LULESH/cuda/README.md:18-113): staged MPI,
// CUDA IPC puts with a token protocol (comm/comm_ipc_common.h:26-261), or
// direct remote stores with a float atomicAdd for the nodal force sum
// (lulesh-comms-direct.cu:50-404).  Here a part is a set holding some
// subdomains of the problem plus a proxy for every neighbour subdomain that
// lives on another part.  A proxy has the neighbour's own array layout; the
// halo messages (halo_plan.cpp) fill exactly the layers the local kernels
// read from it, and the cycle kernels are those of the in-device subdomain
// set, which read a neighbour through the domain table either way.  So:
//   * the nodal force sum adds every node's corners in corner order over
//     the whole mesh (the message carries corner forces, not partial sums):
//     no float atomics, and the single-domain result bit for bit;
//   * the transport is the caller's (NCCL send/recv, host staging, or a
//     device copy when all parts share one process): this file gathers a
//     message into a contiguous device buffer and scatters one into the
//     proxies, both through pointer tables built once from the plan.
#include <algorithm>
#include <climits>
#include <cstring>
#include <set>

#include "domain_dev.hpp"
#include "halo_plan.hpp"
#include "set.hpp"

namespace lulesh {

namespace {

// the arrays a proxy carries: x..zd, the corner forces, delv_* and volo
size_t proxy_bytes(const DomSizes &z)
{
    return 6 * align256(8 * z.N) + 3 * align256(8 * 8 * z.Ep) + 4 * align256(8 * z.E);
}

double *field_of_id(const DomDev &D, int id)
{
    switch (id) {
        case LULESH_F_X: return D.x;
        case LULESH_F_Y: return D.y;
        case LULESH_F_Z: return D.z;
        case LULESH_F_XD: return D.xd;
        case LULESH_F_YD: return D.yd;
        case LULESH_F_ZD: return D.zd;
        case LULESH_F_DELV_XI: return D.delv_xi;
        case LULESH_F_DELV_ETA: return D.delv_eta;
        case LULESH_F_DELV_ZETA: return D.delv_zeta;
        case LULESH_F_FX_ELEM: return D.fx_elem;
        case LULESH_F_FY_ELEM: return D.fy_elem;
        case LULESH_F_FZ_ELEM: return D.fz_elem;
        case LULESH_F_VOLO: return D.volo;
        default: return nullptr;
    }
}

__global__ void k_halo_gather(const double *const *__restrict__ src, double *__restrict__ out,
                              long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        out[i] = *src[i];
}

__global__ void k_halo_scatter(double *const *__restrict__ dst, const double *__restrict__ in,
                               long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        *dst[i] = in[i];
}

// the four values the parts reduce with an element-wise minimum
__global__ void k_dt_pack(const TimeCtl *T, long long *out)
{
    out[0] = (long long)T->min_courant;  // positive doubles: bit patterns order as int64
    out[1] = (long long)T->min_hydro;
    out[2] = T->bad_vol;
    out[3] = T->bad_q;
}

__global__ void k_dt_unpack(TimeCtl *T, const long long *in)
{
    T->min_courant = (unsigned long long)in[0];
    T->min_hydro = (unsigned long long)in[1];
    T->bad_vol = (int)in[2];
    T->bad_q = (int)in[3];
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Spin until *flag >= expect, for at most budget_ns of device time (and a
// hard cap on polls, should the timer not advance); on timeout the job
// stops with LULESH_TIMEOUT and the kernel returns.
__global__ void k_wait_flag(const volatile unsigned int *flag, unsigned int expect,
                            unsigned long long budget_ns, long long max_polls, TimeCtl *T)
{
    const unsigned long long t0 = global_ns();
    for (long long k = 0; k < max_polls; ++k) {
        if (*flag >= expect) {
            __threadfence();
            return;
        }
        if (global_ns() - t0 > budget_ns) break;
        __nanosleep(1000);
    }
    T->status = LULESH_TIMEOUT;
    T->done = 1;
    T->active = 0;
}

int grid_for(long long n)
{
    const long long b = (n + 255) / 256;
    return (int)std::max(1LL, std::min(b, 148LL * 16));
}

int upload_table(const std::vector<double *> &ptrs, lulesh_set::HaloTable *t)
{
    t->n = (long long)ptrs.size();
    if (ptrs.empty()) return LULESH_OK;
    int st = cuda_status(cudaMalloc(&t->ptrs, sizeof(double *) * ptrs.size()), "halo table");
    if (st != LULESH_OK) return st;
    return cuda_status(cudaMemcpy(t->ptrs, ptrs.data(), sizeof(double *) * ptrs.size(),
                                  cudaMemcpyHostToDevice),
                       "halo table");
}

int peer_slot(const lulesh_set *s, int peer)
{
    for (size_t i = 0; i < s->peers.size(); ++i)
        if (s->peers[i] == peer) return (int)i;
    return -1;
}

bool check_part(lulesh_set *s, int kind, int peer, int *slot)
{
    if (!s || kind < 0 || kind >= HALO_KINDS) {
        set_error("halo: bad set or message kind");
        return false;
    }
    *slot = peer_slot(s, peer);
    if (*slot < 0) {
        set_error("halo: part " + std::to_string(peer) + " is not a peer of this part");
        return false;
    }
    return true;
}

// The mailbox of part `part`: the message of each (kind, sender) it
// receives, in kind-major, ascending-sender order, each at a 256-byte
// boundary, then one 32-bit arrival flag per (kind, sender) in the same
// order.  Computed from the plan alone, so a sender finds its place in a
// receiver's mailbox without asking it.
struct MailboxLayout {
    std::vector<int> peers;
    std::vector<size_t> offset;  // bytes, [kind * peers.size() + slot]
    std::vector<long long> count;
    size_t flags = 0, bytes = 0;
};

MailboxLayout mailbox_layout(int nx, int tp, int nparts, int part)
{
    MailboxLayout L;
    L.peers = halo_peers(tp, nparts, part);
    std::vector<HaloItem> items;
    size_t off = 0;
    for (int kind = 0; kind < HALO_KINDS; ++kind)
        for (int q : L.peers) {
            halo_plan(nx, tp, nparts, q, part, kind, items);
            L.offset.push_back(off);
            L.count.push_back((long long)items.size());
            off += align256(sizeof(double) * items.size());
        }
    L.flags = off;
    L.bytes = off + align256(sizeof(unsigned int) * HALO_KINDS * L.peers.size());
    return L;
}

// Direct transport, sender side: gather this part's message for one peer
// and store it straight into the peer's mailbox (peer memory, NVLink), then
// make the stores visible system-wide before the flag kernel runs.
__global__ void k_halo_put(const double *const *__restrict__ src, double *dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        dst[i] = *src[i];
    __threadfence_system();
}

// ... then raise the arrival flag (after the put kernel completed, in
// stream order)
__global__ void k_flag_raise(unsigned int *flag, unsigned int value)
{
    __threadfence_system();
    atomicExch_system(flag, value);
}

// Direct transport, receiver side: wait (bounded, in device time and in
// polls) until the sender's flag reaches `expect`, then scatter the message
// from this part's mailbox into the proxies.  On timeout the job stops with
// LULESH_TIMEOUT and nothing is scattered.
__global__ void k_halo_take(const volatile unsigned int *flag, unsigned int expect,
                            unsigned long long budget_ns, long long max_polls,
                            double *const *__restrict__ dst, const double *in, long long n,
                            TimeCtl *T)
{
    __shared__ int arrived;
    if (threadIdx.x == 0) {
        arrived = 0;
        const unsigned long long t0 = global_ns();
        for (long long k = 0; k < max_polls; ++k) {
            if (*flag >= expect) {
                arrived = 1;
                break;
            }
            if (global_ns() - t0 > budget_ns) break;
            __nanosleep(500);
        }
        if (!arrived) {  // the rest of this cycle's kernels skip as well
            T->status = LULESH_TIMEOUT;
            T->done = 1;
            T->active = 0;
        }
        __threadfence();
    }
    __syncthreads();
    if (!arrived) return;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
         i += (long long)gridDim.x * blockDim.x)
        *dst[i] = in[i];
}

}  // namespace

int part_build(lulesh_set *s)
{
    const int tp = s->tp, T = tp * tp * tp;
    const lulesh_job &j = s->jobs[0];
    // neighbours owned by other parts
    std::set<int> remote;
    for (int d = 0; d < s->ndom; ++d) {
        const DomDev &D = s->hdoms[d];
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int c = D.col + dx, r = D.row + dy, p = D.plane + dz;
                    if ((dx | dy | dz) == 0 || c < 0 || r < 0 || p < 0 || c >= tp || r >= tp ||
                        p >= tp)
                        continue;
                    const int nr = c + tp * (r + tp * p);
                    if (halo_part_of(nr, tp, s->nparts) != s->part) remote.insert(nr);
                }
    }
    s->proxy_rank.assign(remote.begin(), remote.end());
    const DomSizes z = sizes_of(j.nx, j.numReg, 0);
    const size_t per = proxy_bytes(z);
    if (!s->proxy_rank.empty()) {
        int st = cuda_status(cudaMalloc(&s->proxy_arena, per * s->proxy_rank.size()),
                             "proxy arena");
        if (st != LULESH_OK) return st;
        st = cuda_status(cudaMemsetAsync(s->proxy_arena, 0, per * s->proxy_rank.size(), s->stream),
                         "proxy arena");
        if (st != LULESH_OK) return st;
    }
    Carver cv{static_cast<char *>(s->proxy_arena)};
    s->hproxies.clear();
    for (int r : s->proxy_rank) {
        DomDev P{};
        P.nx = j.nx;
        P.en = j.nx + 1;
        P.numElem = (int)z.E;
        P.numNode = (int)z.N;
        P.Ep = (int)z.Ep;
        P.allElem = (int)z.E;  // no ghost tail: a proxy's ghosts are never read
        P.col = r % tp;
        P.row = (r / tp) % tp;
        P.plane = r / (tp * tp);
        P.tp = tp;
        P.tc = 0;
        P.numReg = j.numReg;
        for (int k = 0; k < 27; ++k) P.nbr[k] = -1;
        for (int f = 0; f < 6; ++f) P.ghost[f] = -1;
        P.x = cv.take<double>(z.N); P.y = cv.take<double>(z.N); P.z = cv.take<double>(z.N);
        P.xd = cv.take<double>(z.N); P.yd = cv.take<double>(z.N); P.zd = cv.take<double>(z.N);
        P.fx_elem = cv.take<double>(8 * z.Ep);
        P.fy_elem = cv.take<double>(8 * z.Ep);
        P.fz_elem = cv.take<double>(8 * z.Ep);
        P.delv_xi = cv.take<double>(z.E);
        P.delv_eta = cv.take<double>(z.E);
        P.delv_zeta = cv.take<double>(z.E);
        P.volo = cv.take<double>(z.E);
        s->hproxies.push_back(P);
    }
    // pointer tables: sends read the local domains, receives write the proxies
    s->peers = halo_peers(tp, s->nparts, s->part);
    const size_t np = s->peers.size();
    s->halo_send.assign(HALO_KINDS * np, lulesh_set::HaloTable{});
    s->halo_recv.assign(HALO_KINDS * np, lulesh_set::HaloTable{});
    std::vector<HaloItem> items;
    std::vector<double *> ptrs;
    for (int kind = 0; kind < HALO_KINDS; ++kind)
        for (size_t i = 0; i < np; ++i) {
            const int q = s->peers[i];
            halo_plan(j.nx, tp, s->nparts, s->part, q, kind, items);
            ptrs.clear();
            for (const HaloItem &it : items) {
                const int d = it.rank - s->first_rank;
                if (d < 0 || d >= s->ndom || it.rank >= T) {
                    set_error("halo plan: sender rank not local");
                    return LULESH_INVALID_ARG;
                }
                ptrs.push_back(field_of_id(s->hdoms[d], it.field) + it.index);
            }
            int st = upload_table(ptrs, &s->halo_send[kind * np + i]);
            if (st != LULESH_OK) return st;
            halo_plan(j.nx, tp, s->nparts, q, s->part, kind, items);
            ptrs.clear();
            for (const HaloItem &it : items) {
                const auto pos = std::find(s->proxy_rank.begin(), s->proxy_rank.end(), it.rank);
                if (pos == s->proxy_rank.end()) {
                    set_error("halo plan: received rank has no proxy");
                    return LULESH_INVALID_ARG;
                }
                ptrs.push_back(field_of_id(s->hproxies[pos - s->proxy_rank.begin()], it.field) +
                               it.index);
            }
            st = upload_table(ptrs, &s->halo_recv[kind * np + i]);
            if (st != LULESH_OK) return st;
        }
    // the mailbox of the direct transport (its own allocation, so that it
    // can be exported to the peers' processes with cudaIpcGetMemHandle)
    const MailboxLayout L = mailbox_layout(j.nx, tp, s->nparts, s->part);
    s->mailbox_bytes = L.bytes;
    int st = cuda_status(cudaMalloc(&s->mailbox, L.bytes), "mailbox");
    if (st != LULESH_OK) return st;
    st = cuda_status(cudaMemsetAsync(s->mailbox, 0, L.bytes, s->stream), "mailbox");
    if (st != LULESH_OK) return st;
    s->peer_mailbox.assign(np, nullptr);
    s->peer_mailbox_ipc.assign(np, false);
    return LULESH_OK;
}

void part_release(lulesh_set *s)
{
    for (auto *v : {&s->halo_send, &s->halo_recv})
        for (auto &t : *v)
            if (t.ptrs) cudaFree(t.ptrs);
    s->halo_send.clear();
    s->halo_recv.clear();
    if (s->proxy_arena) cudaFree(s->proxy_arena);
    s->proxy_arena = nullptr;
    for (size_t i = 0; i < s->peer_mailbox.size(); ++i)
        if (s->peer_mailbox[i] && s->peer_mailbox_ipc[i]) cudaIpcCloseMemHandle(s->peer_mailbox[i]);
    s->peer_mailbox.clear();
    if (s->mailbox) cudaFree(s->mailbox);
    s->mailbox = nullptr;
}

}  // namespace lulesh

using namespace lulesh;

extern "C" {

int lulesh_part_finish_setup(lulesh_set *s)
{
    if (!s) return LULESH_INVALID_ARG;
    if (!s->mass_pending) return LULESH_OK;
    int st = nodal_mass_on_device(s);
    if (st != LULESH_OK) return st;
    s->mass_pending = false;
    return cuda_status(cudaStreamSynchronize(s->stream), "nodal mass");
}

long long lulesh_halo_count(lulesh_set *s, int kind, int peer, int to_peer)
{
    int slot;
    if (!check_part(s, kind, peer, &slot)) return LULESH_INVALID_ARG;
    const size_t i = kind * s->peers.size() + slot;
    return to_peer ? s->halo_send[i].n : s->halo_recv[i].n;
}

int lulesh_halo_pack(lulesh_set *s, int kind, int peer, double *dev_buf)
{
    int slot;
    if (!check_part(s, kind, peer, &slot)) return LULESH_INVALID_ARG;
    const lulesh_set::HaloTable &t = s->halo_send[kind * s->peers.size() + slot];
    if (t.n == 0) return LULESH_OK;
    if (!dev_buf) return LULESH_INVALID_ARG;
    k_halo_gather<<<grid_for(t.n), 256, 0, s->stream>>>(t.ptrs, dev_buf, t.n);
    return cuda_status(cudaGetLastError(), "halo pack");
}

int lulesh_halo_unpack(lulesh_set *s, int kind, int peer, const double *dev_buf)
{
    int slot;
    if (!check_part(s, kind, peer, &slot)) return LULESH_INVALID_ARG;
    const lulesh_set::HaloTable &t = s->halo_recv[kind * s->peers.size() + slot];
    if (t.n == 0) return LULESH_OK;
    if (!dev_buf) return LULESH_INVALID_ARG;
    k_halo_scatter<<<grid_for(t.n), 256, 0, s->stream>>>(t.ptrs, dev_buf, t.n);
    return cuda_status(cudaGetLastError(), "halo unpack");
}

int lulesh_part_phase(lulesh_set *s, int phase)
{
    if (!s) return LULESH_INVALID_ARG;
    if (s->mass_pending) {
        set_error("lulesh_part_phase: exchange MASS and call lulesh_part_finish_setup first");
        return LULESH_INVALID_ARG;
    }
    if (s->flags & (LULESH_FLAG_MIXED | LULESH_FLAG_COMM_STAGED) || s->unstructured) {
        set_error("lulesh_part_phase: FP64 structured sets with the fused exchange only");
        return LULESH_INVALID_ARG;
    }
    // plain stream order between phases: the transport's copies and
    // collectives sit between them on the same stream
    SetArgs ae = s->args(s->elem_blocks), an = s->args(s->node_blocks),
            ag = s->args(s->ghost_blocks), as = s->args(s->sync_blocks);
    ae.pdl = an.pdl = ag.pdl = as.pdl = 0;
    cudaStream_t st = s->stream;
    switch (phase) {
        case LULESH_PHASE_TIME_INCREMENT: launch_time_increment(s->dtc, s->njobs, s->P, st, false); break;
        case LULESH_PHASE_FORCE: launch_force(ae, s->n_elem_blocks, s->P, st, s->eb, false); break;
        case LULESH_PHASE_NODAL: launch_nodal(an, s->n_node_blocks, s->P, st, s->nb, false); break;
        case LULESH_PHASE_POSVEL_SYNC:
            if (s->tp > 1 && s->n_sync_blocks > 0) launch_posvel_sync(as, s->n_sync_blocks, st);
            break;
        case LULESH_PHASE_KINEMATICS:
            launch_kinematics(ae, s->n_elem_blocks, s->P, st, s->eb, false);
            break;
        case LULESH_PHASE_MONOQ_GHOST:
            // nothing to copy unless the EOS reads ghost faces (the proxies
            // hold the neighbours' layers after the MONOQ messages)
            if (LULESH_FUSED_MONOQ_GHOST && s->tp > 1 && s->n_ghost_blocks > 0)
                launch_monoq_ghost(ag, s->n_ghost_blocks, st);
            break;
        case LULESH_PHASE_EOS:
            launch_eos(ae, s->n_elem_blocks, s->P, st, s->eb, false,
                       !LULESH_FUSED_MONOQ_GHOST && s->tp > 1);
            break;
        default: set_error("lulesh_part_phase: unknown phase"); return LULESH_INVALID_ARG;
    }
    return cuda_status(cudaGetLastError(), "part phase");
}

int lulesh_part_dt_pack(lulesh_set *s, long long *dev_buf)
{
    if (!s || !dev_buf) return LULESH_INVALID_ARG;
    k_dt_pack<<<1, 1, 0, s->stream>>>(s->dtc, dev_buf);
    return cuda_status(cudaGetLastError(), "dt pack");
}

int lulesh_part_dt_unpack(lulesh_set *s, const long long *dev_buf)
{
    if (!s || !dev_buf) return LULESH_INVALID_ARG;
    k_dt_unpack<<<1, 1, 0, s->stream>>>(s->dtc, dev_buf);
    return cuda_status(cudaGetLastError(), "dt unpack");
}

int lulesh_part_mailbox(lulesh_set *s, void **dev_ptr, size_t *bytes, void *ipc_handle)
{
    if (!s || !s->mailbox) {
        set_error("lulesh_part_mailbox: not a part of a multi-GPU problem");
        return LULESH_INVALID_ARG;
    }
    if (dev_ptr) *dev_ptr = s->mailbox;
    if (bytes) *bytes = s->mailbox_bytes;
    if (ipc_handle) {
        cudaIpcMemHandle_t h;
        const int st = cuda_status(cudaIpcGetMemHandle(&h, s->mailbox), "mailbox IPC handle");
        if (st != LULESH_OK) return st;
        std::memcpy(ipc_handle, &h, sizeof h);
    }
    return LULESH_OK;
}

int lulesh_part_set_peer_mailbox(lulesh_set *s, int peer, const void *dev_ptr,
                                 const void *ipc_handle)
{
    int slot;
    if (!check_part(s, 0, peer, &slot)) return LULESH_INVALID_ARG;
    if ((dev_ptr == nullptr) == (ipc_handle == nullptr)) {
        set_error("lulesh_part_set_peer_mailbox: give a device pointer or an IPC handle");
        return LULESH_INVALID_ARG;
    }
    if (s->peer_mailbox[slot] && s->peer_mailbox_ipc[slot])
        cudaIpcCloseMemHandle(s->peer_mailbox[slot]);
    s->peer_mailbox[slot] = nullptr;
    if (dev_ptr) {
        s->peer_mailbox[slot] = const_cast<void *>(dev_ptr);
        s->peer_mailbox_ipc[slot] = false;
        return LULESH_OK;
    }
    cudaIpcMemHandle_t h;
    std::memcpy(&h, ipc_handle, sizeof h);
    void *p = nullptr;
    const int st = cuda_status(cudaIpcOpenMemHandle(&p, h, cudaIpcMemLazyEnablePeerAccess),
                               "open peer mailbox");
    if (st != LULESH_OK) return st;
    s->peer_mailbox[slot] = p;
    s->peer_mailbox_ipc[slot] = true;
    return LULESH_OK;
}

int lulesh_halo_put(lulesh_set *s, int kind, int peer, unsigned int seq)
{
    int slot;
    if (!check_part(s, kind, peer, &slot)) return LULESH_INVALID_ARG;
    if (!s->peer_mailbox[slot]) {
        set_error("lulesh_halo_put: the peer's mailbox is not set");
        return LULESH_INVALID_ARG;
    }
    const lulesh_set::HaloTable &t = s->halo_send[kind * s->peers.size() + slot];
    // where this part's message lands in the peer's mailbox
    const MailboxLayout L = mailbox_layout(s->jobs[0].nx, s->tp, s->nparts, peer);
    int me = -1;
    for (size_t i = 0; i < L.peers.size(); ++i)
        if (L.peers[i] == s->part) me = (int)i;
    const size_t idx = kind * L.peers.size() + me;
    if (me < 0 || L.count[idx] != t.n) {
        set_error("lulesh_halo_put: mailbox layout mismatch");
        return LULESH_INVALID_ARG;
    }
    char *base = static_cast<char *>(s->peer_mailbox[slot]);
    if (t.n > 0)
        k_halo_put<<<grid_for(t.n), 256, 0, s->stream>>>(
            t.ptrs, reinterpret_cast<double *>(base + L.offset[idx]), t.n);
    unsigned int *flag = reinterpret_cast<unsigned int *>(base + L.flags) + idx;
    k_flag_raise<<<1, 1, 0, s->stream>>>(flag, seq);
    return cuda_status(cudaGetLastError(), "halo put");
}

int lulesh_halo_take(lulesh_set *s, int kind, int peer, unsigned int seq, double timeout_ms)
{
    int slot;
    if (!check_part(s, kind, peer, &slot)) return LULESH_INVALID_ARG;
    if (!(timeout_ms > 0.0) || timeout_ms > 60000.0) {
        set_error("lulesh_halo_take: 0 < timeout_ms <= 60000");
        return LULESH_INVALID_ARG;
    }
    const lulesh_set::HaloTable &t = s->halo_recv[kind * s->peers.size() + slot];
    const MailboxLayout L = mailbox_layout(s->jobs[0].nx, s->tp, s->nparts, s->part);
    const size_t idx = kind * L.peers.size() + slot;
    char *base = static_cast<char *>(s->mailbox);
    const unsigned int *flag = reinterpret_cast<const unsigned int *>(base + L.flags) + idx;
    const unsigned long long ns = (unsigned long long)(timeout_ms * 1e6);
    const long long max_polls = (long long)(timeout_ms * 2e3) * 4 + 1000;
    k_halo_take<<<grid_for(t.n > 0 ? t.n : 1), 256, 0, s->stream>>>(
        flag, seq, ns, max_polls, t.ptrs, reinterpret_cast<const double *>(base + L.offset[idx]),
        t.n, s->dtc);
    return cuda_status(cudaGetLastError(), "halo take");
}

int lulesh_wait_flag(lulesh_set *s, const unsigned int *dev_flag, unsigned int expect,
                     double timeout_ms)
{
    if (!s || !dev_flag || !(timeout_ms > 0.0) || timeout_ms > 60000.0) {
        set_error("lulesh_wait_flag: need a flag and 0 < timeout_ms <= 60000");
        return LULESH_INVALID_ARG;
    }
    const unsigned long long ns = (unsigned long long)(timeout_ms * 1e6);
    // one poll per ~1 us of sleep: the cap ends the wait even if the device
    // timer stood still
    const long long max_polls = (long long)(timeout_ms * 1e3) * 4 + 1000;
    k_wait_flag<<<1, 1, 0, s->stream>>>(dev_flag, expect, ns, max_polls, s->dtc);
    return cuda_status(cudaGetLastError(), "wait flag");
}

}  // extern "C"
