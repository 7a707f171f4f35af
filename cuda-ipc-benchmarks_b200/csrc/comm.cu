// comm.cu -- the reference comm-backend interface over subdomains resident
// on one GPU.
//
// Reference contract (LULESH/cuda/src): CommRecv posts receives in a fixed
// order (lulesh-comms.cu:62-365), CommSendGpu packs faces/edges/corners of
// the given fields (lulesh-comms-gpu.cu:348-801), CommSBNGpu adds them into
// the shared nodes (805-1227), CommSyncPosVelGpu copies positions and
// velocities (1231-1661), CommMonoQGpu fills the delv_* ghost faces
// (1665-1806).  comm_backend.h:75-138 (shmRecvOffset) defines where, in
// the receiver's buffer, each message lands.
//
// In-device backend ("remote pack", the reference's mode C): a sender's
// pack kernel writes straight into the receiver's receive buffer at the
// posting-order offset; there is no intermediate send buffer, no host
// staging, no MPI.  Unpacking is deterministic: each receiving node adds
// (SBN) or copies (PosVel) the messages that cover it in posting order,
// one thread per node, so no float atomics are needed.
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "set.hpp"

namespace lulesh {

// ---- message geometry ---------------------------------------------------------

// The 26 receive slots in CommRecv posting order.  (dc,dr,dp) is the
// sender's position relative to the receiver; `lower` marks senders of
// lower rank, which are received only when doRecv (faces/edges/corners of
// lulesh-comms.cu:129-365 and comm_backend.h:102-128).
struct Slot {
    int dc, dr, dp, kind;  // kind 0 face, 1 edge, 2 corner
};
static const Slot kSlots[26] = {
    {0, 0, -1, 0},  {0, 0, 1, 0},   {0, -1, 0, 0},  {0, 1, 0, 0},   {-1, 0, 0, 0},
    {1, 0, 0, 0},   {-1, -1, 0, 1}, {0, -1, -1, 1}, {-1, 0, -1, 1}, {1, 1, 0, 1},
    {0, 1, 1, 1},   {1, 0, 1, 1},   {-1, 1, 0, 1},  {0, -1, 1, 1},  {-1, 0, 1, 1},
    {1, -1, 0, 1},  {0, 1, -1, 1},  {1, 0, -1, 1},  {-1, -1, -1, 2}, {-1, -1, 1, 2},
    {1, -1, -1, 2}, {1, -1, 1, 2},  {-1, 1, -1, 2}, {-1, 1, 1, 2},  {1, 1, -1, 2},
    {1, 1, 1, 2}};

// the same slots for device code: (dc, dr, dp, kind)
__constant__ int4 c_slots[26] = {
    {0, 0, -1, 0},  {0, 0, 1, 0},   {0, -1, 0, 0},  {0, 1, 0, 0},   {-1, 0, 0, 0},
    {1, 0, 0, 0},   {-1, -1, 0, 1}, {0, -1, -1, 1}, {-1, 0, -1, 1}, {1, 1, 0, 1},
    {0, 1, 1, 1},   {1, 0, 1, 1},   {-1, 1, 0, 1},  {0, -1, 1, 1},  {-1, 0, 1, 1},
    {1, -1, 0, 1},  {0, 1, -1, 1},  {1, 0, -1, 1},  {-1, -1, -1, 2}, {-1, -1, 1, 2},
    {1, -1, -1, 2}, {1, -1, 1, 2},  {-1, 1, -1, 2}, {-1, 1, 1, 2},  {1, 1, -1, 2},
    {1, 1, 1, 2}};

// a direction is "higher" when its most significant non-zero component
// (plane, then row, then col) is positive: the neighbour has a higher rank
static inline __host__ __device__ bool dir_higher(int dc, int dr, int dp)
{
    if (dp != 0) return dp > 0;
    if (dr != 0) return dr > 0;
    return dc > 0;
}

// padded message slot sizes of SetupCommBuffers, lulesh.cu:457-460
static inline void slot_sizes(int nx, int *maxPlane, int *maxEdge)
{
    const int pad = 16;
    const int edge = nx + 1;
    *maxPlane = ((edge * edge + pad - 1) / pad) * pad;
    *maxEdge = ((edge + pad - 1) / pad) * pad;
}

// offset of the message from direction (dc,dr,dp) in the receiver's buffer,
// -1 if the receiver posts no such receive (shmRecvOffset)
static long recv_offset(const DomDev &R, int dc, int dr, int dp, int xferFields, bool doRecv,
                        bool planeOnly)
{
    int maxPlane, maxEdge;
    slot_sizes(R.nx, &maxPlane, &maxEdge);
    const long maxPlaneComm = (long)xferFields * maxPlane;
    const long maxEdgeComm = (long)xferFields * maxEdge;
    long pmsg = 0, emsg = 0, cmsg = 0;
    for (int k = 0; k < 26; ++k) {
        const Slot &s = kSlots[k];
        if (planeOnly && s.kind > 0) break;
        const int c = R.col + s.dc, r = R.row + s.dr, p = R.plane + s.dp;
        const bool exists = c >= 0 && r >= 0 && p >= 0 && c < R.tp && r < R.tp && p < R.tp;
        const bool posted = exists && (doRecv || dir_higher(s.dc, s.dr, s.dp));
        if (!posted) continue;
        const bool match = (s.dc == dc && s.dr == dr && s.dp == dp);
        if (s.kind == 0) {
            if (match) return pmsg * maxPlaneComm;
            ++pmsg;
        } else if (s.kind == 1) {
            if (match) return pmsg * maxPlaneComm + emsg * maxEdgeComm;
            ++emsg;
        } else {
            if (match) return pmsg * maxPlaneComm + emsg * maxEdgeComm + cmsg * 16;
            ++cmsg;
        }
    }
    return -1;
}

// One message: domain src sends toward direction (tx,ty,tz) to domain dst.
struct Msg {
    int src, dst;
    int tx, ty, tz;
    int count;      // values per field
    long recv_off;  // doubles into dst's commRecv
};

struct MsgTable {
    Msg *msgs = nullptr;
    int2 *blocks = nullptr;  // (msg, first item)
    int nmsg = 0, nblocks = 0;
};

// device pointer of a Domain field by lulesh_field_id
__device__ __forceinline__ double *field_ptr(const DomDev &D, int id)
{
    switch (id) {
        case LULESH_F_X: return D.x;
        case LULESH_F_Y: return D.y;
        case LULESH_F_Z: return D.z;
        case LULESH_F_XD: return D.xd;
        case LULESH_F_YD: return D.yd;
        case LULESH_F_ZD: return D.zd;
        case LULESH_F_FX: return D.fx;
        case LULESH_F_FY: return D.fy;
        case LULESH_F_FZ: return D.fz;
        case LULESH_F_NODALMASS: return D.nodalMass;
        case LULESH_F_DELV_XI: return D.delv_xi;
        case LULESH_F_DELV_ETA: return D.delv_eta;
        default: return D.delv_zeta;
    }
}

struct FieldList {
    int n;
    int id[LULESH_MAX_FIELDS_PER_COMM];
};

// ---- pack: CommSendGpu ----------------------------------------------------

// item -> sender index.  Nodal messages have extent nx+1 per free axis and
// sit on the sender's node faces; element (MonoQ) messages have extent nx
// and take the sender's boundary element layer.  Free axes run x fastest,
// then y, then z (SendPlane/SendEdge, lulesh-comms-gpu.cu:60-322).
__device__ __forceinline__ int msg_source_index(const DomDev &S, const Msg &m, int item,
                                                bool elems)
{
    const int ext = elems ? S.nx : S.en;
    const int hi = ext - 1;
    int c[3];
    const int t[3] = {m.tx, m.ty, m.tz};
    int rem = item;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        if (t[a] == 0) {
            c[a] = rem % ext;
            rem /= ext;
        } else {
            c[a] = (t[a] < 0) ? 0 : hi;
        }
    }
    return (c[2] * ext + c[1]) * ext + c[0];
}

__global__ void k_pack(const DomDev *doms, const TimeCtl *tcs, const Msg *msgs,
                       const int2 *blocks, FieldList fl, int elems, int gate)
{
    const int2 b = blocks[blockIdx.x];
    const Msg m = msgs[b.x];
    const DomDev &S = doms[m.src];
    if (gate && !tcs[S.tc].active) return;
    const int item = b.y + threadIdx.x;
    if (item >= m.count) return;
    const DomDev &R = doms[m.dst];
    TimeCtl *T = const_cast<TimeCtl *>(&tcs[R.tc]);
    const int src = chk_index(msg_source_index(S, m, item, elems != 0),
                              elems ? S.numElem : S.numNode, T, kChkNode);
    for (int f = 0; f < fl.n; ++f) {
        const int d = chk_index(m.recv_off + item + (long long)f * m.count, R.commRecvLen, T,
                                kChkLink);
        R.commRecv[d] = field_ptr(S, fl.id[f])[src];
    }
}

// ---- unpack: CommSBNGpu / CommSyncPosVelGpu ---------------------------------

// Receiving node (px,py,pz) of R: walk the posted receives in order and
// fold every message that covers the node.  add != 0: sum (SBN), else the
// last covering message wins (PosVel).
__global__ void k_unpack_nodes(const DomDev *doms, const TimeCtl *tcs, const int2 *blocks,
                               FieldList fl, int xferFields, int doRecv, int add, int gate)
{
    const int2 b = blocks[blockIdx.x];
    const DomDev &R = doms[b.x];
    if (gate && !tcs[R.tc].active) return;
    const int i = b.y + threadIdx.x;
    if (i >= R.numNode) return;
    const int en = R.en, n = R.nx;
    const int p[3] = {i % en, (i / en) % en, i / (en * en)};
    if (p[0] != 0 && p[0] != n && p[1] != 0 && p[1] != n && p[2] != 0 && p[2] != n) return;
    int maxPlane, maxEdge;
    {
        const int pad = 16, edge = n + 1;
        maxPlane = ((edge * edge + pad - 1) / pad) * pad;
        maxEdge = ((edge + pad - 1) / pad) * pad;
    }
    const long maxPlaneComm = (long)xferFields * maxPlane;
    const long maxEdgeComm = (long)xferFields * maxEdge;
    double acc[LULESH_MAX_FIELDS_PER_COMM];
    for (int f = 0; f < fl.n; ++f) acc[f] = field_ptr(R, fl.id[f])[i];
    bool touched = false;
    long pmsg = 0, emsg = 0, cmsg = 0;
    for (int k = 0; k < 26; ++k) {
        const int dc = c_slots[k].x, dr = c_slots[k].y, dp = c_slots[k].z, kind = c_slots[k].w;
        const int c = R.col + dc, r = R.row + dr, pl = R.plane + dp;
        const bool exists = c >= 0 && r >= 0 && pl >= 0 && c < R.tp && r < R.tp && pl < R.tp;
        if (!exists || !(doRecv || dir_higher(dc, dr, dp))) continue;
        long off;
        if (kind == 0)
            off = pmsg++ * maxPlaneComm;
        else if (kind == 1)
            off = pmsg * maxPlaneComm + emsg++ * maxEdgeComm;
        else
            off = pmsg * maxPlaneComm + emsg * maxEdgeComm + cmsg++ * 16;
        // does the message from (dc,dr,dp) cover this node, and at which item
        const int s[3] = {dc, dr, dp};
        bool cover = true;
        int item = 0, stride = 1, count = 1;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (s[a] < 0)
                cover = cover && (p[a] == 0);
            else if (s[a] > 0)
                cover = cover && (p[a] == n);
            else {
                item += p[a] * stride;
                stride *= en;
                count *= en;
            }
        }
        if (!cover) continue;
        touched = true;
        for (int f = 0; f < fl.n; ++f) {
            const double v = R.commRecv[chk_index(off + item + (long long)f * count,
                                                  R.commRecvLen,
                                                  const_cast<TimeCtl *>(&tcs[R.tc]), kChkLink)];
            acc[f] = add ? acc[f] + v : v;
        }
    }
    if (!touched) return;
    for (int f = 0; f < fl.n; ++f) field_ptr(R, fl.id[f])[i] = acc[f];
}

// ---- unpack: CommMonoQGpu ----------------------------------------------------

__global__ void k_unpack_monoq(const DomDev *doms, const TimeCtl *tcs, const int2 *blocks,
                               int gate)
{
    const int2 b = blocks[blockIdx.x];
    const DomDev &R = doms[b.x];
    if (gate && !tcs[R.tc].active) return;
    const int f = b.y >> 24;
    const int item = (b.y & 0xffffff) + threadIdx.x;
    const int nx = R.nx;
    if (item >= nx * nx || R.ghost[f] < 0) return;
    // receive slots 0..5 are the faces in ghost order; MonoQ posts with
    // doRecv, so every existing neighbour face is present
    int maxPlane;
    {
        const int pad = 16, edge = nx + 1;
        maxPlane = ((edge * edge + pad - 1) / pad) * pad;
    }
    int pmsg = 0;
    for (int k = 0; k < f; ++k)
        if (R.ghost[k] >= 0) ++pmsg;
    const long off = (long)pmsg * 3 * maxPlane;
    const int count = nx * nx;
    TimeCtl *T = const_cast<TimeCtl *>(&tcs[R.tc]);
    const int g = chk_index(R.ghost[f] + item, R.allElem, T, kChkLink);
    const long long len = R.commRecvLen;
    R.delv_xi[g] = R.commRecv[chk_index(off + item, len, T, kChkLink)];
    R.delv_eta[g] = R.commRecv[chk_index(off + count + item, len, T, kChkLink)];
    R.delv_zeta[g] = R.commRecv[chk_index(off + 2 * count + item, len, T, kChkLink)];
}

// ---- host side --------------------------------------------------------------

struct CommCache {
    std::map<std::tuple<int, int, int, int, int>, MsgTable> tables;
    int2 *surface_blocks = nullptr;
    int n_surface_blocks = 0;
};
// One cache per set.  Sets on different host threads may build their
// tables at the same time, so the map itself is guarded; a set's own entry
// is used only by the thread driving that set (map nodes do not move).
static std::map<const lulesh_set *, CommCache> g_comm;
static std::mutex g_comm_mu;

static CommCache &cache_of(const lulesh_set *s)
{
    std::lock_guard<std::mutex> lk(g_comm_mu);
    return g_comm[s];
}

// messages that rank `rank` (or every rank, -1) sends
static int build_msgs(lulesh_set *s, int rank, int xferFields, bool doSend, bool planeOnly,
                      bool elems, MsgTable *out)
{
    std::vector<Msg> msgs;
    std::vector<int2> blocks;
    for (int d = 0; d < s->ndom; ++d) {
        if (rank >= 0 && s->dom_rank[d] != rank) continue;
        const DomDev &S = s->hdoms[d];
        if (S.tp <= 1) continue;
        for (int k = 0; k < 26; ++k) {
            // sender-side direction t; the receiver sees the sender at -t
            const int tx = -kSlots[k].dc, ty = -kSlots[k].dr, tz = -kSlots[k].dp;
            const int kind = kSlots[k].kind;
            if (planeOnly && kind > 0) continue;
            const int nb = S.nbr[(tx + 1) + 3 * (ty + 1) + 9 * (tz + 1)];
            if (nb < 0) continue;
            if (dir_higher(tx, ty, tz) && !doSend) continue;
            const DomDev &R = s->hdoms[nb];
            const long off = recv_offset(R, -tx, -ty, -tz, xferFields,
                                         /*doRecv=*/doSend, planeOnly);
            if (off < 0) {
                set_error("comm: receiver posted no matching receive");
                return LULESH_INVALID_ARG;
            }
            const int ext = elems ? S.nx : S.en;
            int count = 1;
            if (tx == 0) count *= ext;
            if (ty == 0) count *= ext;
            if (tz == 0) count *= ext;
            const int mi = (int)msgs.size();
            msgs.push_back(Msg{d, nb, tx, ty, tz, count, off});
            for (int it = 0; it < count; it += 128) blocks.push_back(make_int2(mi, it));
        }
    }
    out->nmsg = (int)msgs.size();
    out->nblocks = (int)blocks.size();
    if (msgs.empty()) return LULESH_OK;
    int st = cuda_status(cudaMalloc(&out->msgs, sizeof(Msg) * msgs.size()), "comm table");
    if (st != LULESH_OK) return st;
    st = cuda_status(cudaMalloc(&out->blocks, sizeof(int2) * blocks.size()), "comm table");
    if (st != LULESH_OK) return st;
    st = cuda_status(cudaMemcpy(out->msgs, msgs.data(), sizeof(Msg) * msgs.size(),
                                cudaMemcpyHostToDevice),
                     "comm table");
    if (st != LULESH_OK) return st;
    return cuda_status(cudaMemcpy(out->blocks, blocks.data(), sizeof(int2) * blocks.size(),
                                  cudaMemcpyHostToDevice),
                       "comm table");
}

static int get_msgs(lulesh_set *s, int rank, int xferFields, bool doSend, bool planeOnly,
                    bool elems, MsgTable **out)
{
    CommCache &cc = cache_of(s);
    auto key = std::make_tuple(rank, xferFields, (int)doSend, (int)planeOnly, (int)elems);
    auto it = cc.tables.find(key);
    if (it == cc.tables.end()) {
        MsgTable t;
        int st = build_msgs(s, rank, xferFields, doSend, planeOnly, elems, &t);
        if (st != LULESH_OK) return st;
        it = cc.tables.emplace(key, t).first;
    }
    *out = &it->second;
    return LULESH_OK;
}

static int surface_blocks(lulesh_set *s, int rank, std::vector<int2> *out)
{
    for (int d = 0; d < s->ndom; ++d) {
        if (rank >= 0 && s->dom_rank[d] != rank) continue;
        const DomDev &D = s->hdoms[d];
        if (D.tp <= 1) continue;
        for (int i = 0; i < D.numNode; i += kNodeBlock) out->push_back(make_int2(d, i));
    }
    return LULESH_OK;
}

static int node_blocks_for(lulesh_set *s, int rank, int2 **blocks, int *n)
{
    if (rank < 0) {
        *blocks = s->node_blocks;
        *n = s->n_node_blocks;
        return LULESH_OK;
    }
    CommCache &cc = cache_of(s);
    auto key = std::make_tuple(rank, -1, -1, -1, -1);
    auto it = cc.tables.find(key);
    if (it == cc.tables.end()) {
        std::vector<int2> b;
        surface_blocks(s, rank, &b);
        MsgTable t;
        t.nblocks = (int)b.size();
        if (!b.empty()) {
            int st = cuda_status(cudaMalloc(&t.blocks, sizeof(int2) * b.size()), "comm table");
            if (st != LULESH_OK) return st;
            st = cuda_status(cudaMemcpy(t.blocks, b.data(), sizeof(int2) * b.size(),
                                        cudaMemcpyHostToDevice),
                             "comm table");
            if (st != LULESH_OK) return st;
        }
        it = cc.tables.emplace(key, t).first;
    }
    *blocks = it->second.blocks;
    *n = it->second.nblocks;
    return LULESH_OK;
}

static bool fields_ok(int xferFields, const int *ids, FieldList *fl)
{
    if (xferFields < 1 || xferFields > LULESH_MAX_FIELDS_PER_COMM || !ids) return false;
    fl->n = xferFields;
    for (int f = 0; f < xferFields; ++f) {
        if (ids[f] < LULESH_F_X || ids[f] > LULESH_F_DELV_ZETA) return false;
        fl->id[f] = ids[f];
    }
    return true;
}

void comm_release(const lulesh_set *s)
{
    std::lock_guard<std::mutex> lk(g_comm_mu);
    auto it = g_comm.find(s);
    if (it == g_comm.end()) return;
    for (auto &kv : it->second.tables) {
        if (kv.second.msgs) cudaFree(kv.second.msgs);
        if (kv.second.blocks) cudaFree(kv.second.blocks);
    }
    g_comm.erase(it);
}

// One cycle with the halo exchange done by the reference's Comm* sequence
// (CalcForceForNodes lulesh.cu:2894-2923, LagrangeNodal 3046-3099,
// LagrangeElements 4143-4214).  Every launch is gated on the job's active
// flag so the cycle can be replayed from a CUDA graph.
int comm_sbn_impl(lulesh_set *s, int rank, const FieldList &fl, int gate);
int comm_posvel_impl(lulesh_set *s, int rank, int gate);
int comm_monoq_impl(lulesh_set *s, int rank, int gate);
int comm_send_impl(lulesh_set *s, int rank, int xferFields, const FieldList &fl, bool doSend,
                   bool planeOnly, bool elems, int gate);

// Build (allocate and upload) the message tables the staged cycle uses, so
// that capturing the cycle into a graph performs no allocation.
int comm_prepare(lulesh_set *s)
{
    if (s->tp <= 1) return LULESH_OK;
    MsgTable *t;
    int st;
    if ((st = get_msgs(s, -1, 3, true, false, false, &t)) != LULESH_OK) return st;  // SBN
    if ((st = get_msgs(s, -1, 6, false, false, false, &t)) != LULESH_OK) return st; // PosVel
    return get_msgs(s, -1, 3, true, true, true, &t);                                // MonoQ
}

int enqueue_cycle_staged(lulesh_set *s)
{
    cudaStream_t st = s->stream;
    int r;
    launch_time_increment(s->dtc, s->njobs, s->P, st, s->pdl);
    if ((r = cuda_status(cudaGetLastError(), "staged time increment")) != LULESH_OK) return r;
    launch_force_fp64(s, st);
    if ((r = cuda_status(cudaGetLastError(), "staged force")) != LULESH_OK) return r;
    // AddNodeForcesFromElems over local corners only, then SBN exchange
    launch_nodal_gather_local(s->args(s->node_blocks), s->n_node_blocks, st);
    if ((r = cuda_status(cudaGetLastError(), "staged local node sums")) != LULESH_OK) return r;
    FieldList f3{3, {LULESH_F_FX, LULESH_F_FY, LULESH_F_FZ}};
    if (s->tp > 1) {
        if ((r = comm_send_impl(s, -1, 3, f3, true, false, false, 1)) != LULESH_OK) return r;
        if ((r = comm_sbn_impl(s, -1, f3, 1)) != LULESH_OK) return r;
    }
    launch_nodal_update(s->args(s->node_blocks), s->n_node_blocks, s->P, st);
    if ((r = cuda_status(cudaGetLastError(), "staged node update")) != LULESH_OK) return r;
    if (s->tp > 1) {
        FieldList f6{6, {LULESH_F_X, LULESH_F_Y, LULESH_F_Z, LULESH_F_XD, LULESH_F_YD,
                         LULESH_F_ZD}};
        if ((r = comm_send_impl(s, -1, 6, f6, false, false, false, 1)) != LULESH_OK) return r;
        if ((r = comm_posvel_impl(s, -1, 1)) != LULESH_OK) return r;
    }
    launch_kinematics(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st);
    if ((r = cuda_status(cudaGetLastError(), "staged kinematics")) != LULESH_OK) return r;
    if (s->tp > 1) {
        FieldList fq{3, {LULESH_F_DELV_XI, LULESH_F_DELV_ETA, LULESH_F_DELV_ZETA}};
        if ((r = comm_send_impl(s, -1, 3, fq, true, true, true, 1)) != LULESH_OK) return r;
        if ((r = comm_monoq_impl(s, -1, 1)) != LULESH_OK) return r;
    }
    launch_eos(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st);
    return cuda_status(cudaGetLastError(), "staged cycle launch");
}

int comm_send_impl(lulesh_set *s, int rank, int xferFields, const FieldList &fl, bool doSend,
                   bool planeOnly, bool elems, int gate)
{
    MsgTable *t;
    int st = get_msgs(s, rank, xferFields, doSend, planeOnly, elems, &t);
    if (st != LULESH_OK) return st;
    if (t->nblocks == 0) return LULESH_OK;
    k_pack<<<t->nblocks, 128, 0, s->stream>>>(s->ddoms, s->dtc, t->msgs, t->blocks, fl,
                                              elems ? 1 : 0, gate);
    return cuda_status(cudaGetLastError(), "CommSend pack");
}

int comm_sbn_impl(lulesh_set *s, int rank, const FieldList &fl, int gate)
{
    int2 *b;
    int n;
    int st = node_blocks_for(s, rank, &b, &n);
    if (st != LULESH_OK || n == 0) return st;
    k_unpack_nodes<<<n, kNodeBlock, 0, s->stream>>>(s->ddoms, s->dtc, b, fl, fl.n, 1, 1, gate);
    return cuda_status(cudaGetLastError(), "CommSBN unpack");
}

int comm_posvel_impl(lulesh_set *s, int rank, int gate)
{
    int2 *b;
    int n;
    int st = node_blocks_for(s, rank, &b, &n);
    if (st != LULESH_OK || n == 0) return st;
    FieldList f6{6, {LULESH_F_X, LULESH_F_Y, LULESH_F_Z, LULESH_F_XD, LULESH_F_YD, LULESH_F_ZD}};
    k_unpack_nodes<<<n, kNodeBlock, 0, s->stream>>>(s->ddoms, s->dtc, b, f6, 6, 0, 0, gate);
    return cuda_status(cudaGetLastError(), "CommSyncPosVel unpack");
}

int comm_monoq_impl(lulesh_set *s, int rank, int gate)
{
    if (s->n_ghost_blocks == 0) return LULESH_OK;
    if (rank >= 0) {
        std::vector<int2> gb;
        for (int d = 0; d < s->ndom; ++d) {
            if (s->dom_rank[d] != rank) continue;
            const DomDev &D = s->hdoms[d];
            for (int f = 0; f < 6; ++f)
                if (D.ghost[f] >= 0)
                    for (int i = 0; i < D.nx * D.nx; i += kElemBlock)
                        gb.push_back(make_int2(d, (f << 24) | i));
        }
        if (gb.empty()) return LULESH_OK;
        int2 *tmp = nullptr;
        int st = cuda_status(cudaMalloc(&tmp, sizeof(int2) * gb.size()), "monoq table");
        if (st != LULESH_OK) return st;
        cudaMemcpy(tmp, gb.data(), sizeof(int2) * gb.size(), cudaMemcpyHostToDevice);
        k_unpack_monoq<<<(int)gb.size(), kElemBlock, 0, s->stream>>>(s->ddoms, s->dtc, tmp, gate);
        st = cuda_status(cudaGetLastError(), "CommMonoQ unpack");
        cudaStreamSynchronize(s->stream);
        cudaFree(tmp);
        return st;
    }
    k_unpack_monoq<<<s->n_ghost_blocks, kElemBlock, 0, s->stream>>>(s->ddoms, s->dtc,
                                                                     s->ghost_blocks, gate);
    return cuda_status(cudaGetLastError(), "CommMonoQ unpack");
}

}  // namespace lulesh

using namespace lulesh;

extern "C" {

long lulesh_comm_recv_offset(lulesh_set *s, int recvRank, int dCol, int dRow, int dPlane,
                             int xferFields, int doRecv, int planeOnly)
{
    if (!s || s->tp <= 1 || recvRank < 0 || recvRank >= s->tp * s->tp * s->tp) return -1;
    for (int d = 0; d < s->ndom; ++d)
        if (s->dom_rank[d] == recvRank)
            return recv_offset(s->hdoms[d], dCol, dRow, dPlane, xferFields, doRecv != 0,
                               planeOnly != 0);
    return -1;
}

static int check_rank(lulesh_set *s, int rank)
{
    if (!s) return LULESH_INVALID_ARG;
    if (rank < -1 || rank >= s->tp * s->tp * s->tp) {
        set_error("comm: rank out of range");
        return LULESH_INVALID_ARG;
    }
    return LULESH_OK;
}

int lulesh_comm_recv(lulesh_set *s, int rank, int msgType, int xferFields, int dx, int dy,
                     int dz, int doRecv, int planeOnly)
{
    int st = check_rank(s, rank);
    if (st != LULESH_OK) return st;
    if (xferFields < 1 || xferFields > LULESH_MAX_FIELDS_PER_COMM ||
        (msgType != LULESH_MSG_COMM_SBN && msgType != LULESH_MSG_SYNC_POS_VEL &&
         msgType != LULESH_MSG_MONOQ)) {
        set_error("CommRecv: bad message type or field count");
        return LULESH_INVALID_ARG;
    }
    if (s->tp <= 1) return LULESH_OK;  // numRanks() == 1
    const int n = s->hdoms[0].nx;
    const int want = (msgType == LULESH_MSG_MONOQ) ? n : n + 1;
    if (dx != want || dy != want || dz != want) {
        set_error("CommRecv: dx/dy/dz must be the message extents of this mesh");
        return LULESH_INVALID_ARG;
    }
    // receives are implicit: the buffer region of each posted message is
    // fixed by the posting order, which the senders replay
    s->posted_msg = msgType;
    s->posted_fields = xferFields;
    s->posted_do_recv = doRecv;
    s->posted_plane_only = planeOnly;
    return LULESH_OK;
}

int lulesh_comm_send(lulesh_set *s, int rank, int msgType, int xferFields, const int *fieldIds,
                     int dx, int dy, int dz, int doSend, int planeOnly)
{
    int st = check_rank(s, rank);
    if (st != LULESH_OK) return st;
    FieldList fl;
    if (!fields_ok(xferFields, fieldIds, &fl)) {
        set_error("CommSend: bad field list");
        return LULESH_INVALID_ARG;
    }
    if (s->tp <= 1) return LULESH_OK;
    const bool elems = (msgType == LULESH_MSG_MONOQ);
    const int n = s->hdoms[0].nx;
    const int want = elems ? n : n + 1;
    if (dx != want || dy != want || dz != want) {
        set_error("CommSend: dx/dy/dz must be the message extents of this mesh");
        return LULESH_INVALID_ARG;
    }
    return comm_send_impl(s, rank, xferFields, fl, doSend != 0, planeOnly != 0, elems, 0);
}

int lulesh_comm_sbn(lulesh_set *s, int rank, int xferFields, const int *fieldIds)
{
    int st = check_rank(s, rank);
    if (st != LULESH_OK) return st;
    FieldList fl;
    if (!fields_ok(xferFields, fieldIds, &fl)) {
        set_error("CommSBN: bad field list");
        return LULESH_INVALID_ARG;
    }
    if (s->tp <= 1) return LULESH_OK;
    return comm_sbn_impl(s, rank, fl, 0);
}

int lulesh_comm_sync_posvel(lulesh_set *s, int rank)
{
    int st = check_rank(s, rank);
    if (st != LULESH_OK) return st;
    if (s->tp <= 1) return LULESH_OK;
    return comm_posvel_impl(s, rank, 0);
}

int lulesh_comm_monoq(lulesh_set *s, int rank)
{
    int st = check_rank(s, rank);
    if (st != LULESH_OK) return st;
    if (s->tp <= 1) return LULESH_OK;
    return comm_monoq_impl(s, rank, 0);
}

}  // extern "C"
