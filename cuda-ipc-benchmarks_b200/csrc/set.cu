// set.cu -- lifetime, stepping and results of a lulesh_set (the C ABI).
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "domain_dev.hpp"
#include "halo_plan.hpp"
#include "set.hpp"

// The fused subdomain cycle needs no PosVel sync (CommSyncPosVel,
// lulesh-comms.cu:115-168).  The reference syncs because each rank sums a
// shared node's forces as its own partial sum plus the neighbour's, in its
// own order, so the two copies of the node can differ in the last bits.
// Here every subdomain gathers every corner of its nodes, the neighbours'
// included, in the single-domain corner order, and the node masses are the
// single-domain sums: both copies of a shared node take the same operations
// on the same values and stay equal bit for bit (checked against the single
// domain, every field, 2^3, 3^3 and 4^3 subdomains, up to 400 cycles).
// Leaving the copy out takes 2x2x2 of -s 50 from 349.5 to 343.9 us per
// cycle.  1 puts the k_posvel_sync launch back in the fused cycle.  The
// staged Comm* path keeps the reference's exchange; the parts of a
// multi-GPU problem exchange POSVEL only when their driver asks for it.
#ifndef LULESH_FUSED_POSVEL_SYNC
#define LULESH_FUSED_POSVEL_SYNC 0
#endif

namespace lulesh {

static thread_local std::string g_last_error;

void set_error(const std::string &msg) { g_last_error = msg; }

int cuda_status(cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return LULESH_OK;
    set_error(std::string(what) + ": " + cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return LULESH_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return LULESH_NO_DEVICE;
    return LULESH_CUDA_ERROR;
}

#define LCHECK(call)                                            \
    do {                                                        \
        int _st = cuda_status((call), #call);                   \
        if (_st != LULESH_OK) return _st;                       \
    } while (0)

// ---- creation -------------------------------------------------------------

static int validate_job(const lulesh_job &j)
{
    if (j.nx > LULESH_MAX_NX) {
        set_error("nx above LULESH_MAX_NX (645): its 32-bit corner indices would overflow; "
                  "run the mesh as tp^3 subdomains");
        return LULESH_INVALID_ARG;
    }
    if (j.nx < 1 || j.numReg < 1 || j.numReg > 1000 || j.balance < 0 || j.balance > 30 ||
        j.cost < 0 || j.cost > 1000) {
        set_error("invalid job parameters (nx >= 1, numReg in [1,1000], balance in [0,30], "
                  "cost in [0,1000])");
        return LULESH_INVALID_ARG;
    }
    return LULESH_OK;
}

int build_tables(lulesh_set *s)
{
    // domains in creation order, or largest first: big domains then start
    // their blocks first and small ones fill the tail of each launch
    std::vector<int> dord(s->ndom);
    for (int d = 0; d < s->ndom; ++d) dord[d] = d;
    if (s->order == 1)
        std::stable_sort(dord.begin(), dord.end(), [s](int a, int b) {
            return s->hdoms[a].numElem > s->hdoms[b].numElem;
        });
    std::vector<int2> eb, nb, gb, sb;
    for (int d : dord) {
        const DomDev &D = s->hdoms[d];
        for (int i = 0; i < D.numElem; i += s->eb) eb.push_back(make_int2(d, i));
        for (int i = 0; i < D.numNode; i += s->nb) nb.push_back(make_int2(d, i));
        if (D.tp > 1) {
            for (int f = 0; f < 6; ++f)
                if (D.ghost[f] >= 0)
                    for (int i = 0; i < D.nx * D.nx; i += kElemBlock)
                        gb.push_back(make_int2(d, (f << 24) | i));
            // the max-side node faces (k_posvel_sync): en^2, nx*en, nx^2 nodes
            const int items[3] = {D.en * D.en, D.nx * D.en, D.nx * D.nx};
            for (int f = 0; f < 3; ++f)
                for (int i = 0; i < items[f]; i += kNodeBlock) sb.push_back(make_int2(d, (f << 24) | i));
        }
    }
    // node blocks last-to-first (LULESH_NODAL_REVERSE, set.hpp)
    if (LULESH_NODAL_REVERSE) std::reverse(nb.begin(), nb.end());
    s->n_elem_blocks = (int)eb.size();
    s->n_node_blocks = (int)nb.size();
    s->n_ghost_blocks = (int)gb.size();
    s->n_sync_blocks = (int)sb.size();
    size_t bytes = sizeof(int2) * (eb.size() + nb.size() + gb.size() + sb.size() + 1);
    if (s->elem_blocks) {  // rebuilding: the old tables may still be in use
        LCHECK(cudaStreamSynchronize(s->stream));
        LCHECK(cudaFree(s->elem_blocks));
        s->elem_blocks = nullptr;
    }
    int2 *t = nullptr;
    LCHECK(cudaMalloc(&t, bytes));
    s->elem_blocks = t;
    s->node_blocks = t + eb.size();
    s->ghost_blocks = t + eb.size() + nb.size();
    s->sync_blocks = t + eb.size() + nb.size() + gb.size();
    LCHECK(cudaMemcpyAsync(s->elem_blocks, eb.data(), sizeof(int2) * eb.size(),
                           cudaMemcpyHostToDevice, s->stream));
    LCHECK(cudaMemcpyAsync(s->node_blocks, nb.data(), sizeof(int2) * nb.size(),
                           cudaMemcpyHostToDevice, s->stream));
    if (!gb.empty())
        LCHECK(cudaMemcpyAsync(s->ghost_blocks, gb.data(), sizeof(int2) * gb.size(),
                               cudaMemcpyHostToDevice, s->stream));
    if (!sb.empty())
        LCHECK(cudaMemcpyAsync(s->sync_blocks, sb.data(), sizeof(int2) * sb.size(),
                               cudaMemcpyHostToDevice, s->stream));
    return LULESH_OK;
}

// Fill the arena for every domain.  `layout[d]` gives (job, tp, col, row,
// plane, rank) of domain d.
struct DomPlace {
    int job, tp, col, row, plane, rank;
};

static int create_common(lulesh_set *s, const std::vector<DomPlace> &place, int device)
{
    if (device >= 0) LCHECK(cudaSetDevice(device));
    LCHECK(cudaGetDevice(&s->device));
    if (!s->stream) {
        LCHECK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->own_stream = true;
    }
    s->P = default_params();
    s->ndom = (int)place.size();
    const bool mixed = (s->flags & LULESH_FLAG_MIXED) != 0;

    // arena (an lmesh domain is read first: the file gives its sizes)
    size_t total = 0;
    std::vector<long> commd(s->ndom);
    HostDomain mesh;
    if (s->unstructured) {
        const lulesh_job &j = s->jobs[0];
        std::string err;
        if (!build_domain_lmesh(mesh, s->mesh_path.c_str(), j.numReg, j.balance, j.cost,
                                &err)) {
            set_error(err);
            return LULESH_FILE_ERROR;
        }
        commd[0] = 0;
        total = domain_bytes(sizes_of(mesh, 0), mixed);
        unsigned long long h = 1469598103934665603ull;
        auto mix = [&h](const void *p, size_t n) {
            const unsigned char *b = static_cast<const unsigned char *>(p);
            for (size_t i = 0; i < n; ++i) h = (h ^ b[i]) * 1099511628211ull;
        };
        mix(&mesh.numElem, sizeof mesh.numElem);
        mix(&mesh.numNode, sizeof mesh.numNode);
        mix(mesh.nodelist.data(), sizeof(int) * mesh.nodelist.size());
        mix(mesh.x.data(), sizeof(double) * mesh.x.size());
        mix(mesh.y.data(), sizeof(double) * mesh.y.size());
        mix(mesh.z.data(), sizeof(double) * mesh.z.size());
        s->mesh_hash = h;
    } else {
        for (int d = 0; d < s->ndom; ++d) {
            const lulesh_job &j = s->jobs[place[d].job];
            commd[d] = comm_buffer_doubles(j.nx, place[d].tp);
            total += domain_bytes(sizes_of(j.nx, j.numReg, commd[d]), mixed);
        }
    }
    s->arena_bytes = total;
    LCHECK(cudaMalloc(&s->arena, total));
    if (mixed) LCHECK(cudaMalloc(&s->dcorner32, sizeof(CornerF32) * s->ndom));

    // subdomain sets: every domain's x..zd side by side at the start of the
    // arena (the node region), so one L2 window can cover them all; the
    // arena's size is the same, the rest of each domain follows
    size_t node_region = 0;
    if (!s->unstructured && s->tp > 1)
        for (int d = 0; d < s->ndom; ++d) {
            const size_t e1 = (size_t)s->jobs[place[d].job].nx + 1;
            node_region += node_region_bytes(e1 * e1 * e1);
        }
    Carver ncv{static_cast<char *>(s->arena)};
    Carver cv{static_cast<char *>(s->arena) + node_region};
    s->node_region_bytes = node_region;
    s->hdoms.resize(s->ndom);
    s->dom_rank.resize(s->ndom);
    s->dom_job.resize(s->ndom);
    s->job_origin.assign(s->njobs, -1);
    std::vector<CornerF32> hc32(s->ndom);
    std::vector<double> job_dt(s->njobs, 0.0);

    for (int d = 0; d < s->ndom; ++d) {
        const DomPlace &pl = place[d];
        const lulesh_job &j = s->jobs[pl.job];
        HostDomain h;
        if (s->unstructured)
            h = std::move(mesh);
        else if (pl.tp == 1 && !(s->flags & LULESH_FLAG_HOST_SETUP))
            build_domain_light(h, j.nx, j.numReg, j.balance, j.cost);
        else
            // subdomains: the nodal mass over the whole problem is summed on
            // the device (nodal_mass_on_device) unless the host builds it all
            build_domain(h, j.nx, pl.tp, pl.col, pl.row, pl.plane, pl.rank, j.numReg, j.balance,
                         j.cost,
                         /*global_mass=*/pl.tp > 1 && (s->flags & LULESH_FLAG_HOST_SETUP));
        DomDev D{};
        int su = upload_domain(h, pl.job, commd[d], mixed, cv, s->stream, &D, &hc32[d],
                               node_region ? &ncv : nullptr);
        if (su != LULESH_OK) return su;
        s->hdoms[d] = D;
        s->dom_rank[d] = pl.rank;
        s->dom_job[d] = pl.job;
        if (pl.col == 0 && pl.row == 0 && pl.plane == 0) {
            s->job_origin[pl.job] = d;
            job_dt[pl.job] = h.deltatime;  // the origin domain's initial dt
        }
    }
    // a part of a problem split over GPUs: the job's dt starts from the
    // origin domain's even where that domain lives on another part
    for (int j = 0; j < s->njobs; ++j)
        if (s->job_origin[j] < 0) job_dt[j] = origin_deltatime(s->jobs[j].nx, s->tp);
    // proxies of the neighbours held by other parts, and the halo tables
    if (s->nparts > 1) {
        const int pst = part_build(s);
        if (pst != LULESH_OK) return pst;
    }
    // neighbour tables of subdomain sets (rank = col + tp*(row + tp*plane)):
    // a local neighbour of rank r is domain r - first_rank, a remote one
    // its proxy
    auto index_of_rank = [s](int r) -> int {
        if (halo_part_of(r, s->tp, s->nparts) == s->part) return r - s->first_rank;
        for (size_t k = 0; k < s->proxy_rank.size(); ++k)
            if (s->proxy_rank[k] == r) return s->ndom + (int)k;
        return -1;
    };
    for (int d = 0; d < s->ndom; ++d) {
        DomDev &D = s->hdoms[d];
        if (D.tp <= 1) continue;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int c = D.col + dx, r = D.row + dy, p = D.plane + dz;
                    int nbr = -1;
                    if (c >= 0 && r >= 0 && p >= 0 && c < D.tp && r < D.tp && p < D.tp &&
                        !(dx == 0 && dy == 0 && dz == 0))
                        nbr = index_of_rank(c + D.tp * (r + D.tp * p));
                    D.nbr[(dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)] = nbr;
                }
    }
    const size_t ntab = s->hdoms.size() + s->hproxies.size();
    LCHECK(cudaMalloc(&s->ddoms, sizeof(DomDev) * ntab));
    LCHECK(cudaMemcpyAsync(s->ddoms, s->hdoms.data(), sizeof(DomDev) * s->ndom,
                           cudaMemcpyHostToDevice, s->stream));
    if (!s->hproxies.empty())
        LCHECK(cudaMemcpyAsync(s->ddoms + s->ndom, s->hproxies.data(),
                               sizeof(DomDev) * s->hproxies.size(), cudaMemcpyHostToDevice,
                               s->stream));
    if (mixed)
        LCHECK(cudaMemcpyAsync(s->dcorner32, hc32.data(), sizeof(CornerF32) * s->ndom,
                               cudaMemcpyHostToDevice, s->stream));

    // time control blocks
    std::vector<TimeCtl> tc(s->njobs);
    for (int j = 0; j < s->njobs; ++j) tc[j] = initial_timectl(job_dt[j], s->jobs[j].its);
    LCHECK(cudaMalloc(&s->dtc, sizeof(TimeCtl) * s->njobs));
    LCHECK(cudaMallocHost(&s->htc_pinned, sizeof(TimeCtl) * s->njobs));
    LCHECK(cudaMemcpyAsync(s->dtc, tc.data(), sizeof(TimeCtl) * s->njobs,
                           cudaMemcpyHostToDevice, s->stream));
    int st = build_tables(s);
    if (st != LULESH_OK) return st;
    // subdomains: the init-time nodal mass exchange (lulesh.cu:4811-4831)
    // as a gather over the neighbours, on the device; a part of several
    // GPUs does it once its proxies hold the neighbours' volumes
    if (s->tp > 1 && !(s->flags & LULESH_FLAG_HOST_SETUP)) {
        if (s->nparts > 1) {
            s->mass_pending = true;
        } else if ((st = nodal_mass_on_device(s)) != LULESH_OK) {
            return st;
        }
    }
    LCHECK(cudaStreamSynchronize(s->stream));
    return LULESH_OK;
}

void launch_force_fp64(lulesh_set *s, cudaStream_t st)
{
    launch_force(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st, s->eb, s->unstructured);
}

int enqueue_cycle(lulesh_set *s)
{
    if (s->flags & LULESH_FLAG_COMM_STAGED) return enqueue_cycle_staged(s);
    cudaStream_t st = s->stream;
    const bool mixed = (s->flags & LULESH_FLAG_MIXED) != 0;
    launch_time_increment(s->dtc, s->njobs, s->P, st, s->pdl);
    if (mixed)
        launch_force_mixed(s->args(s->elem_blocks), s->n_elem_blocks, s->P, s->dcorner32, st);
    else
        launch_force_fp64(s, st);
    if (mixed)
        launch_nodal_mixed(s->args(s->node_blocks), s->n_node_blocks, s->P, s->dcorner32, st);
    else
        launch_nodal(s->args(s->node_blocks), s->n_node_blocks, s->P, st, s->nb,
                         s->unstructured);
    if (LULESH_FUSED_POSVEL_SYNC && s->tp > 1 && s->n_sync_blocks > 0)
        launch_posvel_sync(s->args(s->sync_blocks), s->n_sync_blocks, st);
    if (mixed)
        launch_kinematics_mixed(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st);
    else
        launch_kinematics(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st, s->eb,
                              s->unstructured);
    if (LULESH_FUSED_MONOQ_GHOST && s->tp > 1 && s->n_ghost_blocks > 0)
        launch_monoq_ghost(s->args(s->ghost_blocks), s->n_ghost_blocks, st);
    launch_eos(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st, s->eb, s->unstructured,
               !LULESH_FUSED_MONOQ_GHOST && s->tp > 1);
    return cuda_status(cudaGetLastError(), "cycle launch");
}

// A single domain keeps its node coordinate and velocity arrays (x..zd,
// ~50 MB at -s 100, contiguous in the arena) persisting in L2: force reads
// them, nodal reads and writes them, kinematics reads them again, every
// cycle; so does a subdomain set, whose domains' x..zd share the node
// region at the start of the arena.  The access-policy window is a stream
// attribute, captured into the cycle graph's kernel nodes.  Only when
// those arrays take at most half of the L2: measured on B200, the window
// takes -s 100 (49.5 MB) from 332.0 to 327.4 us per cycle, but -s 120
// (85 MB) from 559.7 to 610.2 us (566.1 with the persisting lines capped at
// 48 MB); the results are the same.  Batches do not use it.
// 0 leaves every set's stream without an access-policy window
#ifndef LULESH_L2_WINDOW
#define LULESH_L2_WINDOW 1
#endif

// per device: sets holding a window, the persisting-L2 limit found before
// the first and the one set now
struct L2Limit {
    int sets = 0;
    size_t before = 0, now = 0;
};
static std::mutex g_l2_mu;
static L2Limit g_l2[64];

// Remove the window from the set's stream (it may be the caller's) and
// release the lines it made persistent.
static void clear_l2_window(lulesh_set *s)
{
    if (!s->l2_window || !s->stream) return;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != s->device) cudaSetDevice(s->device);
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.num_bytes = 0;
    cudaStreamSetAttribute(s->stream, cudaStreamAttributeAccessPolicyWindow, &v);
    cudaCtxResetPersistingL2Cache();
    {
        std::lock_guard<std::mutex> lock(g_l2_mu);
        L2Limit &g = g_l2[s->device];
        if (--g.sets == 0) {
            // the persisting share of L2 goes back to ordinary lines
            cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, g.before);
            g.now = g.before;
        }
    }
    if (prev >= 0 && prev != s->device) cudaSetDevice(prev);
    s->l2_window = false;
}

static int l2_node_window_on_device(lulesh_set *s);

// the limit and the stream attribute belong to the set's device: make it
// current for the call, whatever device the calling thread has
static int l2_node_window(lulesh_set *s)
{
    if (!LULESH_L2_WINDOW || (s->ndom != 1 && !s->node_region_bytes) || s->l2_window)
        return LULESH_OK;
    int prev = -1;
    LCHECK(cudaGetDevice(&prev));
    if (prev != s->device) LCHECK(cudaSetDevice(s->device));
    const int st = l2_node_window_on_device(s);
    if (prev != s->device) cudaSetDevice(prev);
    return st;
}

static int l2_node_window_on_device(lulesh_set *s)
{
    if (s->device < 0 || s->device >= 64) return LULESH_OK;
    const DomDev &D = s->hdoms[0];
    const char *lo = reinterpret_cast<const char *>(D.x);
    const char *hi = reinterpret_cast<const char *>(D.zd + D.numNode);
    if (s->node_region_bytes) {  // every domain's x..zd: the node region
        lo = static_cast<const char *>(s->arena);
        hi = lo + s->node_region_bytes;
    }
    int maxwin = 0, maxpersist = 0, l2 = 0;
    LCHECK(cudaDeviceGetAttribute(&maxwin, cudaDevAttrMaxAccessPolicyWindowSize, s->device));
    LCHECK(cudaDeviceGetAttribute(&maxpersist, cudaDevAttrMaxPersistingL2CacheSize, s->device));
    LCHECK(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, s->device));
    if (maxwin <= 0 || maxpersist <= 0 || l2 <= 0) return LULESH_OK;
    size_t bytes = (size_t)(hi - lo);
    if (bytes > (size_t)l2 / 2) return LULESH_OK;
    if (bytes > (size_t)maxwin) bytes = (size_t)maxwin;
    const size_t persist = bytes < (size_t)maxpersist ? bytes : (size_t)maxpersist;
    // a limit of the process's context: raised while any set on this device
    // holds a window, and put back to what it was when the last one goes
    {
        std::lock_guard<std::mutex> lock(g_l2_mu);
        L2Limit &g = g_l2[s->device];
        if (g.sets == 0) {
            LCHECK(cudaDeviceGetLimit(&g.before, cudaLimitPersistingL2CacheSize));
            g.now = g.before;
        }
        if (persist > g.now) {
            LCHECK(cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, persist));
            g.now = persist;
        }
        ++g.sets;
        s->l2_window = true;  // counted: clear_l2_window undoes it
    }
    cudaStreamAttrValue v{};
    v.accessPolicyWindow.base_ptr = const_cast<char *>(lo);
    v.accessPolicyWindow.num_bytes = bytes;
    v.accessPolicyWindow.hitRatio = (float)((double)persist / (double)bytes);
    v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    const cudaError_t e = cudaStreamSetAttribute(s->stream, cudaStreamAttributeAccessPolicyWindow, &v);
    if (e != cudaSuccess) {
        clear_l2_window(s);
        return cuda_status(e, "cudaStreamSetAttribute(accessPolicyWindow)");
    }
    return LULESH_OK;
}

static int ensure_graph(lulesh_set *s)
{
    if (s->graph_ready) return LULESH_OK;
    if (s->nparts > 1) {
        set_error("a part of a multi-GPU problem has no one-GPU cycle graph");
        return LULESH_INVALID_ARG;
    }
    const int pst = prepare_capture(s);
    if (pst != LULESH_OK) return pst;
    LCHECK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int st = enqueue_cycle(s);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (st != LULESH_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    LCHECK(e);
    s->graph = g;
    LCHECK(cudaGraphInstantiate(&s->exec, g, 0));
    s->graph_ready = true;
    return LULESH_OK;
}

// graph of graph_cycles consecutive cycles (one launch for many cycles)
static int ensure_graph_k(lulesh_set *s)
{
    if (s->graph_k_ready || s->graph_cycles <= 1) return LULESH_OK;
    int st = ensure_graph(s);  // prepares comm tables when staged
    if (st != LULESH_OK) return st;
    LCHECK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    for (int c = 0; c < s->graph_cycles && st == LULESH_OK; ++c) st = enqueue_cycle(s);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &g);
    if (st != LULESH_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    LCHECK(e);
    s->graph_k = g;
    LCHECK(cudaGraphInstantiate(&s->exec_k, g, 0));
    s->graph_k_ready = true;
    return LULESH_OK;
}

void drop_graph(lulesh_set *s)
{
    if (s->exec_k) cudaGraphExecDestroy(s->exec_k);
    if (s->graph_k) cudaGraphDestroy(s->graph_k);
    s->exec_k = nullptr;
    s->graph_k = nullptr;
    s->graph_k_ready = false;
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->exec = nullptr;
    s->graph = nullptr;
    s->graph_ready = false;
    if (s->exec_run) cudaGraphExecDestroy(s->exec_run);
    if (s->graph_run) cudaGraphDestroy(s->graph_run);
    s->exec_run = nullptr;
    s->graph_run = nullptr;
}

int prepare_capture(lulesh_set *s)
{
    const int wst = l2_node_window(s);
    if (wst != LULESH_OK) return wst;
    if (s->flags & LULESH_FLAG_COMM_STAGED) return comm_prepare(s);
    return LULESH_OK;
}

static int read_states(lulesh_set *s)
{
    LCHECK(cudaMemcpyAsync(s->htc_pinned, s->dtc, sizeof(TimeCtl) * s->njobs,
                           cudaMemcpyDeviceToHost, s->stream));
    LCHECK(cudaStreamSynchronize(s->stream));
    return LULESH_OK;
}

static void fill_state(const TimeCtl &T, lulesh_job_state *o)
{
    o->status = T.status;
    o->bad_elem = (T.status == -1) ? T.bad_vol : (T.status == -2 ? T.bad_q : -1);
    if (T.status == 0 && T.bad_vol != INT_MAX) {
        o->status = -1;
        o->bad_elem = T.bad_vol;
    } else if (T.status == 0 && T.bad_q != INT_MAX) {
        o->status = -2;
        o->bad_elem = T.bad_q;
    }
    o->cycle = T.cycle;
    o->done = T.done;
    o->time = T.time;
    o->deltatime = T.deltatime;
    o->dtcourant = T.dtcourant;
    o->dthydro = T.dthydro;
}

int run_status(lulesh_set *s)
{
    const int st = read_states(s);
    if (st != LULESH_OK) return st;
    for (int j = 0; j < s->njobs; ++j) {
        lulesh_job_state o;
        fill_state(s->htc_pinned[j], &o);
        if (o.status != LULESH_OK) return o.status;
    }
    return LULESH_OK;
}

// ---- field table ----------------------------------------------------------

struct FieldRef {
    void *ptr;
    size_t bytes;
};

static bool field_of(const lulesh_set *s, int d, const char *name, FieldRef *out)
{
    const DomDev &D = s->hdoms[d];
    const size_t E = D.numElem, N = D.numNode, Ep = D.Ep, A = D.allElem;
    // symmetry sets: en^2 on -s meshes, the largest set of an lmesh
    const size_t en2 =
        D.unstructured
            ? (size_t)std::max(1, std::max(D.numSymmX, std::max(D.numSymmY, D.numSymmZ)))
            : (size_t)D.en * D.en;
    const size_t nr = D.numReg;
    struct Row {
        const char *n;
        void *p;
        size_t b;
    } rows[] = {
        {"e", D.e, 8 * E}, {"p", D.p, 8 * E}, {"q", D.q, 8 * E}, {"ql", D.ql, 8 * E},
        {"qq", D.qq, 8 * E}, {"v", D.v, 8 * E}, {"volo", D.volo, 8 * E},
        {"delv", D.delv, 8 * E}, {"vdov", D.vdov, 8 * E}, {"arealg", D.arealg, 8 * E},
        {"ss", D.ss, 8 * E}, {"elemMass", D.elemMass, 8 * E}, {"vnew", D.vnew, 8 * E},
        {"delx_xi", D.delx_xi, 8 * E}, {"delx_eta", D.delx_eta, 8 * E},
        {"delx_zeta", D.delx_zeta, 8 * E}, {"delv_xi", D.delv_xi, 8 * A},
        {"delv_eta", D.delv_eta, 8 * A}, {"delv_zeta", D.delv_zeta, 8 * A},
        {"x", D.x, 8 * N}, {"y", D.y, 8 * N}, {"z", D.z, 8 * N}, {"xd", D.xd, 8 * N},
        {"yd", D.yd, 8 * N}, {"zd", D.zd, 8 * N}, {"xdd", D.xdd, 8 * N},
        {"ydd", D.ydd, 8 * N}, {"zdd", D.zdd, 8 * N}, {"fx", D.fx, 8 * N},
        {"fy", D.fy, 8 * N}, {"fz", D.fz, 8 * N}, {"nodalMass", D.nodalMass, 8 * N},
        {"fx_elem", D.fx_elem, 64 * Ep}, {"fy_elem", D.fy_elem, 64 * Ep},
        {"fz_elem", D.fz_elem, 64 * Ep}, {"nodelist", D.nodelist, 32 * Ep},
        {"lxim", D.lxim, 4 * E}, {"lxip", D.lxip, 4 * E}, {"letam", D.letam, 4 * E},
        {"letap", D.letap, 4 * E}, {"lzetam", D.lzetam, 4 * E}, {"lzetap", D.lzetap, 4 * E},
        {"elemBC", D.elemBC, 4 * E}, {"matElemlist", D.matElemlist, 4 * E},
        {"regNumList", D.regNumList, 4 * E}, {"regElemlist", D.regElemlist, 4 * E},
        {"eosOrder", D.eosOrder, 4 * E}, {"nodeElemCount", D.nodeElemCount, 4 * N}, {"nodeElemStart", D.nodeElemStart, 4 * N},
        {"nodeElemCornerList", D.nodeElemCornerList, 32 * E}, {"symmX", D.symmX, 4 * en2},
        {"symmY", D.symmY, 4 * en2}, {"symmZ", D.symmZ, 4 * en2},
        {"regCSR", D.regCSR, 4 * nr}, {"regReps", D.regReps, 4 * nr},
        {"regSorted", D.regSorted, 4 * nr},
    };
    for (const Row &r : rows)
        if (std::strcmp(r.n, name) == 0) {
            out->ptr = r.p;
            out->bytes = r.b;
            return true;
        }
    return false;
}

}  // namespace lulesh

using namespace lulesh;

// ============================================================================
// C ABI

extern "C" {

const char *lulesh_last_error(void) { return g_last_error.c_str(); }

const char *lulesh_status_string(int st)
{
    switch (st) {
        case LULESH_OK: return "ok";
        case LULESH_VOLUME_ERROR: return "VolumeError";
        case LULESH_QSTOP_ERROR: return "QStopError";
        case LULESH_FILE_ERROR: return "LFileError";
        case LULESH_CUDA_ERROR: return "CUDA error";
        case LULESH_INVALID_ARG: return "invalid argument";
        case LULESH_OOM: return "out of device memory";
        case LULESH_TIMEOUT: return "timeout";
        case LULESH_NO_DEVICE: return "no CUDA device";
        case LULESH_BOUNDS_ERROR: return "index out of range (checked build)";
        default: return "unknown status";
    }
}

size_t lulesh_footprint_bytes(const lulesh_job *jobs, int njobs, int tp)
{
    if (!jobs || njobs <= 0 || tp < 1) return 0;
    size_t total = 0;
    for (int j = 0; j < njobs; ++j) {
        const long comm = comm_buffer_doubles(jobs[j].nx, tp);
        const size_t per = domain_bytes(sizes_of(jobs[j].nx, jobs[j].numReg, comm), false);
        total += per * (size_t)tp * tp * tp;
        // block tables, domain records and time control
        const size_t E = (size_t)jobs[j].nx * jobs[j].nx * jobs[j].nx;
        const size_t N = (size_t)(jobs[j].nx + 1) * (jobs[j].nx + 1) * (jobs[j].nx + 1);
        total += tp * tp * tp * (8 * (E / kElemBlock + N / kNodeBlock + 2) + sizeof(DomDev)) +
                 sizeof(TimeCtl);
    }
    return total;
}

int lulesh_create(const lulesh_job *job, int tp, int flags, int device, lulesh_set **out)
{
    if (!job || !out || tp < 1 || tp > 16) {
        set_error("lulesh_create: bad arguments");
        return LULESH_INVALID_ARG;
    }
    *out = nullptr;
    int st = validate_job(*job);
    if (st != LULESH_OK) return st;
    if ((flags & LULESH_FLAG_MIXED) && tp > 1) {
        set_error("mixed precision runs on single domains and batches");
        return LULESH_INVALID_ARG;
    }
    lulesh_set *s = new lulesh_set;
    s->flags = flags;
    s->tp = tp;
    s->njobs = 1;
    s->jobs.push_back(*job);
    std::vector<DomPlace> place;
    const int n = tp * tp * tp;
    for (int r = 0; r < n; ++r) {
        // InitMeshDecomp, lulesh.cu:4653-4664 (one domain per rank)
        place.push_back(DomPlace{0, tp, r % tp, (r / tp) % tp, r / (tp * tp), r});
    }
    st = create_common(s, place, device);
    if (st != LULESH_OK) {
        lulesh_destroy(s);
        return st;
    }
    *out = s;
    return LULESH_OK;
}

int lulesh_create_part(const lulesh_job *job, int tp, int nparts, int part, int flags,
                       int device, lulesh_set **out)
{
    if (!job || !out || tp < 1 || tp > 16 || nparts < 1 || nparts > tp * tp * tp || part < 0 ||
        part >= nparts) {
        set_error("lulesh_create_part: bad arguments (1 <= nparts <= tp^3, 0 <= part < nparts)");
        return LULESH_INVALID_ARG;
    }
    *out = nullptr;
    if (nparts == 1) return lulesh_create(job, tp, flags, device, out);
    int st = validate_job(*job);
    if (st != LULESH_OK) return st;
    if (flags & (LULESH_FLAG_MIXED | LULESH_FLAG_COMM_STAGED)) {
        set_error("a part of a multi-GPU problem runs FP64 with the fused exchange");
        return LULESH_INVALID_ARG;
    }
    lulesh_set *s = new lulesh_set;
    s->flags = flags;
    s->tp = tp;
    s->njobs = 1;
    s->nparts = nparts;
    s->part = part;
    s->jobs.push_back(*job);
    // this part's run of consecutive ranks (halo_part_of)
    std::vector<DomPlace> place;
    s->first_rank = -1;
    for (int r = 0; r < tp * tp * tp; ++r) {
        if (halo_part_of(r, tp, nparts) != part) continue;
        if (s->first_rank < 0) s->first_rank = r;
        place.push_back(DomPlace{0, tp, r % tp, (r / tp) % tp, r / (tp * tp), r});
    }
    st = create_common(s, place, device);
    if (st != LULESH_OK) {
        lulesh_destroy(s);
        return st;
    }
    *out = s;
    return LULESH_OK;
}

int lulesh_create_batch(const lulesh_job *jobs, int njobs, int flags, int device,
                        lulesh_set **out)
{
    if (!jobs || !out || njobs < 1) {
        set_error("lulesh_create_batch: bad arguments");
        return LULESH_INVALID_ARG;
    }
    *out = nullptr;
    for (int j = 0; j < njobs; ++j) {
        int st = validate_job(jobs[j]);
        if (st != LULESH_OK) return st;
    }
    if (flags & LULESH_FLAG_COMM_STAGED) {
        set_error("batches have no halo exchange");
        return LULESH_INVALID_ARG;
    }
    lulesh_set *s = new lulesh_set;
    s->flags = flags;
    s->tp = 1;
    s->njobs = njobs;
    s->jobs.assign(jobs, jobs + njobs);
    std::vector<DomPlace> place;
    for (int j = 0; j < njobs; ++j) place.push_back(DomPlace{j, 1, 0, 0, 0, 0});
    int st = create_common(s, place, device);
    if (st != LULESH_OK) {
        lulesh_destroy(s);
        return st;
    }
    *out = s;
    return LULESH_OK;
}

int lulesh_create_from_mesh(const char *path, const lulesh_job *job, int flags, int device,
                            lulesh_set **out)
{
    if (!path || !job || !out) {
        set_error("lulesh_create_from_mesh: bad arguments");
        return LULESH_INVALID_ARG;
    }
    *out = nullptr;
    lulesh_job j = *job;
    j.nx = 1;  // the mesh file gives the sizes
    int st = validate_job(j);
    if (st != LULESH_OK) return st;
    if (flags & (LULESH_FLAG_COMM_STAGED | LULESH_FLAG_MIXED)) {
        set_error("unstructured meshes run as one FP64 domain");
        return LULESH_INVALID_ARG;
    }
    lulesh_set *s = new lulesh_set;
    s->flags = flags;
    s->tp = 1;
    s->njobs = 1;
    s->jobs.assign(1, j);
    s->mesh_path = path;
    s->unstructured = true;
    st = create_common(s, {DomPlace{0, 1, 0, 0, 0, 0}}, device);
    if (st != LULESH_OK) {
        lulesh_destroy(s);
        return st;
    }
    *out = s;
    return LULESH_OK;
}

int lulesh_destroy(lulesh_set *s)
{
    if (!s) return LULESH_OK;
    if (s->stream) cudaStreamSynchronize(s->stream);
    drop_graph(s);
    clear_l2_window(s);
    comm_release(s);
    part_release(s);
    if (s->elem_blocks) cudaFree(s->elem_blocks);
    if (s->ddoms) cudaFree(s->ddoms);
    if (s->dtc) cudaFree(s->dtc);
    if (s->htc_pinned) cudaFreeHost(s->htc_pinned);
    if (s->dcorner32) cudaFree(s->dcorner32);
    if (s->run_ctl) cudaFree(s->run_ctl);
    if (s->arena) cudaFree(s->arena);
    if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return LULESH_OK;
}

int lulesh_set_stream(lulesh_set *s, void *stream)
{
    if (!s) return LULESH_INVALID_ARG;
    LCHECK(cudaStreamSynchronize(s->stream));
    drop_graph(s);
    clear_l2_window(s);
    if (s->own_stream) cudaStreamDestroy(s->stream);
    if (stream) {
        s->stream = static_cast<cudaStream_t>(stream);
        s->own_stream = false;
    } else {
        LCHECK(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        s->own_stream = true;
    }
    return LULESH_OK;
}

int lulesh_lagrange_leapfrog(lulesh_set *s) { return lulesh_step(s, 1); }

int lulesh_step(lulesh_set *s, int ncycles)
{
    if (!s || ncycles < 0) return LULESH_INVALID_ARG;
    if (s->nparts > 1) {
        set_error("a part of a multi-GPU problem advances through lulesh_part_phase and the "
                  "halo exchange");
        return LULESH_INVALID_ARG;
    }
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    LCHECK(cudaStreamIsCapturing(s->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) {
        // the caller is capturing the set's stream into a graph of its own:
        // the cycle's kernels become nodes of that graph
        if (!s->graph_ready) {
            set_error("lulesh_step: call lulesh_step(set, 0) before capturing the set's stream");
            return LULESH_INVALID_ARG;
        }
        for (int i = 0; i < ncycles; ++i) {
            const int est = enqueue_cycle(s);
            if (est != LULESH_OK) return est;
        }
        return LULESH_OK;
    }
    int st = ensure_graph(s);
    if (st != LULESH_OK) return st;
    if (s->graph_cycles > 1 && ncycles >= s->graph_cycles) {
        if ((st = ensure_graph_k(s)) != LULESH_OK) return st;
        for (; ncycles >= s->graph_cycles; ncycles -= s->graph_cycles)
            LCHECK(cudaGraphLaunch(s->exec_k, s->stream));
    }
    for (int i = 0; i < ncycles; ++i) LCHECK(cudaGraphLaunch(s->exec, s->stream));
    return LULESH_OK;
}

int lulesh_set_graph_cycles(lulesh_set *s, int k)
{
    if (!s || k < 1 || k > 100000) return LULESH_INVALID_ARG;
    if (k != s->graph_cycles) {
        LCHECK(cudaStreamSynchronize(s->stream));
        if (s->exec_k) cudaGraphExecDestroy(s->exec_k);
        if (s->graph_k) cudaGraphDestroy(s->graph_k);
        s->exec_k = nullptr;
        s->graph_k = nullptr;
        s->graph_k_ready = false;
        s->graph_cycles = k;
    }
    return LULESH_OK;
}

int lulesh_sync(lulesh_set *s)
{
    if (!s) return LULESH_INVALID_ARG;
    LCHECK(cudaStreamSynchronize(s->stream));
    return LULESH_OK;
}

int lulesh_run(lulesh_set *s, int check_every)
{
    if (!s) return LULESH_INVALID_ARG;
    if (check_every <= 0) check_every = 64;
    for (;;) {
        int st = lulesh_step(s, check_every);
        if (st != LULESH_OK) return st;
        st = read_states(s);
        if (st != LULESH_OK) return st;
        bool all_done = true;
        for (int j = 0; j < s->njobs; ++j)
            if (!s->htc_pinned[j].done) all_done = false;
        if (all_done) break;
    }
    return run_status(s);
}

int lulesh_host_cycle(lulesh_set *s, const lulesh_job_state *in, lulesh_job_state *out)
{
    if (!s || s->njobs != 1) {
        set_error("lulesh_host_cycle drives one job");
        return LULESH_INVALID_ARG;
    }
    int st = ensure_graph(s);
    if (st != LULESH_OK) return st;
    if (in) {
        // host -> device: the time state the host decided on
        TimeCtl &T = s->htc_pinned[0];
        T.time = in->time;
        T.deltatime = in->deltatime;
        LCHECK(cudaMemcpyAsync(&s->dtc[0].time, &T.time, 2 * sizeof(double),
                               cudaMemcpyHostToDevice, s->stream));
    }
    LCHECK(cudaGraphLaunch(s->exec, s->stream));
    // device -> host: the whole time-control record (dt, time, status)
    LCHECK(cudaMemcpyAsync(s->htc_pinned, s->dtc, sizeof(TimeCtl), cudaMemcpyDeviceToHost,
                           s->stream));
    LCHECK(cudaStreamSynchronize(s->stream));
    if (out) fill_state(s->htc_pinned[0], out);
    lulesh_job_state tmp;
    fill_state(s->htc_pinned[0], &tmp);
    return tmp.status;
}

static const char *kPhaseNames[] = {"time_increment", "force", "nodal", "posvel_sync",
                                    "kinematics", "monoq_ghost", "eos"};

const char *lulesh_phase_name(int phase)
{
    if (phase < 0 || phase >= (int)(sizeof kPhaseNames / sizeof kPhaseNames[0])) return "";
    return kPhaseNames[phase];
}

int lulesh_profile_phases(lulesh_set *s, int ncycles, double *ms_out, int *nphases)
{
    if (!s || !ms_out || !nphases || ncycles < 1) return LULESH_INVALID_ARG;
    if (s->flags & LULESH_FLAG_COMM_STAGED) {
        set_error("phase profiling covers the fused cycle");
        return LULESH_INVALID_ARG;
    }
    const int np = 7;
    cudaEvent_t ev[np + 1];
    for (int k = 0; k <= np; ++k) LCHECK(cudaEventCreate(&ev[k]));
    double acc[np] = {0};
    cudaStream_t st = s->stream;
    const bool mixed = (s->flags & LULESH_FLAG_MIXED) != 0;
    for (int c = 0; c < ncycles; ++c) {
        LCHECK(cudaEventRecord(ev[0], st));
        launch_time_increment(s->dtc, s->njobs, s->P, st, s->pdl);
        LCHECK(cudaEventRecord(ev[1], st));
        if (mixed)
            launch_force_mixed(s->args(s->elem_blocks), s->n_elem_blocks, s->P, s->dcorner32, st);
        else
            launch_force_fp64(s, st);
        LCHECK(cudaEventRecord(ev[2], st));
        if (mixed)
            launch_nodal_mixed(s->args(s->node_blocks), s->n_node_blocks, s->P, s->dcorner32, st);
        else
            launch_nodal(s->args(s->node_blocks), s->n_node_blocks, s->P, st, s->nb,
                         s->unstructured);
        LCHECK(cudaEventRecord(ev[3], st));
        if (LULESH_FUSED_POSVEL_SYNC && s->tp > 1 && s->n_sync_blocks > 0)
            launch_posvel_sync(s->args(s->sync_blocks), s->n_sync_blocks, st);
        LCHECK(cudaEventRecord(ev[4], st));
        if (mixed)
            launch_kinematics_mixed(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st);
        else
            launch_kinematics(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st, s->eb,
                              s->unstructured);
        LCHECK(cudaEventRecord(ev[5], st));
        if (LULESH_FUSED_MONOQ_GHOST && s->tp > 1 && s->n_ghost_blocks > 0)
            launch_monoq_ghost(s->args(s->ghost_blocks), s->n_ghost_blocks, st);
        LCHECK(cudaEventRecord(ev[6], st));
        launch_eos(s->args(s->elem_blocks), s->n_elem_blocks, s->P, st, s->eb, s->unstructured,
                   !LULESH_FUSED_MONOQ_GHOST && s->tp > 1);
        LCHECK(cudaEventRecord(ev[7], st));
        LCHECK(cudaEventSynchronize(ev[7]));
        for (int k = 0; k < np; ++k) {
            float ms = 0.f;
            LCHECK(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
            acc[k] += ms;
        }
    }
    for (int k = 0; k <= np; ++k) cudaEventDestroy(ev[k]);
    for (int k = 0; k < np; ++k) ms_out[k] = acc[k] / ncycles;
    *nphases = np;
    return LULESH_OK;
}

int lulesh_num_jobs(const lulesh_set *s) { return s ? s->njobs : 0; }
int lulesh_num_domains(const lulesh_set *s) { return s ? s->ndom : 0; }

int lulesh_job_state_get(lulesh_set *s, int job, lulesh_job_state *out)
{
    if (!s || !out || job < 0 || job >= s->njobs) return LULESH_INVALID_ARG;
    int st = read_states(s);
    if (st != LULESH_OK) return st;
    fill_state(s->htc_pinned[job], out);
    return LULESH_OK;
}

// the job's origin domain is on another part of a multi-GPU problem
static bool origin_missing(const lulesh_set *s, int job)
{
    if (s->job_origin[job] >= 0) return false;
    set_error("this part does not hold the subdomain at the mesh origin (rank 0)");
    return true;
}

int lulesh_origin_energy(lulesh_set *s, int job, double *energy)
{
    if (!s || !energy || job < 0 || job >= s->njobs) return LULESH_INVALID_ARG;
    if (origin_missing(s, job)) return LULESH_INVALID_ARG;
    const DomDev &D = s->hdoms[s->job_origin[job]];
    LCHECK(cudaStreamSynchronize(s->stream));
    LCHECK(cudaMemcpy(energy, D.e + D.octant, sizeof(double), cudaMemcpyDeviceToHost));
    return LULESH_OK;
}

int lulesh_symmetry(lulesh_set *s, int job, double *max_abs, double *total_abs, double *max_rel)
{
    if (!s || job < 0 || job >= s->njobs) return LULESH_INVALID_ARG;
    if (origin_missing(s, job)) return LULESH_INVALID_ARG;
    const DomDev &D = s->hdoms[s->job_origin[job]];
    if (D.unstructured) {
        set_error("the plane-0 symmetry check needs a structured (-s) mesh");
        return LULESH_INVALID_ARG;
    }
    const int nx = D.nx;
    std::vector<double> e((size_t)nx * nx);
    LCHECK(cudaStreamSynchronize(s->stream));
    LCHECK(cudaMemcpy(e.data(), D.e, sizeof(double) * e.size(), cudaMemcpyDeviceToHost));
    double ma = 0.0, ta = 0.0, mr = 0.0;
    for (int j = 0; j < nx; ++j)
        for (int k = j + 1; k < nx; ++k) {
            const double ad = std::fabs(e[j * nx + k] - e[k * nx + j]);
            ta += ad;
            if (ma < ad) ma = ad;
            const double rd = ad / e[k * nx + j];
            if (mr < rd) mr = rd;
        }
    if (max_abs) *max_abs = ma;
    if (total_abs) *total_abs = ta;
    if (max_rel) *max_rel = mr;
    return LULESH_OK;
}

int lulesh_field_bytes(lulesh_set *s, int d, const char *name, size_t *nbytes)
{
    if (!s || !name || !nbytes || d < 0 || d >= s->ndom) return LULESH_INVALID_ARG;
    FieldRef f;
    if (!field_of(s, d, name, &f)) {
        set_error(std::string("unknown field ") + name);
        return LULESH_INVALID_ARG;
    }
    *nbytes = f.bytes;
    return LULESH_OK;
}

int lulesh_get_field(lulesh_set *s, int d, const char *name, void *dst, size_t nbytes)
{
    if (!s || !name || !dst || d < 0 || d >= s->ndom) return LULESH_INVALID_ARG;
    FieldRef f;
    if (!field_of(s, d, name, &f) || f.bytes != nbytes) {
        set_error(std::string("field size/name mismatch: ") + name);
        return LULESH_INVALID_ARG;
    }
    LCHECK(cudaStreamSynchronize(s->stream));
    LCHECK(cudaMemcpy(dst, f.ptr, nbytes, cudaMemcpyDeviceToHost));
    return LULESH_OK;
}

int lulesh_set_field(lulesh_set *s, int d, const char *name, const void *src, size_t nbytes)
{
    if (!s || !name || !src || d < 0 || d >= s->ndom) return LULESH_INVALID_ARG;
    FieldRef f;
    if (!field_of(s, d, name, &f) || f.bytes != nbytes) {
        set_error(std::string("field size/name mismatch: ") + name);
        return LULESH_INVALID_ARG;
    }
    LCHECK(cudaStreamSynchronize(s->stream));
    LCHECK(cudaMemcpy(f.ptr, src, nbytes, cudaMemcpyHostToDevice));
    return LULESH_OK;
}

int lulesh_domain_view_get(lulesh_set *s, int d, lulesh_domain_view *o)
{
    if (!s || !o || d < 0 || d >= s->ndom) return LULESH_INVALID_ARG;
    const DomDev &D = s->hdoms[d];
    std::memset(o, 0, sizeof *o);
    o->numElem = D.numElem;
    o->numNode = D.numNode;
    o->padded_numElem = D.Ep;
    o->sizeX = o->sizeY = o->sizeZ = D.nx;
    o->colLoc = D.col;
    o->rowLoc = D.row;
    o->planeLoc = D.plane;
    o->tp = D.tp;
    o->numReg = D.numReg;
    o->allElem = D.allElem;
    o->numSymmX = D.numSymmX;
    o->numSymmY = D.numSymmY;
    o->numSymmZ = D.numSymmZ;
#define V(f) o->f = D.f
    V(nodelist); V(lxim); V(lxip); V(letam); V(letap); V(lzetam); V(lzetap); V(elemBC);
    V(nodeElemCount); V(nodeElemStart); V(nodeElemCornerList); V(symmX); V(symmY); V(symmZ);
    V(matElemlist); V(regCSR); V(regReps); V(regNumList); V(regElemlist); V(regSorted);
    V(e); V(p); V(q); V(ql); V(qq); V(v); V(volo); V(delv); V(vdov); V(arealg); V(ss);
    V(elemMass); V(x); V(y); V(z); V(xd); V(yd); V(zd); V(xdd); V(ydd); V(zdd); V(fx); V(fy);
    V(fz); V(nodalMass); V(vnew); V(delx_xi); V(delx_eta); V(delx_zeta); V(delv_xi);
    V(delv_eta); V(delv_zeta); V(fx_elem); V(fy_elem); V(fz_elem);
#undef V
    return LULESH_OK;
}

int lulesh_write_solution(lulesh_set *s, int d, const char *path)
{
    if (!s || !path || d < 0 || d >= s->ndom) return LULESH_INVALID_ARG;
    const DomDev &D = s->hdoms[d];
    std::vector<double> x(D.numNode), y(D.numNode), z(D.numNode);
    LCHECK(cudaStreamSynchronize(s->stream));
    LCHECK(cudaMemcpy(x.data(), D.x, 8 * x.size(), cudaMemcpyDeviceToHost));
    LCHECK(cudaMemcpy(y.data(), D.y, 8 * y.size(), cudaMemcpyDeviceToHost));
    LCHECK(cudaMemcpy(z.data(), D.z, 8 * z.size(), cudaMemcpyDeviceToHost));
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        set_error(std::string("cannot open ") + path);
        return LULESH_FILE_ERROR;
    }
    for (int i = 0; i < D.numNode; ++i)
        std::fprintf(f, "%10d\n%.10f\n%.10f\n%.10f\n", i, x[i], y[i], z[i]);
    std::fclose(f);
    return LULESH_OK;
}

}  // extern "C"
