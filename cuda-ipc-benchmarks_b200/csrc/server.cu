// server.cu -- continuous batching of sedov jobs on one GPU.
//
// Submitted jobs draw their region runs (glibc rand) on host worker threads
// (build_domain_light); their geometry and per-element region arrays are
// generated on the device at admission (setup.cu).  lulesh_server_step then
//   1. waits for the previous step, reads every slot's time control and
//      origin energy (one gather kernel + two small copies issued at the end
//      of that step) and retires finished jobs, freeing their memory;
//   2. when the resident set changed, rebuilds the domain table and block
//      tables, writes the time state of newly admitted jobs and re-captures
//      the cycle graph (updating the executable graph in place);
//   3. launches the cycle graph cycles_per_step times: every resident job,
//      whatever its size, advances in the same five launches per cycle;
//   4. while those cycles run, admits queued jobs in arrival order while a
//      slot is free and the job's device footprint fits under the cap
//      (stream-ordered allocations from a memory pool, uploaded on a side
//      stream); they join the tables at the next step.
// Kernels and arithmetic are those of a single-job set, so each job's
// result equals its own plain run bit for bit.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <climits>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "domain_dev.hpp"
#include "kernels.cuh"
#include "set.hpp"

namespace lulesh {

// elements per block of the served cycle's element kernels (64, 128 or 256)
#ifndef LULESH_SERVER_ELEM_BLOCK
#define LULESH_SERVER_ELEM_BLOCK 128
#endif
constexpr int kServerElemBlock = LULESH_SERVER_ELEM_BLOCK;
static_assert(valid_elem_block(kServerElemBlock), "64, 128 or 256 elements per block");

struct SJob {
    long long id = 0;
    lulesh_job job{};
    std::unique_ptr<HostDomain> host;
    std::atomic<bool> ready{false};
    size_t bytes = 0;
    void *mem = nullptr;
    int slot = -1;
    DomDev dom{};
    TimeCtl t0{};        // initial time state, written at the next rebuild
    bool fresh = false;  // admitted after the last graph launch
    double t_submit = 0, t_admit = 0;
};

static double mono_now()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

// origin energy e[0] of every resident domain into out[slot]
__global__ void k_gather_origin(const DomDev *doms, int n, double *out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[doms[i].tc] = doms[i].e[0];
}

}  // namespace lulesh

using namespace lulesh;

struct lulesh_server {
    lulesh_server_config cfg{};
    int device = 0;
    cudaStream_t stream = nullptr, upload = nullptr;
    cudaMemPool_t pool = nullptr;
    Params P{};
    // host meshing
    std::vector<std::thread> workers;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::shared_ptr<SJob>> prep_q;
    bool stop = false;
    // jobs
    std::deque<std::shared_ptr<SJob>> pending;
    std::vector<std::shared_ptr<SJob>> active;
    std::vector<int> free_slots;
    size_t used_bytes = 0;
    long long next_id = 0;
    std::vector<lulesh_server_result> results;
    // device tables
    TimeCtl *dtc = nullptr, *htc = nullptr;
    double *denergy = nullptr, *henergy = nullptr;
    DomDev *ddoms = nullptr;
    int2 *dblocks = nullptr;
    size_t blocks_cap = 0;
    int2 *node_b = nullptr, *elem_b = nullptr;
    int n_node = 0, n_elem = 0;
    int n_table = 0;  // domains in the launched tables
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool dirty = true;
    cudaEvent_t step_done = nullptr;
    bool in_flight = false;

    SetArgs args(const int2 *b) const
    {
        SetArgs a;
        a.doms = ddoms;
        a.tcs = dtc;
        a.blocks = b;
        a.materialize = 0;
        a.pdl = LULESH_PDL;  // the cycle kernels overlap each other's tails
        return a;
    }
};

#define SCHECK(call)                                            \
    do {                                                        \
        int _st = cuda_status((call), #call);                   \
        if (_st != LULESH_OK) return _st;                       \
    } while (0)

static void prep_worker(lulesh_server *s)
{
    for (;;) {
        std::shared_ptr<SJob> j;
        {
            std::unique_lock<std::mutex> lk(s->mu);
            s->cv.wait(lk, [&] { return s->stop || !s->prep_q.empty(); });
            if (s->stop && s->prep_q.empty()) return;
            j = s->prep_q.front();
            s->prep_q.pop_front();
        }
        auto h = std::make_unique<HostDomain>();
        build_domain_light(*h, j->job.nx, j->job.numReg, j->job.balance, j->job.cost);
        j->host = std::move(h);
        j->ready.store(true, std::memory_order_release);
    }
}

static int rebuild(lulesh_server *s)
{
    // domain table, largest jobs first so their blocks start early
    std::vector<std::shared_ptr<SJob>> order = s->active;
    std::stable_sort(order.begin(), order.end(),
                     [](const std::shared_ptr<SJob> &a, const std::shared_ptr<SJob> &b) {
                         return a->dom.numElem > b->dom.numElem;
                     });
    std::vector<DomDev> hd;
    std::vector<int2> nb, eb;
    for (size_t d = 0; d < order.size(); ++d) {
        const DomDev &D = order[d]->dom;
        hd.push_back(D);
        for (int i = 0; i < D.numNode; i += kNodeBlock) nb.push_back(make_int2((int)d, i));
        for (int i = 0; i < D.numElem; i += kServerElemBlock) eb.push_back(make_int2((int)d, i));
    }
    // the nodal kernel walks last to first, as for sets (build_tables)
    if (LULESH_NODAL_REVERSE) std::reverse(nb.begin(), nb.end());
    if (!hd.empty())
        SCHECK(cudaMemcpyAsync(s->ddoms, hd.data(), sizeof(DomDev) * hd.size(),
                               cudaMemcpyHostToDevice, s->stream));
    // jobs admitted since the last launch get their time state now, on the
    // compute stream after the previous step: no launched cycle sees it
    SCHECK(cudaStreamSynchronize(s->upload));
    for (auto &j : s->active)
        if (j->fresh) {
            SCHECK(cudaMemcpyAsync(s->dtc + j->slot, &j->t0, sizeof(TimeCtl),
                                   cudaMemcpyHostToDevice, s->stream));
            j->fresh = false;
        }
    const size_t need = nb.size() + eb.size();
    if (need > s->blocks_cap) {
        if (s->dblocks) SCHECK(cudaFreeAsync(s->dblocks, s->stream));
        size_t cap = need + need / 2 + 1024;
        SCHECK(cudaMallocAsync(&s->dblocks, sizeof(int2) * cap, s->stream));
        s->blocks_cap = cap;
    }
    s->node_b = s->dblocks;
    s->elem_b = s->dblocks + nb.size();
    s->n_node = (int)nb.size();
    s->n_elem = (int)eb.size();
    if (!nb.empty())
        SCHECK(cudaMemcpyAsync(s->node_b, nb.data(), sizeof(int2) * nb.size(),
                               cudaMemcpyHostToDevice, s->stream));
    if (!eb.empty())
        SCHECK(cudaMemcpyAsync(s->elem_b, eb.data(), sizeof(int2) * eb.size(),
                               cudaMemcpyHostToDevice, s->stream));
    // the host vectors above are pageable: the copies complete before return
    SCHECK(cudaStreamSynchronize(s->stream));

    if (hd.empty()) {
        if (s->exec) cudaGraphExecDestroy(s->exec);
        if (s->graph) cudaGraphDestroy(s->graph);
        s->exec = nullptr;
        s->graph = nullptr;
    } else {
        SCHECK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
        launch_time_increment(s->dtc, s->cfg.max_jobs, s->P, s->stream, LULESH_PDL != 0);
        launch_force(s->args(s->elem_b), s->n_elem, s->P, s->stream, kServerElemBlock);
        launch_nodal(s->args(s->node_b), s->n_node, s->P, s->stream);
        launch_kinematics(s->args(s->elem_b), s->n_elem, s->P, s->stream, kServerElemBlock);
        launch_eos(s->args(s->elem_b), s->n_elem, s->P, s->stream, kServerElemBlock);
        cudaGraph_t g = nullptr;
        SCHECK(cudaStreamEndCapture(s->stream, &g));
        // same five kernels every time, only their grids and tables change:
        // update the executable graph in place, instantiate only if that fails
        if (s->exec) {
            cudaGraphExecUpdateResultInfo info{};
            if (cudaGraphExecUpdate(s->exec, g, &info) != cudaSuccess) {
                (void)cudaGetLastError();
                cudaGraphExecDestroy(s->exec);
                s->exec = nullptr;
            }
        }
        if (s->graph) cudaGraphDestroy(s->graph);
        s->graph = g;
        if (!s->exec) SCHECK(cudaGraphInstantiate(&s->exec, g, 0));
    }
    s->n_table = (int)hd.size();
    s->dirty = false;
    return LULESH_OK;
}

extern "C" {

double lulesh_server_clock(void) { return mono_now(); }

int lulesh_server_create(const lulesh_server_config *cfg, lulesh_server **out)
{
    if (!cfg || !out || cfg->max_jobs < 1 || cfg->max_jobs > 100000 || cfg->cycles_per_step < 1 ||
        cfg->prepare_threads < 1 || cfg->hbm_cap_bytes == 0) {
        set_error("lulesh_server_create: bad configuration");
        return LULESH_INVALID_ARG;
    }
    *out = nullptr;
    auto s = new lulesh_server;
    s->cfg = *cfg;
    s->P = default_params();
    auto fail = [&](int st) {
        lulesh_server_destroy(s);
        return st;
    };
    int st;
    if (cfg->device >= 0 && (st = cuda_status(cudaSetDevice(cfg->device), "set device")))
        return fail(st);
    if ((st = cuda_status(cudaGetDevice(&s->device), "get device"))) return fail(st);    if ((st = cuda_status(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking), "stream")))
        return fail(st);
    if ((st = cuda_status(cudaStreamCreateWithFlags(&s->upload, cudaStreamNonBlocking), "stream")))
        return fail(st);
    if ((st = cuda_status(cudaDeviceGetDefaultMemPool(&s->pool, s->device), "mem pool")))
        return fail(st);
    unsigned long long keep = ~0ull;  // keep freed job memory cached in the pool
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    const int M = cfg->max_jobs;
    if ((st = cuda_status(cudaMalloc(&s->dtc, sizeof(TimeCtl) * M), "slots"))) return fail(st);
    if ((st = cuda_status(cudaMallocHost(&s->htc, sizeof(TimeCtl) * M), "slots"))) return fail(st);
    if ((st = cuda_status(cudaMalloc(&s->denergy, sizeof(double) * M), "slots"))) return fail(st);
    if ((st = cuda_status(cudaMallocHost(&s->henergy, sizeof(double) * M), "slots")))
        return fail(st);
    if ((st = cuda_status(cudaMalloc(&s->ddoms, sizeof(DomDev) * M), "slots"))) return fail(st);
    if ((st = cuda_status(cudaEventCreateWithFlags(&s->step_done, cudaEventDisableTiming), "event")))
        return fail(st);
    // every slot starts empty: done, so the time-increment kernel skips it
    std::vector<TimeCtl> empty(M);
    for (int i = 0; i < M; ++i) {
        empty[i] = initial_timectl(0.0, 0);
        empty[i].done = 1;
        s->htc[i] = empty[i];
        s->free_slots.push_back(M - 1 - i);
    }
    if ((st = cuda_status(cudaMemcpy(s->dtc, empty.data(), sizeof(TimeCtl) * M,
                                     cudaMemcpyHostToDevice),
                          "slots")))
        return fail(st);
    for (int t = 0; t < cfg->prepare_threads; ++t) s->workers.emplace_back(prep_worker, s);
    *out = s;
    return LULESH_OK;
}

int lulesh_server_destroy(lulesh_server *s)
{
    if (!s) return LULESH_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->prep_q.clear();
    }
    s->cv.notify_all();
    for (auto &w : s->workers) w.join();
    if (s->stream) cudaStreamSynchronize(s->stream);
    for (auto &j : s->active)
        if (j->mem) cudaFreeAsync(j->mem, s->stream);
    if (s->dblocks) cudaFreeAsync(s->dblocks, s->stream);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    if (s->dtc) cudaFree(s->dtc);
    if (s->htc) cudaFreeHost(s->htc);
    if (s->denergy) cudaFree(s->denergy);
    if (s->henergy) cudaFreeHost(s->henergy);
    if (s->ddoms) cudaFree(s->ddoms);
    if (s->step_done) cudaEventDestroy(s->step_done);
    if (s->upload) cudaStreamDestroy(s->upload);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return LULESH_OK;
}

int lulesh_server_submit(lulesh_server *s, const lulesh_job *job, long long *id)
{
    if (!s || !job || job->nx < 1 || job->nx > LULESH_MAX_NX || job->numReg < 1 || job->balance < 0 ||
        job->cost < 0) {
        set_error("lulesh_server_submit: bad job");
        return LULESH_INVALID_ARG;
    }
    auto j = std::make_shared<SJob>();
    j->job = *job;
    j->bytes = domain_bytes(sizes_of(job->nx, job->numReg, 0), false);
    if (j->bytes > s->cfg.hbm_cap_bytes) {
        set_error("lulesh_server_submit: job larger than the server's memory cap");
        return LULESH_OOM;
    }
    j->t_submit = mono_now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        j->id = s->next_id++;
        s->prep_q.push_back(j);
    }
    s->cv.notify_one();
    s->pending.push_back(j);
    if (id) *id = j->id;
    return LULESH_OK;
}

int lulesh_server_step(lulesh_server *s, int *n_active, int *n_queued)
{
    if (!s) return LULESH_INVALID_ARG;
    // 1. previous step done: retire finished jobs
    if (s->in_flight) {
        SCHECK(cudaEventSynchronize(s->step_done));
        s->in_flight = false;
        const double now = mono_now();
        std::vector<std::shared_ptr<SJob>> keep;
        for (auto &j : s->active) {
            const TimeCtl &T = s->htc[j->slot];
            if (j->fresh || !T.done) {  // a fresh job's record was not read back
                keep.push_back(j);
                continue;
            }
            lulesh_server_result r{};
            r.id = j->id;
            r.status = T.status;
            r.bad_elem = (T.status == -1) ? T.bad_vol : (T.status == -2 ? T.bad_q : -1);
            r.cycle = T.cycle;
            r.origin_energy = s->henergy[j->slot];
            r.time = T.time;
            r.t_submit = j->t_submit;
            r.t_admit = j->t_admit;
            r.t_done = now;
            s->results.push_back(r);
            SCHECK(cudaFreeAsync(j->mem, s->stream));
            s->used_bytes -= j->bytes;
            s->free_slots.push_back(j->slot);
            s->dirty = true;
        }
        s->active.swap(keep);
    }
    // 2. resident set changed: new tables and graph
    if (s->dirty) {
        int st = rebuild(s);
        if (st != LULESH_OK) return st;
    }
    // 3. advance every resident job
    if (s->n_table > 0) {
        for (int c = 0; c < s->cfg.cycles_per_step; ++c)
            SCHECK(cudaGraphLaunch(s->exec, s->stream));
        const int n = s->n_table;
        k_gather_origin<<<(n + 127) / 128, 128, 0, s->stream>>>(s->ddoms, n, s->denergy);
        SCHECK(cudaGetLastError());
        SCHECK(cudaMemcpyAsync(s->htc, s->dtc, sizeof(TimeCtl) * s->cfg.max_jobs,
                               cudaMemcpyDeviceToHost, s->stream));
        SCHECK(cudaMemcpyAsync(s->henergy, s->denergy, sizeof(double) * s->cfg.max_jobs,
                               cudaMemcpyDeviceToHost, s->stream));
        SCHECK(cudaEventRecord(s->step_done, s->stream));
        s->in_flight = true;
    }
    // 4. admit in arrival order while the step runs: the uploads (side
    //    stream, host-blocking pageable copies) overlap the GPU's cycles;
    //    the jobs join the tables, and get their time state, at the next step
    while (!s->pending.empty()) {
        auto &j = s->pending.front();
        if (!j->ready.load(std::memory_order_acquire)) break;
        if (s->free_slots.empty() || s->used_bytes + j->bytes > s->cfg.hbm_cap_bytes) break;
        const int slot = s->free_slots.back();
        void *mem = nullptr;
        SCHECK(cudaMallocAsync(&mem, j->bytes, s->upload));
        Carver cv{static_cast<char *>(mem)};
        int st = upload_domain(*j->host, slot, 0, false, cv, s->upload, &j->dom, nullptr);
        if (st != LULESH_OK) {
            cudaFreeAsync(mem, s->upload);
            return st;
        }
        j->t0 = initial_timectl(j->host->deltatime, j->job.its);
        SCHECK(cudaStreamSynchronize(s->upload));
        j->host.reset();
        j->mem = mem;
        j->slot = slot;
        j->fresh = true;
        j->t_admit = mono_now();
        s->free_slots.pop_back();
        s->used_bytes += j->bytes;
        s->active.push_back(j);
        s->pending.pop_front();
        s->dirty = true;
    }
    if (n_active) *n_active = (int)s->active.size();
    if (n_queued) *n_queued = (int)s->pending.size();
    return LULESH_OK;
}

int lulesh_server_poll(lulesh_server *s, lulesh_server_result *out, int max, int *n)
{
    if (!s || !n || (max > 0 && !out)) return LULESH_INVALID_ARG;
    const int k = std::min<int>(max, (int)s->results.size());
    for (int i = 0; i < k; ++i) out[i] = s->results[i];
    s->results.erase(s->results.begin(), s->results.begin() + k);
    *n = k;
    return LULESH_OK;
}

}  // extern "C"
