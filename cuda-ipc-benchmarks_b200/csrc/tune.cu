// tune.cu -- launch shapes of a set and the autotuner that picks them.
//
// A set of many uneven jobs (a batch) runs every cycle as one graph over
// the block tables of all its domains.  What the hardware sees depends on
// the tile each block covers (elements per block of the element kernels,
// nodes per block of the nodal kernel), on the order of the tables (large
// domains first lets small ones fill the tail of each launch) and on how many
// cycles one graph launch carries (host launch cost for small jobs).  None
// of these change a result: every block computes the same elements with the
// same arithmetic, and the dt minimum is an exact min.
//
// The autotuner measures instead of modelling: it saves the set's whole
// device state (arena + time-control blocks), runs each candidate from
// that same state with CUDA events on the set's stream, and restores the
// state at the end, so tuning a live set does not advance it.
#include <vector>

#include "set.hpp"

namespace lulesh {

#define TCHECK(call)                                            \
    do {                                                        \
        int _st = cuda_status((call), #call);                   \
        if (_st != LULESH_OK) return _st;                       \
    } while (0)

static bool shapes_fixed(const lulesh_set *s)
{
    return s->tp > 1 || s->unstructured ||
           (s->flags & (LULESH_FLAG_COMM_STAGED | LULESH_FLAG_MIXED)) != 0;
}

static int apply(lulesh_set *s, const lulesh_tuning &t)
{
    if (!valid_elem_block(t.elem_block) || !valid_node_block(t.node_block) || t.order < 0 ||
        t.order > 1 || t.graph_cycles < 1 || t.graph_cycles > 100000) {
        set_error("lulesh_set_tuning: elem_block in {64,128,256}, node_block in "
                  "{128,256,512}, order 0 or 1, graph_cycles >= 1");
        return LULESH_INVALID_ARG;
    }
    if (shapes_fixed(s) && (t.elem_block != kElemBlock || t.node_block != kNodeBlock)) {
        set_error("lulesh_set_tuning: subdomain, staged and mixed sets use 128-wide blocks");
        return LULESH_INVALID_ARG;
    }
    TCHECK(cudaStreamSynchronize(s->stream));
    if (t.elem_block != s->eb || t.node_block != s->nb || t.order != s->order) {
        s->eb = t.elem_block;
        s->nb = t.node_block;
        s->order = t.order;
        drop_graph(s);
        const int st = build_tables(s);
        if (st != LULESH_OK) return st;
        TCHECK(cudaStreamSynchronize(s->stream));
    }
    return lulesh_set_graph_cycles(s, t.graph_cycles);
}

// Saved device state of a set.
struct Snapshot {
    void *arena = nullptr;
    void *tc = nullptr;
    ~Snapshot()
    {
        if (arena) cudaFree(arena);
        if (tc) cudaFree(tc);
    }
    int save(const lulesh_set *s)
    {
        TCHECK(cudaMalloc(&arena, s->arena_bytes));
        TCHECK(cudaMalloc(&tc, sizeof(TimeCtl) * s->njobs));
        return restore_into(s, true);
    }
    int restore(const lulesh_set *s) { return restore_into(s, false); }

   private:
    int restore_into(const lulesh_set *s, bool save_dir)
    {
        void *a_dst = save_dir ? arena : s->arena, *a_src = save_dir ? s->arena : arena;
        void *t_dst = save_dir ? tc : (void *)s->dtc, *t_src = save_dir ? (void *)s->dtc : tc;
        TCHECK(cudaMemcpyAsync(a_dst, a_src, s->arena_bytes, cudaMemcpyDeviceToDevice,
                               s->stream));
        TCHECK(cudaMemcpyAsync(t_dst, t_src, sizeof(TimeCtl) * s->njobs,
                               cudaMemcpyDeviceToDevice, s->stream));
        return LULESH_OK;
    }
};

// Device time per cycle of `cycles` cycles of the current shape, started
// from the saved state (after an untimed warm-up that builds the graphs).
static int time_shape(lulesh_set *s, Snapshot &snap, int cycles, cudaEvent_t e0, cudaEvent_t e1,
                      double *ms_per_cycle)
{
    int st = snap.restore(s);
    if (st == LULESH_OK) st = lulesh_step(s, s->graph_cycles > 1 ? s->graph_cycles : 1);
    if (st == LULESH_OK) st = snap.restore(s);
    if (st != LULESH_OK) return st;
    TCHECK(cudaEventRecord(e0, s->stream));
    st = lulesh_step(s, cycles);
    if (st != LULESH_OK) return st;
    TCHECK(cudaEventRecord(e1, s->stream));
    TCHECK(cudaEventSynchronize(e1));
    float ms = 0.f;
    TCHECK(cudaEventElapsedTime(&ms, e0, e1));
    *ms_per_cycle = ms / cycles;
    return LULESH_OK;
}

}  // namespace lulesh

using namespace lulesh;

extern "C" {

int lulesh_get_tuning(const lulesh_set *s, lulesh_tuning *out)
{
    if (!s || !out) return LULESH_INVALID_ARG;
    out->elem_block = s->eb;
    out->node_block = s->nb;
    out->order = s->order;
    out->graph_cycles = s->graph_cycles;
    return LULESH_OK;
}

int lulesh_set_tuning(lulesh_set *s, const lulesh_tuning *t)
{
    if (!s || !t) return LULESH_INVALID_ARG;
    return apply(s, *t);
}

int lulesh_autotune(lulesh_set *s, int trial_cycles, int rounds, lulesh_tuning *best,
                    lulesh_tune_trial *trials, int max_trials, int *n_trials)
{
    if (!s || trial_cycles < 1 || rounds < 1 || (max_trials > 0 && !trials)) {
        set_error("lulesh_autotune: trial_cycles >= 1, rounds >= 1");
        return LULESH_INVALID_ARG;
    }
    lulesh_tuning orig{};
    lulesh_get_tuning(s, &orig);
    TCHECK(cudaStreamSynchronize(s->stream));
    Snapshot snap;
    int st = snap.save(s);
    if (st != LULESH_OK) return st;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    TCHECK(cudaEventCreate(&e0));
    TCHECK(cudaEventCreate(&e1));

    // phase 1: block shapes and table order, one cycle per graph launch
    std::vector<lulesh_tuning> cand;
    const bool fixed = shapes_fixed(s);
    const int ebs[] = {64, 128, 256}, nbs[] = {128, 256, 512};
    for (int e : ebs)
        for (int n : nbs)
            for (int o = 0; o <= (s->ndom > 1 ? 1 : 0); ++o) {
                if (fixed && (e != kElemBlock || n != kNodeBlock)) continue;
                cand.push_back(lulesh_tuning{e, n, o, 1});
            }
    std::vector<double> best_ms(cand.size(), 1e300);
    for (int r = 0; r < rounds && st == LULESH_OK; ++r)
        for (size_t c = 0; c < cand.size() && st == LULESH_OK; ++c) {
            double ms = 0;
            st = apply(s, cand[c]);
            if (st == LULESH_OK) st = time_shape(s, snap, trial_cycles, e0, e1, &ms);
            if (st == LULESH_OK && ms < best_ms[c]) best_ms[c] = ms;
        }
    size_t win = 0;
    for (size_t c = 1; c < cand.size(); ++c)
        if (best_ms[c] < best_ms[win]) win = c;

    // phase 2: cycles per graph launch for the winning shape
    std::vector<lulesh_tuning> cand2;
    std::vector<double> best2;
    for (int k : {1, 2, 4, 8, 16}) {
        if (k > trial_cycles) break;
        lulesh_tuning t = cand[win];
        t.graph_cycles = k;
        cand2.push_back(t);
        best2.push_back(1e300);
    }
    for (int r = 0; r < rounds && st == LULESH_OK; ++r)
        for (size_t c = 0; c < cand2.size() && st == LULESH_OK; ++c) {
            double ms = 0;
            const int k = cand2[c].graph_cycles;
            st = apply(s, cand2[c]);
            if (st == LULESH_OK)
                st = time_shape(s, snap, (trial_cycles / k) * k, e0, e1, &ms);
            if (st == LULESH_OK && ms < best2[c]) best2[c] = ms;
        }
    size_t win2 = 0;
    for (size_t c = 1; c < cand2.size(); ++c)
        if (best2[c] < best2[win2]) win2 = c;

    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // state back as it was, winner applied (or the original shape on error)
    const int rs = snap.restore(s);
    if (st == LULESH_OK) st = rs;
    if (st != LULESH_OK) {
        apply(s, orig);
        return st;
    }
    TCHECK(cudaStreamSynchronize(s->stream));
    st = apply(s, cand2[win2]);
    if (st != LULESH_OK) return st;
    if (best) *best = cand2[win2];
    int n = 0;
    for (size_t c = 0; c < cand.size(); ++c)
        if (n < max_trials) trials[n++] = lulesh_tune_trial{cand[c], best_ms[c]};
    for (size_t c = 0; c < cand2.size(); ++c)
        if (n < max_trials) trials[n++] = lulesh_tune_trial{cand2[c], best2[c]};
    if (n_trials) *n_trials = n;
    return LULESH_OK;
}

}  // extern "C"
