// rungraph.cu -- the whole run as one CUDA graph launch.
//
// The reference drives its main loop from the host (lulesh.cu:4858-4873):
// TimeIncrement, LagrangeLeapFrog, and a check of the stop condition every
// cycle.  Here the loop is a WHILE conditional node: its body is one cycle
// (the same launches lulesh_step captures) followed by k_run_continue,
// which keeps the loop going while any job of the set is not done.  A batch
// of jobs, or a single job, then runs to completion in a single launch with
// no host involvement.  Every iteration is counted and the loop stops at a
// cap, so it ends even if a job could never reach its stop condition.
#include "set.hpp"

namespace lulesh {

namespace {

constexpr unsigned long long kDefaultRunCap = 1000000ull;

// ctl[0]: cycles run so far, ctl[1]: cap
__global__ void k_run_continue(cudaGraphConditionalHandle h, const TimeCtl *tcs, int ntc,
                               unsigned long long *ctl)
{
    __shared__ int any;
    if (threadIdx.x == 0) any = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < ntc; i += blockDim.x)
        if (!tcs[i].done) atomicOr(&any, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
        const unsigned long long n = ++ctl[0];
        cudaGraphSetConditional(h, (any && n < ctl[1]) ? 1u : 0u);
    }
}

#define RCHECK(call)                                            \
    do {                                                        \
        int _st = cuda_status((call), #call);                   \
        if (_st != LULESH_OK) return _st;                       \
    } while (0)

int ensure_run_graph(lulesh_set *s)
{
    if (s->exec_run) return LULESH_OK;
    int st = prepare_capture(s);
    if (st != LULESH_OK) return st;
    if (!s->run_ctl) RCHECK(cudaMalloc(&s->run_ctl, 2 * sizeof(unsigned long long)));
    cudaGraph_t g = nullptr;
    RCHECK(cudaGraphCreate(&g, 0));
    cudaGraphConditionalHandle h;
    st = cuda_status(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault),
                     "conditional handle");
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    if (st == LULESH_OK)
        st = cuda_status(cudaGraphAddNode(&node, g, nullptr, 0, &p), "while node");
    if (st == LULESH_OK) {
        cudaGraph_t body = p.conditional.phGraph_out[0];
        st = cuda_status(cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0,
                                                       cudaStreamCaptureModeThreadLocal),
                         "capture loop body");
        if (st == LULESH_OK) {
            // the loop body keeps plain stream order between its kernels
            const bool pdl = s->pdl;
            s->pdl = false;
            int est = enqueue_cycle(s);
            s->pdl = pdl;
            k_run_continue<<<1, 128, 0, s->stream>>>(h, s->dtc, s->njobs, s->run_ctl);
            cudaGraph_t captured = nullptr;
            const int cst = cuda_status(cudaStreamEndCapture(s->stream, &captured), "end capture");
            st = (est != LULESH_OK) ? est : cst;
        }
    }
    if (st == LULESH_OK) st = cuda_status(cudaGraphInstantiate(&s->exec_run, g, 0), "instantiate");
    if (st != LULESH_OK) {
        cudaGraphDestroy(g);
        return st;
    }
    s->graph_run = g;
    return LULESH_OK;
}

}  // namespace
}  // namespace lulesh

using namespace lulesh;

extern "C" int lulesh_run_graph(lulesh_set *s, long long max_cycles)
{
    if (!s) return LULESH_INVALID_ARG;
    int st = ensure_run_graph(s);
    if (st != LULESH_OK) return st;
    const unsigned long long ctl[2] = {
        0ull, max_cycles > 0 ? (unsigned long long)max_cycles : kDefaultRunCap};
    RCHECK(cudaMemcpyAsync(s->run_ctl, ctl, sizeof ctl, cudaMemcpyHostToDevice, s->stream));
    RCHECK(cudaGraphLaunch(s->exec_run, s->stream));
    return run_status(s);  // synchronises the stream
}
