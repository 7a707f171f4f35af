// peak.cu -- the FP64 throughput this GPU delivers, measured.
//
// The force, kinematics and EOS kernels are FP64 SIMT code, so their
// roofline is the FP64 FMA rate rather than HBM bandwidth.  The nominal rate
// (SMs x 64 FP64 lanes x clock) is an upper bound; this measures what
// independent register-only FMA chains reach, which is the denominator the
// benchmark reports the FP64 kernels against.
#include "set.hpp"

namespace {

constexpr int kChains = 16;
constexpr int kThreads = 256;

__global__ void __launch_bounds__(kThreads) k_fma_chains(double *out, int iters, double a,
                                                         double b)
{
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3 + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * kThreads + threadIdx.x] = s;  // keeps the chains live
}

}  // namespace

extern "C" int lulesh_measure_fp64_peak(int device, double *fma_per_s)
{
    using lulesh::cuda_status;
    if (!fma_per_s) return LULESH_INVALID_ARG;
    if (device >= 0) {
        const int st = cuda_status(cudaSetDevice(device), "measure fp64");
        if (st != LULESH_OK) return st;
    }
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    int st = cuda_status(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev),
                         "measure fp64");
    if (st != LULESH_OK) return st;
    const int blocks = sms * 8, iters = 8192;
    double *out = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    st = cuda_status(cudaMalloc(&out, sizeof(double) * blocks * kThreads), "measure fp64");
    if (st == LULESH_OK) st = cuda_status(cudaEventCreate(&e0), "measure fp64");
    if (st == LULESH_OK) st = cuda_status(cudaEventCreate(&e1), "measure fp64");
    float best = 0.f;
    if (st == LULESH_OK) {
        k_fma_chains<<<blocks, kThreads>>>(out, 64, 0.999999, 1e-9);  // warm-up
        for (int rep = 0; rep < 3 && st == LULESH_OK; ++rep) {
            cudaEventRecord(e0);
            k_fma_chains<<<blocks, kThreads>>>(out, iters, 0.999999, 1e-9);
            cudaEventRecord(e1);
            st = cuda_status(cudaEventSynchronize(e1), "measure fp64");
            float ms = 0.f;
            if (st == LULESH_OK) st = cuda_status(cudaEventElapsedTime(&ms, e0, e1), "measure fp64");
            if (st == LULESH_OK && (best == 0.f || ms < best)) best = ms;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (out) cudaFree(out);
    if (st != LULESH_OK) return st;
    *fma_per_s = (double)blocks * kThreads * kChains * iters / (best * 1e-3);
    return LULESH_OK;
}
