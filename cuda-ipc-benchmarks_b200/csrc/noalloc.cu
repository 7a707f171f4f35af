// noalloc.cu -- nodal volume forces without any device allocation.
//
// Some callers cannot allocate device memory: a host code that embeds this
// force computation in its own time loop while its memory manager owns all
// of the GPU's memory (a fixed, pre-partitioned budget leaves nothing for a
// library to cudaMalloc), or a latency-sensitive loop that cannot pay for
// cudaMalloc/cudaFree, which synchronise the whole device and stall every
// other stream.  For them, lulesh_volume_force_noalloc computes what
// CalcVolumeForceForElems does (per-element stress + FB hourglass corner
// forces, then the per-node sum in corner order) using, as its only
// scratch, one file-scope device array of fixed size that exists for as
// long as the library is loaded.
//
// The corner forces of up to kNoAllocMaxElems elements live in that array;
// its last 256 bytes hold the volume-error flag.  Host code never uses the
// array's name as an address: the device address comes from
// cudaGetSymbolAddress, looked up with the device current on every call made
// outside stream capture (a device reset or a caller-created context moves
// the array), and taken from the last such call while a stream captures.
#include <climits>
#include <mutex>
#include <string>

#include "elem_math.cuh"
#include "lulesh_b200.h"
#include "set.hpp"

namespace {

constexpr int kNoAllocMaxElems = LULESH_NOALLOC_MAX_ELEMS;  // nx <= 32
constexpr int kCornerDoubles = 3 * 8 * kNoAllocMaxElems;
constexpr int kBlock = 128;

// corner forces [component][corner][element] followed by a 256-byte tail
// whose first int is the smallest element with a negative volume
static __device__ __align__(256) double g_noalloc_scratch[kCornerDoubles + 32];

std::mutex g_mu;
void *g_addr[64];  // last looked-up address of g_noalloc_scratch, per device ordinal

__global__ void k_flag_reset(int *flag) { *flag = INT_MAX; }

template <bool HG>
__global__ void __launch_bounds__(kBlock)
    k_force_noalloc(int nx, const double *__restrict__ x, const double *__restrict__ y,
                    const double *__restrict__ z, const double *__restrict__ xd,
                    const double *__restrict__ yd, const double *__restrict__ zd,
                    const double *__restrict__ volo, const double *__restrict__ v,
                    const double *__restrict__ p, const double *__restrict__ q,
                    const double *__restrict__ ss, const double *__restrict__ elemMass,
                    double hourg, double *__restrict__ corners, int *flag)
{
    const int numElem = nx * nx * nx;
    const int elem = blockIdx.x * blockDim.x + threadIdx.x;
    if (elem >= numElem) return;
    const int Ep = ((numElem + 31) / 32) * 32;
    const int en = nx + 1;
    const int ix = elem % nx, t = elem / nx, iy = t % nx, iz = t / nx;
    const int n0 = (iz * en + iy) * en + ix;
    const int n[8] = {n0, n0 + 1, n0 + en + 1, n0 + en, n0 + en * en, n0 + en * en + 1,
                      n0 + en * en + en + 1, n0 + en * en + en};

    double xn[8], yn[8], zn[8], dvdxn[8], dvdyn[8], dvdzn[8];
    double hgfx[8], hgfy[8], hgfz[8], hourgam[8][4], B[3][8];
    const double volume = v[elem];
    double det = volo[elem] * volume;
    if (volume < 0.) atomicMin(flag, elem);
    const double ss1 = ss[elem], mass1 = elemMass[elem];
    const double sigxx = -p[elem] - q[elem];
    const double volinv = 1.0 / det;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        xn[i] = x[n[i]];
        yn[i] = y[n[i]];
        zn[i] = z[n[i]];
    }
    const double volume13 = cbrt(det);
    const double coefficient = -hourg * 0.01 * ss1 * mass1 / volume13;
    lulesh::elem_volume_derivative(dvdxn, dvdyn, dvdzn, xn, yn, zn);
    lulesh::hourglass_modes(xn, yn, zn, dvdxn, dvdyn, dvdzn, hourgam, volinv);
    lulesh::shape_function_derivatives(xn, yn, zn, B, &det);
    lulesh::elem_node_normals(B[0], B[1], B[2], xn, yn, zn);
    if (det < 0.) atomicMin(flag, elem);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        hgfx[i] = -(sigxx * B[0][i]);
        hgfy[i] = -(sigxx * B[1][i]);
        hgfz[i] = -(sigxx * B[2][i]);
    }
    if (HG) {
        double vel[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) vel[i] = xd[n[i]];
        lulesh::fb_hourglass_component(vel, hourgam, coefficient, hgfx);
#pragma unroll
        for (int i = 0; i < 8; ++i) vel[i] = yd[n[i]];
        lulesh::fb_hourglass_component(vel, hourgam, coefficient, hgfy);
#pragma unroll
        for (int i = 0; i < 8; ++i) vel[i] = zd[n[i]];
        lulesh::fb_hourglass_component(vel, hourgam, coefficient, hgfz);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        corners[(0 * 8 + k) * Ep + elem] = hgfx[k];
        corners[(1 * 8 + k) * Ep + elem] = hgfy[k];
        corners[(2 * 8 + k) * Ep + elem] = hgfz[k];
    }
}

// per-node sum of the surrounding corners in corner order 0..7 (the
// nodeElemCornerList order of a structured mesh)
__global__ void __launch_bounds__(kBlock)
    k_gather_noalloc(int nx, const double *__restrict__ corners, const int *flag,
                     double *__restrict__ fx, double *__restrict__ fy, double *__restrict__ fz,
                     int *bad_elem)
{
    const int en = nx + 1, numNode = en * en * en;
    const int numElem = nx * nx * nx, Ep = ((numElem + 31) / 32) * 32;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0 && bad_elem) *bad_elem = (*flag == INT_MAX) ? -1 : *flag;
    if (i >= numNode) return;
    const int px = i % en, t = i / en, py = t % en, pz = t / en;
    const int cx[8] = {0, 1, 1, 0, 0, 1, 1, 0}, cy[8] = {0, 0, 1, 1, 0, 0, 1, 1},
              cz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int ex = px - cx[j], ey = py - cy[j], ez = pz - cz[j];
        if ((unsigned)ex < (unsigned)nx && (unsigned)ey < (unsigned)nx &&
            (unsigned)ez < (unsigned)nx) {
            const int e = (ez * nx + ey) * nx + ex;
            sx += corners[(0 * 8 + j) * Ep + e];
            sy += corners[(1 * 8 + j) * Ep + e];
            sz += corners[(2 * 8 + j) * Ep + e];
        }
    }
    fx[i] = sx;
    fy[i] = sy;
    fz[i] = sz;
}

// Device address of the scratch array in the current context, for a call
// enqueued on stream s.  Outside stream capture every call looks it up
// (cudaGetSymbolAddress, with the caller's device current; a host-side
// table lookup once the module is loaded), so the address is always that of
// the current context: after cudaDeviceReset the module is loaded again and
// the array may sit at a new address, and a context the caller created
// holds its own copy.  While s is capturing, the address of the last call
// on this device outside capture is used; with none, the call is refused.
int scratch_address(cudaStream_t s, void **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LULESH_NO_DEVICE;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cs) != cudaSuccess) {
        (void)cudaGetLastError();
        cs = cudaStreamCaptureStatusActive;  // treat an unclear answer as capture
    }
    std::lock_guard<std::mutex> lock(g_mu);
    if (cs == cudaStreamCaptureStatusNone) {
        void *ptr = nullptr;
        if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr)
            return LULESH_CUDA_ERROR;
        g_addr[dev] = ptr;
    } else if (!g_addr[dev]) {
        lulesh::set_error("lulesh_volume_force_noalloc: the first call on a device must come "
                          "before any stream capture");
        return LULESH_INVALID_ARG;
    }
    *out = g_addr[dev];
    return LULESH_OK;
}

}  // namespace

extern "C" int lulesh_volume_force_noalloc(int nx, const double *x, const double *y,
                                           const double *z, const double *xd, const double *yd,
                                           const double *zd, const double *volo, const double *v,
                                           const double *p, const double *q, const double *ss,
                                           const double *elemMass, double hgcoef, double *fx,
                                           double *fy, double *fz, int *bad_elem, void *stream)
{
    if (nx < 1 || (long)nx * nx * nx > kNoAllocMaxElems) {
        lulesh::set_error("lulesh_volume_force_noalloc: nx=" + std::to_string(nx) +
                          " is outside 1.." + std::to_string(LULESH_NOALLOC_MAX_NX) +
                          " (the fixed scratch array holds " +
                          std::to_string(kNoAllocMaxElems) + " elements)");
        return LULESH_INVALID_ARG;
    }
    if (!x || !y || !z || !xd || !yd || !zd || !volo || !v || !p || !q || !ss || !elemMass ||
        !fx || !fy || !fz) {
        lulesh::set_error("lulesh_volume_force_noalloc: null array argument");
        return LULESH_INVALID_ARG;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    void *base = nullptr;
    int st = scratch_address(s, &base);
    if (st != LULESH_OK) return st;
    double *corners = static_cast<double *>(base);
    int *flag = reinterpret_cast<int *>(corners + kCornerDoubles);
    const int numElem = nx * nx * nx, numNode = (nx + 1) * (nx + 1) * (nx + 1);
    k_flag_reset<<<1, 1, 0, s>>>(flag);
    if (hgcoef > 0.0)
        k_force_noalloc<true><<<(numElem + kBlock - 1) / kBlock, kBlock, 0, s>>>(
            nx, x, y, z, xd, yd, zd, volo, v, p, q, ss, elemMass, hgcoef, corners, flag);
    else
        k_force_noalloc<false><<<(numElem + kBlock - 1) / kBlock, kBlock, 0, s>>>(
            nx, x, y, z, xd, yd, zd, volo, v, p, q, ss, elemMass, hgcoef, corners, flag);
    k_gather_noalloc<<<(numNode + kBlock - 1) / kBlock, kBlock, 0, s>>>(nx, corners, flag, fx,
                                                                        fy, fz, bad_elem);
    return (cudaGetLastError() == cudaSuccess) ? LULESH_OK : LULESH_CUDA_ERROR;
}
