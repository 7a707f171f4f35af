// kernels.cu -- the per-cycle kernels of the LULESH Lagrange leapfrog step.
//
// One cycle is five launches (captured in one CUDA graph):
//   time_increment  TimeIncrement on the device (lulesh.cu:1400-1461)
//   force           CalcVolumeForceForElems_kernel (lulesh.cu:2080-2259):
//                   stress + FB hourglass corner forces per element
//   nodal           AddNodeForcesFromElems + CalcAccelerationForNodes +
//                   ApplyAccelerationBoundaryConditionsForNodes +
//                   CalcPositionAndVelocityForNodes (lulesh.cu:1715-1751,
//                   2925-3044) fused: corners summed in corner order with
//                   no atomics, then the node update
//   kinematics      CalcKinematicsAndMonotonicQGradient_kernel
//                   (lulesh.cu:3343-3507)
//   eos             CalcMonotonicQRegionForElems_kernel +
//                   ApplyMaterialPropertiesAndUpdateVolume_kernel +
//                   CalcTimeConstraintsForElems (lulesh.cu:3554-3725,
//                   3988-4097, 4216-4403) fused; the dt minimum is reduced
//                   with warp shuffles and one 64-bit atomicMin per block
// Two halo kernels follow CommSyncPosVel and CommMonoQ: the PosVel sync
// copies a neighbour's max-side node layer, the MonoQ ghost kernel its
// boundary element layer of delv_*.  A subdomain set's fused cycle needs
// neither (every corner of every node is summed in single-domain order, and
// k_eos<..., SUB> reads comm-face neighbours in place), and the parts of a
// multi-GPU problem read their proxies in place after the MONOQ messages.
// Unstructured (lmesh) domains run force, kinematics and EOS with U = true,
// which reads nodelist, the face links and elemBC from memory instead of
// computing them from the element index, and k_nodal_u for the nodal step.
#include <climits>
#include <cstdint>

#include "elem_body.cuh"
#include "elem_math.cuh"
#include "kernels.cuh"
#include "lulesh_b200.h"

namespace lulesh {

// ---------------------------------------------------------------------------
// time increment

__device__ __forceinline__ unsigned long long dbits(double v)
{
    return (unsigned long long)__double_as_longlong(v);
}

__global__ void k_time_increment(TimeCtl *tcs, int ntc, Params P)
{
    pdl_enter();
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= ntc) return;
    TimeCtl &T = tcs[i];
    T.active = 0;
    if (T.done) return;
    // checkErrors (lulesh.cu:2879-2892): a cycle that raised an error ends
    // the job before the next one starts
    if (T.bad_vol != INT_MAX) {
        T.status = -1;
        T.done = 1;
        return;
    }
    if (T.bad_q != INT_MAX) {
        T.status = -2;
        T.done = 1;
        return;
    }
#if LULESH_CHECKED
    if (T.chk != 0) {
        T.status = LULESH_BOUNDS_ERROR;
        T.done = 1;
        return;
    }
#endif
    // while (time < stoptime) ... if (its == num_iters) break (lulesh.cu:4858-4873)
    if (!(T.time < P.stoptime) || (T.its_cap > 0 && T.cycle >= T.its_cap)) {
        T.done = 1;
        return;
    }
    if (T.cycle != 0) {
        // the previous cycle's CalcTimeConstraintsForElems result
        T.dtcourant = __longlong_as_double((long long)T.min_courant);
        T.dthydro = __longlong_as_double((long long)T.min_hydro);
    }
    T.min_courant = dbits(1.0e+20);
    T.min_hydro = dbits(1.0e+20);

    double targetdt = P.stoptime - T.time;
    if ((P.dtfixed <= 0.0) && (T.cycle != 0)) {
        double ratio;
        double gnewdt = 1.0e+20;
        double newdt;
        if (T.dtcourant < gnewdt) gnewdt = T.dtcourant / 2.0;
        if (T.dthydro < gnewdt) gnewdt = T.dthydro * 2.0 / 3.0;
        newdt = gnewdt;
        const double olddt = T.deltatime;
        ratio = newdt / olddt;
        if (ratio >= 1.0) {
            if (ratio < P.deltatimemultlb)
                newdt = olddt;
            else if (ratio > P.deltatimemultub)
                newdt = olddt * P.deltatimemultub;
        }
        if (newdt > P.dtmax) newdt = P.dtmax;
        T.deltatime = newdt;
    }
    // try to prevent very small scaling on the next cycle
    if ((targetdt > T.deltatime) && (targetdt < (4.0 * T.deltatime / 3.0)))
        targetdt = 2.0 * T.deltatime / 3.0;
    if (targetdt < T.deltatime) T.deltatime = targetdt;
    T.time += T.deltatime;
    ++T.cycle;
    T.active = 1;
}

void launch_time_increment(TimeCtl *tcs, int ntc, Params P, cudaStream_t s, bool pdl)
{
    const int b = 128;
    launch_k(k_time_increment, (ntc + b - 1) / b, b, s, pdl, tcs, ntc, P);
}

// ---------------------------------------------------------------------------
// structured-mesh indexing helpers

// corner j of an element sits at lattice offset (CX[j], CY[j], CZ[j]) from
// the element's corner 0 (nodelist order of BuildMesh, lulesh.cu:730-737)
__device__ __constant__ int kCX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
__device__ __constant__ int kCY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
__device__ __constant__ int kCZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};

// ---------------------------------------------------------------------------
// force: CalcVolumeForceForElems_kernel, lulesh.cu:2080-2259

// one element of the force phase: the node gathers, then force_elem
template <bool HG, bool U>
__device__ __forceinline__ void force_one(const DomDev &D, TimeCtl &T, const Params &P, int elem)
{
    // all 48 node gathers are issued before any arithmetic: the velocity
    // loads then overlap the coordinate work instead of stalling the
    // hourglass step (measured on B200 at -s 100: 150 -> 136 us)
    int n[8];
    elem_nodes<U>(D, elem, n);
#pragma unroll
    for (int i = 0; i < 8; ++i) n[i] = chk_index(n[i], D.numNode, &T, kChkNode);
    double xn[8], yn[8], zn[8];
    double xdn[8], ydn[8], zdn[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (HG) {
            xdn[i] = D.xd[n[i]];
            ydn[i] = D.yd[n[i]];
            zdn[i] = D.zd[n[i]];
        } else {
            xdn[i] = ydn[i] = zdn[i] = 0.0;
        }
    }
    const VelRegs vel{xdn, ydn, zdn};
#pragma unroll
    for (int i = 0; i < 8; ++i) xn[i] = D.x[n[i]];
#pragma unroll
    for (int i = 0; i < 8; ++i) yn[i] = D.y[n[i]];
#pragma unroll
    for (int i = 0; i < 8; ++i) zn[i] = D.z[n[i]];
    force_elem<HG>(D, T, P, elem, xn, yn, zn, vel);
}

template <bool HG, int BS, bool U>
__global__ void __launch_bounds__(BS, min_blocks(kForceMinBlocks, BS)) k_force(SetArgs a, Params P)
{
    pdl_enter();
    const int2 blk = a.blocks[LULESH_FORCE_REVERSE ? gridDim.x - 1 - blockIdx.x : blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;
    const int elem = blk.y + threadIdx.x;
    if (elem >= D.numElem) return;
    force_one<HG, U>(D, T, P, elem);
}

template <int BS, bool U = false>
static void launch_force_bs(const SetArgs &a, int nblocks, Params P, cudaStream_t s)
{
    if (P.hgcoef > 0.0)
        launch_k(k_force<true, BS, U>, nblocks, BS, s, a.pdl != 0, a, P);
    else
        launch_k(k_force<false, BS, U>, nblocks, BS, s, a.pdl != 0, a, P);
}

void launch_force(const SetArgs &a, int nblocks, Params P, cudaStream_t s, int bs, bool u)
{
    if (u) {
        launch_force_bs<kElemBlock, true>(a, nblocks, P, s);
        return;
    }
    switch (bs) {
        case 64: launch_force_bs<64>(a, nblocks, P, s); break;
        case 256: launch_force_bs<256>(a, nblocks, P, s); break;
        default: launch_force_bs<kElemBlock>(a, nblocks, P, s); break;
    }
}

// ---------------------------------------------------------------------------
// nodal: corner gather (in nodeElemCornerList order) + node update

// Sum the corner forces around node (px,py,pz) of domain D in corner order
// j = 0..7, the order nodeElemCornerList has on a structured mesh
// (lulesh.cu:1082-1091).  A corner whose element lies in a neighbouring
// subdomain is read from that subdomain's corner array: the result equals
// the undecomposed mesh's sum bit for bit.
__device__ __forceinline__ void gather_corners(const DomDev *doms, const DomDev &D, int px,
                                               int py, int pz, double &fx, double &fy,
                                               double &fz, TimeCtl *T)
{
    const int nx = D.nx;
    fx = fy = fz = 0.0;
    if (D.tp > 1) {
        // subdomains: the source domain of each corner first (this one or
        // a neighbour), then one load path that the warp shares
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int ex = px - kCX[j], ey = py - kCY[j], ez = pz - kCZ[j];
            const int sx = (ex < 0) ? -1 : (ex >= nx ? 1 : 0);
            const int sy = (ey < 0) ? -1 : (ey >= nx ? 1 : 0);
            const int sz = (ez < 0) ? -1 : (ez >= nx ? 1 : 0);
            const DomDev *S = &D;
            bool use = (sx | sy | sz) == 0;
            if (!use) {
                const int nb = D.nbr[(sx + 1) + 3 * (sy + 1) + 9 * (sz + 1)];
                if (nb >= 0) {
                    S = &doms[nb];
                    use = true;
                }
            }
            if (use) {
                const int lx = ex - sx * nx, ly = ey - sy * nx, lz = ez - sz * nx;
                const int idx = chk_index(j * S->Ep + (lz * nx + ly) * nx + lx, 8LL * S->Ep, T,
                                          kChkCorner);
                fx += ld_corner(S->fx_elem + idx);
                fy += ld_corner(S->fy_elem + idx);
                fz += ld_corner(S->fz_elem + idx);
            }
        }
        return;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int ex = px - kCX[j], ey = py - kCY[j], ez = pz - kCZ[j];
        const bool inside = (unsigned)ex < (unsigned)nx && (unsigned)ey < (unsigned)nx &&
                            (unsigned)ez < (unsigned)nx;
        if (inside) {
            const int idx = chk_index(j * D.Ep + (ez * nx + ey) * nx + ex, 8LL * D.Ep, T,
                                      kChkCorner);
            fx += ld_corner(D.fx_elem + idx);
            fy += ld_corner(D.fy_elem + idx);
            fz += ld_corner(D.fz_elem + idx);
        }
    }
}

// CalcAccelerationForNodes (lulesh.cu:2926-2939), the symmetry-plane zeroing
// of ApplyAccelerationBoundaryConditionsForNodes (bc bits 0/1/2 zero the
// x/y/z acceleration) and CalcPositionAndVelocityForNodes (lulesh.cu:
// 2999-3028) for node i with the summed force (fx, fy, fz)
__device__ __forceinline__ void advance_node(const DomDev &D, const TimeCtl &T, const Params &P,
                                             int i, int bc, double fx, double fy, double fz,
                                             int materialize, bool write_f)
{
    const double one_over_nMass = 1. / D.nodalMass[i];
    double xdd = fx * one_over_nMass;
    double ydd = fy * one_over_nMass;
    double zdd = fz * one_over_nMass;
    if (bc & 1) xdd = 0.0;
    if (bc & 2) ydd = 0.0;
    if (bc & 4) zdd = 0.0;

    const double dt = T.deltatime;
    const double u_cut = P.u_cut;
    double xdtmp = D.xd[i] + xdd * dt;
    double ydtmp = D.yd[i] + ydd * dt;
    double zdtmp = D.zd[i] + zdd * dt;
    if (fabs(xdtmp) < u_cut) xdtmp = 0.0;
    if (fabs(ydtmp) < u_cut) ydtmp = 0.0;
    if (fabs(zdtmp) < u_cut) zdtmp = 0.0;
    D.x[i] += xdtmp * dt;
    D.y[i] += ydtmp * dt;
    D.z[i] += zdtmp * dt;
    D.xd[i] = xdtmp;
    D.yd[i] = ydtmp;
    D.zd[i] = zdtmp;
    if (materialize) {
        if (write_f) {
            D.fx[i] = fx;
            D.fy[i] = fy;
            D.fz[i] = fz;
        }
        D.xdd[i] = xdd;
        D.ydd[i] = ydd;
        D.zdd[i] = zdd;
    }
}

// MODE 0: gather every corner (neighbour subdomains included) and update
//         the node: the fused form of the SBN exchange + node update.
// MODE 1: AddNodeForcesFromElems over this domain's own corners only,
//         writing fx/fy/fz (the partial sums the reference exchanges).
// MODE 2: the node update from fx/fy/fz (after CommSBN added neighbours).
template <int MODE, int BS>
__global__ void __launch_bounds__(BS, min_blocks(kNodalMinBlocks, BS)) k_nodal(SetArgs a, Params P)
{
    pdl_enter();
    const int2 blk = a.blocks[blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    const TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;
    const int i = blk.y + threadIdx.x;
    if (i >= D.numNode) return;
    const int en = D.en;
    const int px = i % en;
    const int t = i / en;
    const int py = t % en;
    const int pz = t / en;

    double fx, fy, fz;
    if (MODE == 0) {
        gather_corners(a.doms, D, px, py, pz, fx, fy, fz, &a.tcs[D.tc]);
    } else if (MODE == 1) {
        DomDev L = D;
        L.tp = 1;  // own corners only
        gather_corners(a.doms, L, px, py, pz, fx, fy, fz, &a.tcs[D.tc]);
        D.fx[i] = fx;
        D.fy[i] = fy;
        D.fz[i] = fz;
        return;
    } else {
        fx = D.fx[i];
        fy = D.fy[i];
        fz = D.fz[i];
    }

    // ApplyAccelerationBoundaryConditionsForNodes: symmetry planes are the
    // px/py/pz == 0 node sets of the domains at the mesh origin faces
    const int bc = (D.col == 0 && px == 0 ? 1 : 0) | (D.row == 0 && py == 0 ? 2 : 0) |
                   (D.plane == 0 && pz == 0 ? 4 : 0);
    advance_node(D, T, P, i, bc, fx, fy, fz, a.materialize, MODE == 0);
}

// Unstructured meshes: AddNodeForcesFromElems (lulesh.cu:1715-1751) over
// each node's run of nodeElemCornerList, in list order, then the node
// update.  The runs of a block's consecutive nodes are contiguous in the
// list; when they fit, the block stages them in shared memory with
// coalesced loads (read straight from the list, each thread's run is an
// 8-int stride: one sector per thread per load), and the corner loads go
// out four corners at a time.
template <int BS>
__global__ void __launch_bounds__(BS, min_blocks(kNodalUMinBlocks, BS)) k_nodal_u(SetArgs a, Params P)
{
    pdl_enter();
    __shared__ int s_list[8 * BS];
    const int2 blk = a.blocks[blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    const TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;  // the whole block
    const int first = blk.y;
    const int last = min(first + BS, D.numNode) - 1;
    if (D.nodeCornerEll) {
        // the run slot-major (uniform per block: no staging, no barrier):
        // eight coalesced loads, then the corners, summed in run order
        const int i = first + threadIdx.x;
        if (i > last) return;
        const int N = D.numNode;
        int k[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) k[j] = D.nodeCornerEll[(size_t)j * N + i];
        double fx = 0.0, fy = 0.0, fz = 0.0;
#pragma unroll
        for (int h = 0; h < 8; h += 4) {
            double vx[4], vy[4], vz[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                vx[q] = vy[q] = vz[q] = 0.0;
                if (k[h + q] >= 0) {
                    const int c = chk_index(k[h + q], 8LL * D.Ep, const_cast<TimeCtl *>(&T),
                                            kChkCorner);
                    vx[q] = ld_corner(D.fx_elem + c);
                    vy[q] = ld_corner(D.fy_elem + c);
                    vz[q] = ld_corner(D.fz_elem + c);
                }
            }
#pragma unroll
            for (int q = 0; q < 4; ++q)
                if (k[h + q] >= 0) {  // a run is a prefix of the slots
                    fx += vx[q];
                    fy += vy[q];
                    fz += vz[q];
                }
        }
        advance_node(D, T, P, i, D.nodeBC[i], fx, fy, fz, a.materialize, true);
        return;
    }
    const long long list_len = 8LL * D.numElem;  // corner-list entries
    const int lo = chk_index(D.nodeElemStart[first], list_len, const_cast<TimeCtl *>(&T),
                             kChkCornerRun);
    const int len = D.nodeElemStart[last] + D.nodeElemCount[last] - lo;
    const bool staged = len <= 8 * BS && lo + (long long)len <= list_len;
    if (staged)
        for (int k = threadIdx.x; k < len; k += BS) s_list[k] = D.nodeElemCornerList[lo + k];
    __syncthreads();
    const int i = first + threadIdx.x;
    if (i > last) return;
    int start = D.nodeElemStart[i], count = D.nodeElemCount[i];
#if LULESH_CHECKED
    if (start < 0 || count < 0 || start + (long long)count > list_len ||
        (staged && (start < lo || start + count > lo + len))) {
        atomicCAS(&const_cast<TimeCtl &>(T).chk, 0, (int)kChkCornerRun);
        start = lo;
        count = 0;
    }
#endif
    const int *list = staged ? s_list + (start - lo) : D.nodeElemCornerList + start;

    double fx = 0.0, fy = 0.0, fz = 0.0;
    int j = 0;
    for (; j + 4 <= count; j += 4) {
        int k[4];
        double vx[4], vy[4], vz[4];
#pragma unroll
        for (int q = 0; q < 4; ++q)
            k[q] = chk_index(list[j + q], 8LL * D.Ep, const_cast<TimeCtl *>(&T), kChkCorner);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            vx[q] = ld_corner(D.fx_elem + k[q]);
            vy[q] = ld_corner(D.fy_elem + k[q]);
            vz[q] = ld_corner(D.fz_elem + k[q]);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            fx += vx[q];
            fy += vy[q];
            fz += vz[q];
        }
    }
    for (; j < count; ++j) {
        const int k = chk_index(list[j], 8LL * D.Ep, const_cast<TimeCtl *>(&T), kChkCorner);
        fx += ld_corner(D.fx_elem + k);
        fy += ld_corner(D.fy_elem + k);
        fz += ld_corner(D.fz_elem + k);
    }
    // symmetry nodes of the mesh's X/Y/Z sets: nodeBC bits 0/1/2
    advance_node(D, T, P, i, D.nodeBC[i], fx, fy, fz, a.materialize, true);
}

void launch_nodal(const SetArgs &a, int nblocks, Params P, cudaStream_t s, int bs, bool u)
{
    if (u) {
        launch_k(k_nodal_u<kNodeBlock>, nblocks, kNodeBlock, s, a.pdl != 0, a, P);
        return;
    }
    switch (bs) {
        case 256: launch_k(k_nodal<0, 256>, nblocks, 256, s, a.pdl != 0, a, P); break;
        case 512: launch_k(k_nodal<0, 512>, nblocks, 512, s, a.pdl != 0, a, P); break;
        default: launch_k(k_nodal<0, kNodeBlock>, nblocks, kNodeBlock, s, a.pdl != 0, a, P); break;
    }
}

void launch_nodal_gather_local(const SetArgs &a, int nblocks, cudaStream_t s)
{
    k_nodal<1, kNodeBlock><<<nblocks, kNodeBlock, 0, s>>>(a, Params{});
}

void launch_nodal_update(const SetArgs &a, int nblocks, Params P, cudaStream_t s)
{
    k_nodal<2, kNodeBlock><<<nblocks, kNodeBlock, 0, s>>>(a, P);
}

// ---------------------------------------------------------------------------
// kinematics: CalcKinematicsAndMonotonicQGradient_kernel, lulesh.cu:3343-3507

template <int BS, bool U = false>
__global__ void __launch_bounds__(BS, min_blocks(kKinMinBlocks, BS)) k_kinematics(SetArgs a)
{
    pdl_enter();
    const int2 blk = a.blocks[LULESH_KIN_REVERSE ? gridDim.x - 1 - blockIdx.x : blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;
    const int k = blk.y + threadIdx.x;
    if (k >= D.numElem) return;

    // all node gathers first (measured on B200 at -s 100: 92 -> 84 us)
    int nodes[8];
    elem_nodes<U>(D, k, nodes);
#pragma unroll
    for (int l = 0; l < 8; ++l) nodes[l] = chk_index(nodes[l], D.numNode, &T, kChkNode);
    double x_local[8], y_local[8], z_local[8];
    double xd_local[8], yd_local[8], zd_local[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        xd_local[l] = D.xd[nodes[l]];
        yd_local[l] = D.yd[nodes[l]];
        zd_local[l] = D.zd[nodes[l]];
    }
    const VelRegs vel{xd_local, yd_local, zd_local};
#pragma unroll
    for (int l = 0; l < 8; ++l) x_local[l] = D.x[nodes[l]];
#pragma unroll
    for (int l = 0; l < 8; ++l) y_local[l] = D.y[nodes[l]];
#pragma unroll
    for (int l = 0; l < 8; ++l) z_local[l] = D.z[nodes[l]];
    kin_elem(D, T, k, x_local, y_local, z_local, vel);
}

void launch_kinematics(const SetArgs &a, int nblocks, Params P, cudaStream_t s, int bs, bool u)
{
    (void)P;
    if (u) {
        launch_k(k_kinematics<kElemBlock, true>, nblocks, kElemBlock, s, a.pdl != 0, a);
        return;
    }
    switch (bs) {
        case 64: launch_k(k_kinematics<64>, nblocks, 64, s, a.pdl != 0, a); break;
        case 256: launch_k(k_kinematics<256>, nblocks, 256, s, a.pdl != 0, a); break;
        default: launch_k(k_kinematics<kElemBlock>, nblocks, kElemBlock, s, a.pdl != 0, a); break;
    }
}

// ---------------------------------------------------------------------------
// eos: monotonic Q region + EOS + volume update + dt constraints

// Boundary-condition mask and the six face-neighbour indices of element z,
// computed from its position: the values SetupConnectivityBC stores in
// elemBC and lxim..lzetap (lulesh.cu:537-686).  Interior neighbours are the
// adjacent elements; a face on the mesh boundary is a symmetry plane at the
// minimum and a free surface at the maximum; a face against another
// subdomain is a comm face whose neighbour is a ghost element (ghost face
// offsets in the order planeMin, planeMax, rowMin, rowMax, colMin, colMax).
// Indices the limiter does not read for a given mask are left as is.
__device__ __forceinline__ void elem_face_links(const DomDev &D, int z, int &bc, int &xm,
                                                int &xp, int &em, int &ep, int &zm, int &zp)
{
    const int nx = D.nx, nn = nx * nx;
    const int ix = z % nx, t = z / nx, iy = t % nx, iz = t / nx;
    bc = 0;
    xm = z - 1;
    xp = z + 1;
    em = z - nx;
    ep = z + nx;
    zm = z - nn;
    zp = z + nn;
    const int last = D.tp - 1;
    if (iz == 0) {
        if (D.plane == 0) bc |= ZETA_M_SYMM;
        else { bc |= ZETA_M_COMM; zm = D.ghost[0] + iy * nx + ix; }
    }
    if (iz == nx - 1) {
        if (D.plane == last) bc |= ZETA_P_FREE;
        else { bc |= ZETA_P_COMM; zp = D.ghost[1] + iy * nx + ix; }
    }
    if (iy == 0) {
        if (D.row == 0) bc |= ETA_M_SYMM;
        else { bc |= ETA_M_COMM; em = D.ghost[2] + iz * nx + ix; }
    }
    if (iy == nx - 1) {
        if (D.row == last) bc |= ETA_P_FREE;
        else { bc |= ETA_P_COMM; ep = D.ghost[3] + iz * nx + ix; }
    }
    if (ix == 0) {
        if (D.col == 0) bc |= XI_M_SYMM;
        else { bc |= XI_M_COMM; xm = D.ghost[4] + iz * nx + iy; }
    }
    if (ix == nx - 1) {
        if (D.col == last) bc |= XI_P_FREE;
        else { bc |= XI_P_COMM; xp = D.ghost[5] + iz * nx + iy; }
    }
}

// one direction of the monotonic limiter, lulesh.cu:3595-3624
__device__ __forceinline__ double mono_limiter(const double *delv, int i, int bc, int mmask,
                                               int msymm, int mfree, int pmask, int psymm,
                                               int pfree, int lm, int lp, double mult,
                                               double maxslope, double ptiny, int nlinks,
                                               TimeCtl *T)
{
    const double norm = 1. / (delv[i] + ptiny);
    double delvm, delvp;
    const int mb = bc & mmask, pb = bc & pmask;
    if (mb == msymm)
        delvm = delv[i];
    else if (mb == mfree)
        delvm = 0.0;
    else  // 0 or *_COMM: neighbour or ghost element
        delvm = delv[chk_index(lm, nlinks, T, kChkLink)];
    if (pb == psymm)
        delvp = delv[i];
    else if (pb == pfree)
        delvp = 0.0;
    else
        delvp = delv[chk_index(lp, nlinks, T, kChkLink)];
    delvm = delvm * norm;
    delvp = delvp * norm;
    double phi = .5 * (delvm + delvp);
    delvm *= mult;
    delvp *= mult;
    if (delvm < phi) phi = delvm;
    if (delvp < phi) phi = delvp;
    if (phi < 0.) phi = 0.;
    if (phi > maxslope) phi = maxslope;
    return phi;
}

// mono_limiter with the minus and plus neighbours read from their own
// arrays (dm[lm], dp[lp]): a comm face's neighbour element is then read in
// the neighbouring subdomain instead of from this subdomain's ghost copy.
__device__ __forceinline__ double mono_limiter_split(const double *delv, const double *dm,
                                                     const double *dp, int i, int bc,
                                                     int mmask, int msymm, int mfree,
                                                     int pmask, int psymm, int pfree, int lm,
                                                     int lp, double mult, double maxslope,
                                                     double ptiny, int nm, int np, TimeCtl *T)
{
    const double norm = 1. / (delv[i] + ptiny);
    double delvm, delvp;
    const int mb = bc & mmask, pb = bc & pmask;
    if (mb == msymm)
        delvm = delv[i];
    else if (mb == mfree)
        delvm = 0.0;
    else
        delvm = dm[chk_index(lm, nm, T, kChkLink)];
    if (pb == psymm)
        delvp = delv[i];
    else if (pb == pfree)
        delvp = 0.0;
    else
        delvp = dp[chk_index(lp, np, T, kChkLink)];
    delvm = delvm * norm;
    delvp = delvp * norm;
    double phi = .5 * (delvm + delvp);
    delvm *= mult;
    delvp *= mult;
    if (delvm < phi) phi = delvm;
    if (delvp < phi) phi = delvp;
    if (phi < 0.) phi = 0.;
    if (phi > maxslope) phi = maxslope;
    return phi;
}

// CalcPressureForElems_device, lulesh.cu:3764-3791
__device__ __forceinline__ void calc_pressure(double &p_new, double &bvc, double &pbvc,
                                              double &e_old, double &compression,
                                              double &vnewc, double pmin, double p_cut,
                                              double eosvmax)
{
    const double c1s = 2.0 / 3.0;
    double p_temp;
    bvc = c1s * (compression + 1.);
    pbvc = c1s;
    p_temp = bvc * e_old;
    if (fabs(p_temp) < p_cut) p_temp = 0.0;
    if (vnewc >= eosvmax) p_temp = 0.0;
    if (p_temp < pmin) p_temp = pmin;
    p_new = p_temp;
}

// x / rho0 (the reference density).  With RHO1 the density is 1.0, and
// x / 1.0 is x exactly in IEEE-754 arithmetic, so the division is left
// out; the results are the same bits either way.
template <bool RHO1>
__device__ __forceinline__ double per_rho0(double x, double rho0)
{
    return RHO1 ? x : x / rho0;
}

// CalcEnergyForElems_device, lulesh.cu:3867-3974
template <bool RHO1>
__device__ __forceinline__ void calc_energy(double &p_new, double &e_new, double &q_new,
                                            double &bvc, double &pbvc, double &p_old,
                                            double &e_old, double &q_old, double &compression,
                                            double &compHalfStep, double &vnewc, double &work,
                                            double &delvc, double pmin, double p_cut,
                                            double e_cut, double q_cut, double emin,
                                            double &qq, double &ql, double &rho0,
                                            double &eosvmax)
{
    const double sixth = 1.0 / 6.0;
    double pHalfStep;
    e_new = e_old - 0.5 * delvc * (p_old + q_old) + 0.5 * work;
    if (e_new < emin) e_new = emin;
    calc_pressure(pHalfStep, bvc, pbvc, e_new, compHalfStep, vnewc, pmin, p_cut, eosvmax);
    const double vhalf = 1. / (1. + compHalfStep);
    if (delvc > 0.) {
        q_new = 0.;
    } else {
        double ssc = per_rho0<RHO1>(pbvc * e_new + vhalf * vhalf * bvc * pHalfStep, rho0);
        if (ssc <= .1111111e-36)
            ssc = .3333333e-18;
        else
            ssc = sqrt(ssc);
        q_new = (ssc * ql + qq);
    }
    e_new = e_new + 0.5 * delvc * (3.0 * (p_old + q_old) - 4.0 * (pHalfStep + q_new));
    e_new += 0.5 * work;
    if (fabs(e_new) < e_cut) e_new = 0.;
    if (e_new < emin) e_new = emin;
    calc_pressure(p_new, bvc, pbvc, e_new, compression, vnewc, pmin, p_cut, eosvmax);
    double q_tilde;
    if (delvc > 0.) {
        q_tilde = 0.;
    } else {
        double ssc = per_rho0<RHO1>(pbvc * e_new + vnewc * vnewc * bvc * p_new, rho0);
        if (ssc <= .1111111e-36)
            ssc = .3333333e-18;
        else
            ssc = sqrt(ssc);
        q_tilde = (ssc * ql + qq);
    }
    e_new = e_new - (7.0 * (p_old + q_old) - 8.0 * (pHalfStep + q_new) + (p_new + q_tilde)) *
                        delvc * sixth;
    if (fabs(e_new) < e_cut) e_new = 0.;
    if (e_new < emin) e_new = emin;
    calc_pressure(p_new, bvc, pbvc, e_new, compression, vnewc, pmin, p_cut, eosvmax);
    if (delvc <= 0.) {
        double ssc = per_rho0<RHO1>(pbvc * e_new + vnewc * vnewc * bvc * p_new, rho0);
        if (ssc <= .1111111e-36)
            ssc = .3333333e-18;
        else
            ssc = sqrt(ssc);
        q_new = (ssc * ql + qq);
        if (fabs(q_new) < q_cut) q_new = 0.;
    }
}

// The rep loop of ApplyMaterialPropertiesAndUpdateVolume_kernel
// (lulesh.cu:4045-4083), the reference's cost model: every rep re-evaluates
// the EOS from the same inputs (the loop is pure).
template <bool RHO1>
__device__ __forceinline__ void eos_reps(int rep, double e_temp, double p_temp, double q_temp,
                                         double qq_temp, double ql_temp, double delvc_temp,
                                         double vnewc, double eosvmin, double eosvmax,
                                         double rho0, const Params &P, double &p_new,
                                         double &e_new, double &q_new, double &bvc,
                                         double &pbvc)
{
    double e_old, delvc, p_old, q_old, compression, compHalfStep, qq_old, ql_old, work;
    for (int r = 0; r < rep; r++) {
        e_old = e_temp;
        p_old = p_temp;
        q_old = q_temp;
        qq_old = qq_temp;
        ql_old = ql_temp;
        delvc = delvc_temp;
        work = 0.;
        double vchalf;
        compression = 1. / vnewc - 1.;
        vchalf = vnewc - delvc * .5;
        compHalfStep = 1. / vchalf - 1.;
        if (eosvmin != 0.) {
            if (vnewc <= eosvmin) compHalfStep = compression;
        }
        if (eosvmax != 0.) {
            if (vnewc >= eosvmax) {
                p_old = 0.;
                compression = 0.;
                compHalfStep = 0.;
            }
        }
        calc_energy<RHO1>(p_new, e_new, q_new, bvc, pbvc, p_old, e_old, q_old, compression,
                          compHalfStep, vnewc, work, delvc, P.pmin, P.p_cut, P.e_cut, P.q_cut,
                          P.emin, qq_old, ql_old, rho0, eosvmax);
    }
}

__device__ __forceinline__ double warp_min(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// SUB: a subdomain set's fused cycle, which reads a comm face's neighbour
// element in the neighbouring subdomain (no MonoQ ghost copy)
template <int BS, bool U = false, bool SUB = false>
__global__ void __launch_bounds__(BS, min_blocks(kEosMinBlocks, BS)) k_eos(SetArgs a, Params P)
{
    pdl_enter();
    const int2 blk = a.blocks[LULESH_EOS_REVERSE ? gridDim.x - 1 - blockIdx.x : blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;  // uniform per block
    const int i = blk.y + threadIdx.x;
    double dtc = 1.0e+20, dth = 1.0e+20;
    if (i < D.numElem) {
        // The element of this slot and its rep count.  The reference visits
        // regElemlist and finds the rep by region (giveMyRegion,
        // lulesh.cu:3976-3984); here slots are grouped by rep class
        // (HostDomain::eosOrder), which keeps the trip count uniform per warp
        // with denser loads (measured 98 us vs 99 us regElemlist order and
        // 108 us natural order at -s 100).
        const int zidx = chk_index(D.eosOrder[i], D.numElem, &T, kChkSlot);
        int cls = 0;
        while (cls < D.eosNumClass - 1 && i >= D.eosClassEnd[cls]) ++cls;
        const int rep = D.eosClassRep[cls];

        // ---- CalcMonotonicQRegionForElems_kernel, lulesh.cu:3586-3724
        const double ptiny = 1.e-36;
        int bcMask, lxm, lxp, lem, lep, lzm, lzp;
        if (U) {  // the mesh's own links and boundary mask
            bcMask = D.elemBC[zidx];
            lxm = D.lxim[zidx];
            lxp = D.lxip[zidx];
            lem = D.letam[zidx];
            lep = D.letap[zidx];
            lzm = D.lzetam[zidx];
            lzp = D.lzetap[zidx];
        } else {
            elem_face_links(D, zidx, bcMask, lxm, lxp, lem, lep, lzm, lzp);
        }
        const double mult = P.monoq_limiter_mult, maxs = P.monoq_max_slope;
        double phixi, phieta, phizeta;
        if (SUB) {
            // comm faces: the mirrored element of the neighbour's opposite
            // face layer, where k_monoq_ghost would copy it from
            const int nx = D.nx;
            const int ix = zidx % nx, t = zidx / nx, iy = t % nx, iz = t / nx;
            const DomDev *sxm = &D, *sxp = &D, *sem = &D, *sep = &D, *szm = &D, *szp = &D;
            if (bcMask & XI_M_COMM) {
                sxm = &a.doms[D.nbr[0 + 3 + 9]];
                lxm = (iz * nx + iy) * nx + (nx - 1);
            }
            if (bcMask & XI_P_COMM) {
                sxp = &a.doms[D.nbr[2 + 3 + 9]];
                lxp = (iz * nx + iy) * nx;
            }
            if (bcMask & ETA_M_COMM) {
                sem = &a.doms[D.nbr[1 + 0 + 9]];
                lem = (iz * nx + (nx - 1)) * nx + ix;
            }
            if (bcMask & ETA_P_COMM) {
                sep = &a.doms[D.nbr[1 + 6 + 9]];
                lep = (iz * nx) * nx + ix;
            }
            if (bcMask & ZETA_M_COMM) {
                szm = &a.doms[D.nbr[1 + 3 + 0]];
                lzm = ((nx - 1) * nx + iy) * nx + ix;
            }
            if (bcMask & ZETA_P_COMM) {
                szp = &a.doms[D.nbr[1 + 3 + 18]];
                lzp = iy * nx + ix;
            }
            phixi = mono_limiter_split(D.delv_xi, sxm->delv_xi, sxp->delv_xi, zidx, bcMask, XI_M,
                                       XI_M_SYMM, XI_M_FREE, XI_P, XI_P_SYMM, XI_P_FREE, lxm, lxp,
                                       mult, maxs, ptiny, sxm->allElem, sxp->allElem, &T);
            phieta = mono_limiter_split(D.delv_eta, sem->delv_eta, sep->delv_eta, zidx, bcMask,
                                        ETA_M, ETA_M_SYMM, ETA_M_FREE, ETA_P, ETA_P_SYMM,
                                        ETA_P_FREE, lem, lep, mult, maxs, ptiny, sem->allElem,
                                        sep->allElem, &T);
            phizeta = mono_limiter_split(D.delv_zeta, szm->delv_zeta, szp->delv_zeta, zidx,
                                         bcMask, ZETA_M, ZETA_M_SYMM, ZETA_M_FREE, ZETA_P,
                                         ZETA_P_SYMM, ZETA_P_FREE, lzm, lzp, mult, maxs, ptiny,
                                         szm->allElem, szp->allElem, &T);
        } else {
            phixi = mono_limiter(D.delv_xi, zidx, bcMask, XI_M, XI_M_SYMM, XI_M_FREE, XI_P,
                                 XI_P_SYMM, XI_P_FREE, lxm, lxp, mult, maxs, ptiny, D.allElem, &T);
            phieta = mono_limiter(D.delv_eta, zidx, bcMask, ETA_M, ETA_M_SYMM, ETA_M_FREE, ETA_P,
                                  ETA_P_SYMM, ETA_P_FREE, lem, lep, mult, maxs, ptiny, D.allElem,
                                  &T);
            phizeta = mono_limiter(D.delv_zeta, zidx, bcMask, ZETA_M, ZETA_M_SYMM, ZETA_M_FREE,
                                   ZETA_P, ZETA_P_SYMM, ZETA_P_FREE, lzm, lzp, mult, maxs, ptiny,
                                   D.allElem, &T);
        }
        const double vdov_z = D.vdov[zidx];
        const double vnew_z = D.vnew[zidx];
        double qlin, qquad;
        if (vdov_z > 0.) {
            qlin = 0.;
            qquad = 0.;
        } else {
            double delvxxi = D.delv_xi[zidx] * D.delx_xi[zidx];
            double delvxeta = D.delv_eta[zidx] * D.delx_eta[zidx];
            double delvxzeta = D.delv_zeta[zidx] * D.delx_zeta[zidx];
            if (delvxxi > 0.) delvxxi = 0.;
            if (delvxeta > 0.) delvxeta = 0.;
            if (delvxzeta > 0.) delvxzeta = 0.;
            const double rho = D.elemMass[zidx] / (D.volo[zidx] * vnew_z);
            qlin = -P.qlc_monoq * rho *
                   (delvxxi * (1. - phixi) + delvxeta * (1. - phieta) +
                    delvxzeta * (1. - phizeta));
            qquad = P.qqc_monoq * rho *
                    (delvxxi * delvxxi * (1. - phixi * phixi) +
                     delvxeta * delvxeta * (1. - phieta * phieta) +
                     delvxzeta * delvxzeta * (1. - phizeta * phizeta));
        }
        const double q_old_z = D.q[zidx];
        if (q_old_z > P.qstop) atomicMin(&T.bad_q, zidx);
        if (a.materialize) {
            D.qq[zidx] = qquad;
            D.ql[zidx] = qlin;
        }

        // ---- ApplyMaterialPropertiesAndUpdateVolume_kernel, lulesh.cu:4025-4096
        double eosvmin = P.eosvmin, eosvmax = P.eosvmax;
        double vnewc = vnew_z;
        if (eosvmin != 0.) {
            if (vnewc < eosvmin) vnewc = eosvmin;
        }
        if (eosvmax != 0.) {
            if (vnewc > eosvmax) vnewc = eosvmax;
        }
        double vc = D.v[zidx];
        if (eosvmin != 0.) {
            if (vc < eosvmin) vc = eosvmin;
        }
        if (eosvmax != 0.) {
            if (vc > eosvmax) vc = eosvmax;
        }
        if (vc <= 0.) atomicMin(&T.bad_vol, zidx);

        double p_new = 0., e_new = 0., q_new = 0., bvc = 0., pbvc = 0.;
        const double e_temp = D.e[zidx];
        const double p_temp = D.p[zidx];
        const double delvc_temp = D.delv[zidx];
        const double rho0 = P.refdens;
        // the reference density is 1.0 in every sedov problem (uniform branch)
        const bool rho1 = rho0 == 1.0;
        if (rho1)
            eos_reps<true>(rep, e_temp, p_temp, q_old_z, qquad, qlin, delvc_temp, vnewc,
                           eosvmin, eosvmax, rho0, P, p_new, e_new, q_new, bvc, pbvc);
        else
            eos_reps<false>(rep, e_temp, p_temp, q_old_z, qquad, qlin, delvc_temp, vnewc,
                            eosvmin, eosvmax, rho0, P, p_new, e_new, q_new, bvc, pbvc);
        D.p[zidx] = p_new;
        D.e[zidx] = e_new;
        D.q[zidx] = q_new;

        // CalcSoundSpeedForElems_device, lulesh.cu:3795-3809
        double ssTmp = pbvc * e_new + vnewc * vnewc * bvc * p_new;
        if (!rho1) ssTmp = ssTmp / rho0;
        if (ssTmp <= .1111111e-36)
            ssTmp = .3333333e-18;
        else
            ssTmp = sqrt(ssTmp);
        D.ss[zidx] = ssTmp;

        // UpdateVolumesForElems_device, lulesh.cu:3850-3861
        double tmpV = vnew_z;
        if (fabs(tmpV - 1.0) < P.v_cut) tmpV = 1.0;
        D.v[zidx] = tmpV;

        // CalcTimeConstraintsForElems_kernel body, lulesh.cu:4246-4279
        const double qqc2 = 64.0 * P.qqc * P.qqc;
        const double vdov_tmp = vdov_z;
        if (vdov_tmp != 0.) {
            const double dtdvov = P.dvovmax / (fabs(vdov_tmp) + 1.e-20);
            if (dth > dtdvov) dth = dtdvov;
        }
        const double ss_tmp = ssTmp;
        const double area_tmp = D.arealg[zidx];
        double dtf = ss_tmp * ss_tmp;
        dtf += ((vdov_tmp < 0.) ? qqc2 * area_tmp * area_tmp * vdov_tmp * vdov_tmp : 0.);
        dtf = area_tmp / sqrt(dtf);
        if (vdov_tmp != 0. && dtf < dtc) dtc = dtf;
    }
    // block minimum (exact, order-free), one atomic per block
    __shared__ double s_c[BS / 32], s_h[BS / 32];
    dtc = warp_min(dtc);
    dth = warp_min(dth);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        s_c[warp] = dtc;
        s_h[warp] = dth;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double c = s_c[0], h = s_h[0];
#pragma unroll
        for (int w = 1; w < BS / 32; ++w) {
            c = fmin(c, s_c[w]);
            h = fmin(h, s_h[w]);
        }
        if (c < 1.0e+20) atomicMin(&T.min_courant, dbits(c));
        if (h < 1.0e+20) atomicMin(&T.min_hydro, dbits(h));
    }
}

void launch_eos(const SetArgs &a, int nblocks, Params P, cudaStream_t s, int bs, bool u,
                bool sub)
{
    if (u) {
        launch_k(k_eos<kElemBlock, true>, nblocks, kElemBlock, s, a.pdl != 0, a, P);
        return;
    }
    if (sub) {  // subdomain sets take 128-element blocks only
        launch_k(k_eos<kElemBlock, false, true>, nblocks, kElemBlock, s, a.pdl != 0, a, P);
        return;
    }
    switch (bs) {
        case 64: launch_k(k_eos<64>, nblocks, 64, s, a.pdl != 0, a, P); break;
        case 256: launch_k(k_eos<256>, nblocks, 256, s, a.pdl != 0, a, P); break;
        default: launch_k(k_eos<kElemBlock>, nblocks, kElemBlock, s, a.pdl != 0, a, P); break;
    }
}

// ---------------------------------------------------------------------------
// fused halo kernels of a subdomain set

// CommSyncPosVel semantics (lulesh-comms-gpu.cu:1231-1661): a node shared by
// several subdomains takes x,y,z,xd,yd,zd from the subdomain that holds it
// on its minimum faces only (the "+side owner"), which never writes it here.
// Blocks cover the max-side faces only (sync blocks, build_tables): block b
// takes face blocks[b].y >> 24 of domain blocks[b].x from item
// (blocks[b].y & 0xffffff) on.  Face 0 holds the nodes with px = nx, face 1
// those with py = nx and px < nx, face 2 those with pz = nx and px, py < nx,
// so every node of a max-side face is visited once; the copy itself is
// decided from the node's position, as for the whole node range.
__global__ void k_posvel_sync(SetArgs a)
{
    pdl_enter();
    const int2 blk = a.blocks[blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    const TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;
    const int face = blk.y >> 24;
    const int item = (blk.y & 0xffffff) + threadIdx.x;
    const int en = D.en, nx = D.nx, tp = D.tp;
    int px, py, pz;
    if (face == 0) {
        if (item >= en * en) return;
        px = nx, py = item % en, pz = item / en;
    } else if (face == 1) {
        if (item >= nx * en) return;
        px = item % nx, py = nx, pz = item / nx;
    } else {
        if (item >= nx * nx) return;
        px = item % nx, py = item / nx, pz = nx;
    }
    const int i = (pz * en + py) * en + px;
    const int sx = (px == nx && D.col < tp - 1) ? 1 : 0;
    const int sy = (py == nx && D.row < tp - 1) ? 1 : 0;
    const int sz = (pz == nx && D.plane < tp - 1) ? 1 : 0;
    if ((sx | sy | sz) == 0) return;
    const int nb = D.nbr[(sx + 1) + 3 * (sy + 1) + 9 * (sz + 1)];
    if (nb < 0) return;
    const DomDev &O = a.doms[nb];
    const int j = chk_index(((pz - sz * nx) * en + (py - sy * nx)) * en + (px - sx * nx),
                            O.numNode, &a.tcs[D.tc], kChkNode);
    D.x[i] = O.x[j];
    D.y[i] = O.y[j];
    D.z[i] = O.z[j];
    D.xd[i] = O.xd[j];
    D.yd[i] = O.yd[j];
    D.zd[i] = O.zd[j];
}

void launch_posvel_sync(const SetArgs &a, int nblocks, cudaStream_t s)
{
    launch_k(k_posvel_sync, nblocks, kNodeBlock, s, a.pdl != 0, a);
}

// CommMonoQ semantics (lulesh-comms-gpu.cu:1665-1806): the delv_* ghost
// faces (offsets of SetupConnectivityBC, lulesh.cu:581-615) receive the
// neighbour's boundary element layer.  Block b covers face blocks[b].y>>24
// of domain blocks[b].x, items (blocks[b].y & 0xffffff) onward.
__global__ void k_monoq_ghost(SetArgs a)
{
    pdl_enter();
    const int2 blk = a.blocks[blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    const TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;
    const int f = blk.y >> 24;
    const int item = (blk.y & 0xffffff) + threadIdx.x;
    const int nx = D.nx;
    if (item >= nx * nx || D.ghost[f] < 0) return;
    const int a0 = item / nx, b0 = item % nx;  // (plane|row, row|col) of the face
    int dxn = 0, dyn = 0, dzn = 0, src;
    switch (f) {
        case 0: dzn = -1; src = ((nx - 1) * nx + a0) * nx + b0; break;  // row a0, col b0
        case 1: dzn = 1; src = (0 * nx + a0) * nx + b0; break;
        case 2: dyn = -1; src = (a0 * nx + (nx - 1)) * nx + b0; break;  // plane a0, col b0
        case 3: dyn = 1; src = (a0 * nx + 0) * nx + b0; break;
        case 4: dxn = -1; src = (a0 * nx + b0) * nx + (nx - 1); break;  // plane a0, row b0
        default: dxn = 1; src = (a0 * nx + b0) * nx + 0; break;
    }
    const int nb = D.nbr[(dxn + 1) + 3 * (dyn + 1) + 9 * (dzn + 1)];
    if (nb < 0) return;
    const DomDev &N = a.doms[nb];
    const int g = chk_index(D.ghost[f] + item, D.allElem, &a.tcs[D.tc], kChkLink);
    src = chk_index(src, N.numElem, &a.tcs[D.tc], kChkLink);
    D.delv_xi[g] = N.delv_xi[src];
    D.delv_eta[g] = N.delv_eta[src];
    D.delv_zeta[g] = N.delv_zeta[src];
}

void launch_monoq_ghost(const SetArgs &a, int nblocks, cudaStream_t s)
{
    launch_k(k_monoq_ghost, nblocks, kElemBlock, s, a.pdl != 0, a);
}

}  // namespace lulesh
