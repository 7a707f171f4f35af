// mixed.cu -- mixed-precision variants of the force, nodal and kinematics
// kernels (LULESH_FLAG_MIXED).
//
// FP32: the element-local stress / FB-hourglass arithmetic of
//   CalcVolumeForceForElems_kernel (lulesh.cu:2080-2259) and the
//   characteristic length, velocity gradient and monotonic-Q gradients of
//   CalcKinematicsAndMonotonicQGradient_kernel (lulesh.cu:3343-3507).
//   Every one of these is a function of coordinate DIFFERENCES, so the
//   kernels form x[k] - x[0] in FP64 and hand FP32 only the small,
//   well-conditioned differences; velocities go to FP32 directly.
// FP32 storage, compensated sum: corner forces are stored as FP32 and each
//   node adds its eight corners with Neumaier's compensated summation, then
//   converts (sum + compensation) to FP64.
// FP64 (unchanged): element volume, relative volume and delv (delv is a
//   difference of two numbers near 1, which FP32 would leave with 3-5
//   digits), the node update, the EOS, and the dt reduction.
#include <climits>

#include "elem_math.cuh"
#include "kernels.cuh"

namespace lulesh {

// Resident blocks per SM asked of the compiler for the mixed kernels:
// 4 (128 registers, no spills) measured best on B200 at -s 120, two
// alternating runs each, identical results: force 137 us against 181 at 5
// blocks (96 registers, spills), 147 at 3 and 311 at 6; kinematics 114.8 us
// against 115.7 at 5 and 125.9 at 3; the cycle 498 us against 545 at 5.
#ifndef LULESH_MIXED_FORCE_MINB
#define LULESH_MIXED_FORCE_MINB 4
#endif
#ifndef LULESH_MIXED_KIN_MINB
#define LULESH_MIXED_KIN_MINB 4
#endif

__device__ __forceinline__ void elem_nodes_m(const DomDev &D, int el, int n[8])
{
    const int nx = D.nx, en = D.en;
    const int ix = el % nx, t = el / nx, iy = t % nx, iz = t / nx;
    const int n0 = (iz * en + iy) * en + ix;
    n[0] = n0;
    n[1] = n0 + 1;
    n[2] = n0 + en + 1;
    n[3] = n0 + en;
    n[4] = n0 + en * en;
    n[5] = n0 + en * en + 1;
    n[6] = n0 + en * en + en + 1;
    n[7] = n0 + en * en + en;
}

template <bool HG>
__global__ void __launch_bounds__(kElemBlock, LULESH_MIXED_FORCE_MINB)
    k_force_mixed(SetArgs a, Params P, const CornerF32 *cfs)
{
    pdl_enter();
    const int2 blk = a.blocks[blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;
    const int elem = blk.y + threadIdx.x;
    if (elem >= D.numElem) return;
    const CornerF32 cf = cfs[blk.x];

    int n[8];
    elem_nodes_m(D, elem, n);
#pragma unroll
    for (int i = 0; i < 8; ++i) n[i] = chk_index(n[i], D.numNode, &T, kChkNode);
    // all node gathers first: the velocities arrive while the coordinate
    // arithmetic runs
    float vx[8], vy[8], vz[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        if (HG) {
            vx[i] = (float)D.xd[n[i]];
            vy[i] = (float)D.yd[n[i]];
            vz[i] = (float)D.zd[n[i]];
        }
    }
    const double x0 = D.x[n[0]], y0 = D.y[n[0]], z0 = D.z[n[0]];
    float xn[8], yn[8], zn[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        xn[i] = (float)(D.x[n[i]] - x0);
        yn[i] = (float)(D.y[n[i]] - y0);
        zn[i] = (float)(D.z[n[i]] - z0);
    }
    const double volume = D.v[elem];
    const double detd = D.volo[elem] * volume;
    if (volume < 0.) atomicMin(&T.bad_vol, elem);
    float det = (float)detd;
    const float volinv = 1.0f / det;
    const float coefficient =
        (float)(-P.hgcoef * 0.01 * D.ss[elem] * D.elemMass[elem]) / cbrtf(det);
    const float sigxx = (float)(-D.p[elem] - D.q[elem]);

    float dvdxn[8], dvdyn[8], dvdzn[8], hourgam[8][4];
    elem_volume_derivative(dvdxn, dvdyn, dvdzn, xn, yn, zn);
    hourglass_modes(xn, yn, zn, dvdxn, dvdyn, dvdzn, hourgam, volinv);
    float B[3][8];
    shape_function_derivatives(xn, yn, zn, B, &det);
    elem_node_normals(B[0], B[1], B[2], xn, yn, zn);
    if (det < 0.f) atomicMin(&T.bad_vol, elem);
    float hgfx[8], hgfy[8], hgfz[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        hgfx[i] = -(sigxx * B[0][i]);
        hgfy[i] = -(sigxx * B[1][i]);
        hgfz[i] = -(sigxx * B[2][i]);
    }
    if (HG) {
        fb_hourglass_component(vx, hourgam, coefficient, hgfx);
        fb_hourglass_component(vy, hourgam, coefficient, hgfy);
        fb_hourglass_component(vz, hourgam, coefficient, hgfz);
    }
    // written once, read once by the nodal gather: evict-first
    const int Ep = D.Ep;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        __stcs(cf.fx + elem + Ep * k, hgfx[k]);
        __stcs(cf.fy + elem + Ep * k, hgfy[k]);
        __stcs(cf.fz + elem + Ep * k, hgfz[k]);
    }
}

void launch_force_mixed(const SetArgs &a, int nblocks, Params P, const CornerF32 *cf,
                        cudaStream_t s)
{
    if (P.hgcoef > 0.0)
        launch_k(k_force_mixed<true>, nblocks, kElemBlock, s, a.pdl != 0, a, P, cf);
    else
        launch_k(k_force_mixed<false>, nblocks, kElemBlock, s, a.pdl != 0, a, P, cf);
}

// Neumaier's compensated addition: s + c carries the sum of all terms
__device__ __forceinline__ void comp_add(float &s, float &c, float v)
{
    const float t = s + v;
    if (fabsf(s) >= fabsf(v))
        c += (s - t) + v;
    else
        c += (v - t) + s;
    s = t;
}

// Resident blocks per SM for the mixed node update, whose 24 corner loads
// are all issued before the compensated sums: 10 (48 registers) measured
// best on B200 at -s 120 (57.4 us against 57.7 at 8, 59.2 at 12 and 75.5
// at 16; 83.7 us with the loads interleaved with the sums at 16).
#ifndef LULESH_MIXED_NODAL_MINB
#define LULESH_MIXED_NODAL_MINB 10
#endif

__global__ void __launch_bounds__(kNodeBlock, min_blocks(LULESH_MIXED_NODAL_MINB, kNodeBlock))
    k_nodal_mixed(SetArgs a, Params P, const CornerF32 *cfs)
{
    pdl_enter();
    const int2 blk = a.blocks[blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    const TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;
    const int i = blk.y + threadIdx.x;
    if (i >= D.numNode) return;
    const CornerF32 cf = cfs[blk.x];
    const int en = D.en, nx = D.nx;
    const int px = i % en, t = i / en, py = t % en, pz = t / en;
    float sx = 0.f, sy = 0.f, sz = 0.f, cx = 0.f, cy = 0.f, cz = 0.f;
    const int ox[8] = {0, 1, 1, 0, 0, 1, 1, 0}, oy[8] = {0, 0, 1, 1, 0, 0, 1, 1},
              oz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    // all 24 corner loads first, then the compensated sums in corner order
    float vx[8], vy[8], vz[8];
    bool in[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int ex = px - ox[j], ey = py - oy[j], ez = pz - oz[j];
        in[j] = (unsigned)ex < (unsigned)nx && (unsigned)ey < (unsigned)nx &&
                (unsigned)ez < (unsigned)nx;
        vx[j] = vy[j] = vz[j] = 0.f;
        if (in[j]) {
            const int idx = chk_index(j * D.Ep + (ez * nx + ey) * nx + ex, 8LL * D.Ep,
                                      &a.tcs[D.tc], kChkCorner);
            vx[j] = __ldcs(cf.fx + idx);
            vy[j] = __ldcs(cf.fy + idx);
            vz[j] = __ldcs(cf.fz + idx);
        }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        if (in[j]) {
            comp_add(sx, cx, vx[j]);
            comp_add(sy, cy, vy[j]);
            comp_add(sz, cz, vz[j]);
        }
    }
    const double fx = (double)sx + (double)cx;
    const double fy = (double)sy + (double)cy;
    const double fz = (double)sz + (double)cz;
    const double one_over_nMass = 1. / D.nodalMass[i];
    double xdd = fx * one_over_nMass, ydd = fy * one_over_nMass, zdd = fz * one_over_nMass;
    if (D.col == 0 && px == 0) xdd = 0.0;
    if (D.row == 0 && py == 0) ydd = 0.0;
    if (D.plane == 0 && pz == 0) zdd = 0.0;
    const double dt = T.deltatime, u_cut = P.u_cut;
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
    if (a.materialize) {
        D.fx[i] = fx;
        D.fy[i] = fy;
        D.fz[i] = fz;
        D.xdd[i] = xdd;
        D.ydd[i] = ydd;
        D.zdd[i] = zdd;
    }
}

void launch_nodal_mixed(const SetArgs &a, int nblocks, Params P, const CornerF32 *cf,
                        cudaStream_t s)
{
    launch_k(k_nodal_mixed, nblocks, kNodeBlock, s, a.pdl != 0, a, P, cf);
}

__global__ void __launch_bounds__(kElemBlock, LULESH_MIXED_KIN_MINB)
    k_kinematics_mixed(SetArgs a, Params P)
{
    pdl_enter();
    const int2 blk = a.blocks[LULESH_KIN_REVERSE ? gridDim.x - 1 - blockIdx.x : blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;
    const int k = blk.y + threadIdx.x;
    if (k >= D.numElem) return;
    int nodes[8];
    elem_nodes_m(D, k, nodes);
#pragma unroll
    for (int l = 0; l < 8; ++l) nodes[l] = chk_index(nodes[l], D.numNode, &T, kChkNode);
    // velocities gathered first (used after the FP64 volume)
    float xv[8], yv[8], zv[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        xv[l] = (float)D.xd[nodes[l]];
        yv[l] = (float)D.yd[nodes[l]];
        zv[l] = (float)D.zd[nodes[l]];
    }
    // FP64: volume and relative volume (they feed delv)
    double xd64[8], yd64[8], zd64[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        xd64[l] = D.x[nodes[l]];
        yd64[l] = D.y[nodes[l]];
        zd64[l] = D.z[nodes[l]];
    }
    const double volume = elem_volume(xd64, yd64, zd64);
    const double relativeVolume = volume / D.volo[k];
    D.vnew[k] = relativeVolume;
    D.delv[k] = relativeVolume - D.v[k];
    // FP32: everything else, on coordinates relative to corner 0
    float xl[8], yl[8], zl[8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        xl[l] = (float)(xd64[l] - xd64[0]);
        yl[l] = (float)(yd64[l] - yd64[0]);
        zl[l] = (float)(zd64[l] - zd64[0]);
    }
    D.arealg[k] = (double)elem_characteristic_length(xl, yl, zl, (float)volume);
    const float dt2 = (float)(0.5 * T.deltatime);
    float xh[8], yh[8], zh[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        xh[j] = xl[j] - dt2 * xv[j];
        yh[j] = yl[j] - dt2 * yv[j];
        zh[j] = zl[j] - dt2 * zv[j];
    }
    float B[3][8], detJ, Dv[3];
    shape_function_derivatives(xh, yh, zh, B, &detJ);
    elem_velocity_divergence(xv, yv, zv, B, detJ, Dv);
    D.vdov[k] = (double)(Dv[0] + Dv[1] + Dv[2]);
    const float vol = (float)(D.volo[k] * relativeVolume);
    float dxz, dvz, dxx, dvx, dxe, dve;
    mono_gradient(xl, yl, zl, xv, yv, zv, vol, &dxz, &dvz, &dxx, &dvx, &dxe, &dve);
    D.delx_zeta[k] = dxz;
    D.delv_zeta[k] = dvz;
    D.delx_xi[k] = dxx;
    D.delv_xi[k] = dvx;
    D.delx_eta[k] = dxe;
    D.delv_eta[k] = dve;
    if (relativeVolume < 0) atomicMin(&T.bad_vol, k);
}

void launch_kinematics_mixed(const SetArgs &a, int nblocks, Params P, cudaStream_t s)
{
    launch_k(k_kinematics_mixed, nblocks, kElemBlock, s, a.pdl != 0, a, P);
}

}  // namespace lulesh
