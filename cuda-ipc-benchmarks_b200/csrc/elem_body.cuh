// elem_body.cuh -- per-element bodies of the FP64 force and kinematics
// kernels.  Each body receives the element's eight gathered node values and
// does the rest: element loads, arithmetic, stores.  The launch that
// gathers (kernels.cu) issues all 48 node loads before any arithmetic.
#pragma once

#include <climits>

#include "elem_math.cuh"
#include "kernels.cuh"

namespace lulesh {

// Corner forces are written once and read once: with LULESH_CORNER_STREAM
// (the default) they use evict-first stores and loads, leaving L2 to the
// node and element arrays (nodal 67.6 -> 61.3 us at -s 100 on B200).
#ifndef LULESH_CORNER_STREAM
#define LULESH_CORNER_STREAM 1
#endif

__device__ __forceinline__ void st_corner(double *p, double v)
{
#if LULESH_CORNER_STREAM
    __stcs(p, v);
#else
    *p = v;
#endif
}

__device__ __forceinline__ double ld_corner(const double *p)
{
#if LULESH_CORNER_STREAM
    return __ldcs(p);
#else
    return *p;
#endif
}

// Velocities gathered into registers at kernel start, handed to the body
// where its arithmetic first needs them.
struct VelRegs {
    const double (&xd)[8];
    const double (&yd)[8];
    const double (&zd)[8];
    __device__ __forceinline__ void fetch(double (&x)[8], double (&y)[8], double (&z)[8]) const
    {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            x[i] = xd[i];
            y[i] = yd[i];
            z[i] = zd[i];
        }
    }
};

// The eight node indices of element el on the structured mesh, in the
// nodelist order of BuildMesh (lulesh.cu:730-737): corner j sits at lattice
// offset (x: bits 0x66, y: 0xCC, z: 0xF0 of j) from corner 0.
template <bool U = false>
__device__ __forceinline__ void elem_nodes(const DomDev &D, int el, int n[8])
{
    if (U) {  // an unstructured mesh's own nodelist (stride padded_numElem)
#pragma unroll
        for (int k = 0; k < 8; ++k) n[k] = D.nodelist[(size_t)k * D.Ep + el];
        return;
    }
    const int nx = D.nx, en = D.en;
    const int ix = el % nx;
    const int t = el / nx;
    const int iy = t % nx;
    const int iz = t / nx;
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

// CalcVolumeForceForElems_kernel (lulesh.cu:2080-2259) after the node
// gathers: stress + FB hourglass corner forces of element `elem`, handed
// to store(k, fx, fy, fz) corner by corner.  The velocities are fetched
// from `vel` only when HG (hourglass coefficient > 0).
template <bool HG, class Vel, class Store>
__device__ __forceinline__ void force_elem_to(const DomDev &D, TimeCtl &T, const Params &P,
                                              int elem, const double (&xn)[8],
                                              const double (&yn)[8], const double (&zn)[8],
                                              const Vel &vel, const Store &store)
{
    double dvdxn[8], dvdyn[8], dvdzn[8];
    double hgfx[8], hgfy[8], hgfz[8];
    double hourgam[8][4];

    const double volume = D.v[elem];
    double det = D.volo[elem] * volume;
    if (volume < 0.) atomicMin(&T.bad_vol, elem);
    const double ss1 = D.ss[elem];
    const double mass1 = D.elemMass[elem];
    const double sigxx = -D.p[elem] - D.q[elem];
    const double volinv = 1.0 / det;

    const double hourg = P.hgcoef;
    const double volume13 = cbrt(det);
    const double coefficient = -hourg * 0.01 * ss1 * mass1 / volume13;

    elem_volume_derivative(dvdxn, dvdyn, dvdzn, xn, yn, zn);
    hourglass_modes(xn, yn, zn, dvdxn, dvdyn, dvdzn, hourgam, volinv);

    double B[3][8];
    shape_function_derivatives(xn, yn, zn, B, &det);
    elem_node_normals(B[0], B[1], B[2], xn, yn, zn);
    if (det < 0.) atomicMin(&T.bad_vol, elem);

#pragma unroll
    for (int i = 0; i < 8; ++i) {
        hgfx[i] = -(sigxx * B[0][i]);
        hgfy[i] = -(sigxx * B[1][i]);
        hgfz[i] = -(sigxx * B[2][i]);
    }
    if (HG) {
        double xdn[8], ydn[8], zdn[8];
        vel.fetch(xdn, ydn, zdn);
        fb_hourglass_component(xdn, hourgam, coefficient, hgfx);
        fb_hourglass_component(ydn, hourgam, coefficient, hgfy);
        fb_hourglass_component(zdn, hourgam, coefficient, hgfz);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) store(k, hgfx[k], hgfy[k], hgfz[k]);
}

// the corner arrays at elem + Ep * corner
struct CornerStore {
    const DomDev &D;
    int elem;
    __device__ __forceinline__ void operator()(int k, double fx, double fy, double fz) const
    {
        const int c = elem + D.Ep * k;
        st_corner(D.fx_elem + c, fx);
        st_corner(D.fy_elem + c, fy);
        st_corner(D.fz_elem + c, fz);
    }
};

template <bool HG, class Vel>
__device__ __forceinline__ void force_elem(const DomDev &D, TimeCtl &T, const Params &P, int elem,
                                           const double (&xn)[8], const double (&yn)[8],
                                           const double (&zn)[8], const Vel &vel)
{
    force_elem_to<HG>(D, T, P, elem, xn, yn, zn, vel, CornerStore{D, elem});
}

// CalcKinematicsAndMonotonicQGradient_kernel (lulesh.cu:3343-3507) after
// the node gathers, for element k.
template <class Vel>
__device__ __forceinline__ void kin_elem(const DomDev &D, TimeCtl &T, int k, double (&x_local)[8],
                                         double (&y_local)[8], double (&z_local)[8],
                                         const Vel &vel)
{
    double B[3][8];
    double Dv[3];
    const double volume = elem_volume(x_local, y_local, z_local);
    const double relativeVolume = volume / D.volo[k];
    D.vnew[k] = relativeVolume;
    D.delv[k] = relativeVolume - D.v[k];
    D.arealg[k] = elem_characteristic_length(x_local, y_local, z_local, volume);

    double xd_local[8], yd_local[8], zd_local[8];
    vel.fetch(xd_local, yd_local, zd_local);
    const double dt2 = 0.5 * T.deltatime;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        x_local[j] -= dt2 * xd_local[j];
        y_local[j] -= dt2 * yd_local[j];
        z_local[j] -= dt2 * zd_local[j];
    }
    double detJ;
    shape_function_derivatives(x_local, y_local, z_local, B, &detJ);
    elem_velocity_divergence(xd_local, yd_local, zd_local, B, detJ, Dv);
    const double vdovNew = Dv[0] + Dv[1] + Dv[2];
    D.vdov[k] = vdovNew;

    const double vol = D.volo[k] * relativeVolume;
    // undo the half-step shift exactly as the reference does (the restored
    // coordinates can differ from the originals in the last bit)
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        x_local[j] += dt2 * xd_local[j];
        y_local[j] += dt2 * yd_local[j];
        z_local[j] += dt2 * zd_local[j];
    }
    double dxz, dvz, dxx, dvx, dxe, dve;
    mono_gradient(x_local, y_local, z_local, xd_local, yd_local, zd_local, vol, &dxz, &dvz,
                  &dxx, &dvx, &dxe, &dve);
    D.delx_zeta[k] = dxz;
    D.delv_zeta[k] = dvz;
    D.delx_xi[k] = dxx;
    D.delv_xi[k] = dvx;
    D.delx_eta[k] = dxe;
    D.delv_eta[k] = dve;
    if (relativeVolume < 0) atomicMin(&T.bad_vol, k);
}

}  // namespace lulesh
