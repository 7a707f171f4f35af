// elem_body.cuh -- per-element bodies of the FP64 force and kinematics
// kernels.  Each body receives the element's eight gathered node values and
// does the rest: element loads, arithmetic, stores.  The launch that
// gathers (kernels.cu) issues all 48 node loads before any arithmetic.
#pragma once

#include <climits>

#include "elem_math.cuh"
#include "kernels.cuh"

namespace lulesh {

// The eight node indices of element el on the structured mesh, in the
// nodelist order of BuildMesh (lulesh.cu:730-737): corner j sits at lattice
// offset (x: bits 0x66, y: 0xCC, z: 0xF0 of j) from corner 0.
__device__ __forceinline__ void elem_nodes(const DomDev &D, int el, int n[8])
{
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
// gathers: stress + FB hourglass corner forces of element `elem`, written
// to the corner arrays at elem + Ep * corner.  xdn..zdn are read only when
// HG (hourglass coefficient > 0).
template <bool HG>
__device__ __forceinline__ void force_elem(const DomDev &D, TimeCtl &T, const Params &P, int elem,
                                           const double (&xn)[8], const double (&yn)[8],
                                           const double (&zn)[8], const double (&xdn)[8],
                                           const double (&ydn)[8], const double (&zdn)[8])
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
        fb_hourglass_component(xdn, hourgam, coefficient, hgfx);
        fb_hourglass_component(ydn, hourgam, coefficient, hgfy);
        fb_hourglass_component(zdn, hourgam, coefficient, hgfz);
    }
    const int Ep = D.Ep;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        D.fx_elem[elem + Ep * k] = hgfx[k];
        D.fy_elem[elem + Ep * k] = hgfy[k];
        D.fz_elem[elem + Ep * k] = hgfz[k];
    }
}

// CalcKinematicsAndMonotonicQGradient_kernel (lulesh.cu:3343-3507) after
// the node gathers, for element k.
__device__ __forceinline__ void kin_elem(const DomDev &D, TimeCtl &T, int k, double (&x_local)[8],
                                         double (&y_local)[8], double (&z_local)[8],
                                         const double (&xd_local)[8], const double (&yd_local)[8],
                                         const double (&zd_local)[8])
{
    double B[3][8];
    double Dv[3];
    const double volume = elem_volume(x_local, y_local, z_local);
    const double relativeVolume = volume / D.volo[k];
    D.vnew[k] = relativeVolume;
    D.delv[k] = relativeVolume - D.v[k];
    D.arealg[k] = elem_characteristic_length(x_local, y_local, z_local, volume);

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
