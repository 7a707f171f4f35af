/*
 * lulesh_oracle.c -- CPU oracle for the LULESH Lagrange leapfrog step.
 *
 * TEST INFRASTRUCTURE ONLY (the checker).  Only tests/, __graft_entry__.smoke()
 * and bench.py's cpu_baseline leg may load it.  The product path never does.
 *
 * What it restates: the single-domain step of the reference CUDA build,
 * LULESH/cuda/src/lulesh.cu, kernel by kernel, keeping every floating-point
 * expression in the reference's association order so that, compiled without
 * FMA contraction (-ffp-contract=off), each operation rounds exactly as the
 * written C expression says.  The GPU build contracts multiply-adds into
 * FMAs, so GPU-vs-oracle agreement is to a stated tolerance, not bitwise.
 *
 * Pins (tests/test_oracle_pins.py): the reference omp_4.0 CPU build and the
 * reference CUDA build compiled into oracle/_ref/, the survey-measured omp
 * energies, and the reference's published energies.
 */
#include "lulesh_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* element-face boundary-condition bits, lulesh.cu:151-181 */
#define BC_XI_M 0x00007
#define BC_XI_M_SYMM 0x00001
#define BC_XI_M_FREE 0x00002
#define BC_XI_M_COMM 0x00004
#define BC_XI_P 0x00038
#define BC_XI_P_SYMM 0x00008
#define BC_XI_P_FREE 0x00010
#define BC_XI_P_COMM 0x00020
#define BC_ETA_M 0x001c0
#define BC_ETA_M_SYMM 0x00040
#define BC_ETA_M_FREE 0x00080
#define BC_ETA_M_COMM 0x00100
#define BC_ETA_P 0x00e00
#define BC_ETA_P_SYMM 0x00200
#define BC_ETA_P_FREE 0x00400
#define BC_ETA_P_COMM 0x00800
#define BC_ZETA_M 0x07000
#define BC_ZETA_M_SYMM 0x01000
#define BC_ZETA_M_FREE 0x02000
#define BC_ZETA_M_COMM 0x04000
#define BC_ZETA_P 0x38000
#define BC_ZETA_P_SYMM 0x08000
#define BC_ZETA_P_FREE 0x10000
#define BC_ZETA_P_COMM 0x20000

struct OracleDomain {
    int nx, numElem, numNode, Ep, tp, colLoc, rowLoc, planeLoc, rank;
    int rowMin, rowMax, colMin, colMax, planeMin, planeMax;
    int allElem;
    /* connectivity */
    int *nodelist, *lxim, *lxip, *letam, *letap, *lzetam, *lzetap, *elemBC;
    int *nodeElemCount, *nodeElemStart, *nodeElemCornerList, cornerListLen;
    int *symmX, *symmY, *symmZ, numSymmX, numSymmY, numSymmZ, symmLen;
    int *matElemlist;
    /* regions */
    int numReg, balance, cost;
    int *regElemSize, *regCSR, *regReps, *regNumList, *regElemlist, *regSorted;
    /* element fields */
    double *e, *p, *q, *ql, *qq, *v, *volo, *delv, *vdov, *arealg, *ss,
        *elemMass;
    /* node fields */
    double *x, *y, *z, *xd, *yd, *zd, *xdd, *ydd, *zdd, *fx, *fy, *fz,
        *nodalMass;
    /* per-cycle temporaries (lulesh.cu:2653-2655, 4151-4162) */
    double *vnew, *delx_xi, *delx_eta, *delx_zeta, *delv_xi, *delv_eta,
        *delv_zeta, *fx_elem, *fy_elem, *fz_elem;
    /* parameters, lulesh.cu:1125-1158 */
    double dtfixed, deltatimemultlb, deltatimemultub, stoptime, dtmax;
    double e_cut, p_cut, q_cut, u_cut, v_cut, hgcoef, ss4o3, qstop,
        monoq_max_slope, monoq_limiter_mult, qlc_monoq, qqc_monoq, qqc,
        pmin, emin, dvovmax, eosvmax, eosvmin, refdens;
    /* time state */
    double time, deltatime, dtcourant, dthydro, initial_deltatime;
    int cycle;
    int bad_vol, bad_q;
    /* element holding the energy deposit (0 on -s meshes) */
    int octantCorner;
    /* decomposed stepping: ghost-face offsets into delv_* (SetupConnectivityBC
     * order, INT_MIN for none) and the 26 neighbours' arrays, by direction
     * (dx+1) + 3(dy+1) + 9(dz+1) */
    int ghost[6];
    OracleMirror mirror[27];
    int has_mirror[27];
};

static void *zalloc(size_t n) { return calloc(n ? n : 1, 1); }
#define ZD(n) ((double *)zalloc(sizeof(double) * (size_t)(n)))
#define ZI(n) ((int *)zalloc(sizeof(int) * (size_t)(n)))

/* ------------------------------------------------------------------ */
/* element geometry helpers                                             */
/* ------------------------------------------------------------------ */

/* TRIPLE_PRODUCT of lulesh.cu:287-288 with its argument binding */
static double triple(double a1, double b1, double c1, double a2, double b2,
                     double c2, double a3, double b3, double c3)
{
    return a1 * (b2 * c3 - c2 * b3) + a2 * (c1 * b3 - b1 * c3) +
           a3 * (b1 * c2 - c1 * b2);
}

/* CalcElemVolume, lulesh.cu:221-307 */
static double elem_volume(const double *x, const double *y, const double *z)
{
    const double twelveth = 1.0 / 12.0;
    double dx61 = x[6] - x[1], dy61 = y[6] - y[1], dz61 = z[6] - z[1];
    double dx70 = x[7] - x[0], dy70 = y[7] - y[0], dz70 = z[7] - z[0];
    double dx63 = x[6] - x[3], dy63 = y[6] - y[3], dz63 = z[6] - z[3];
    double dx20 = x[2] - x[0], dy20 = y[2] - y[0], dz20 = z[2] - z[0];
    double dx50 = x[5] - x[0], dy50 = y[5] - y[0], dz50 = z[5] - z[0];
    double dx64 = x[6] - x[4], dy64 = y[6] - y[4], dz64 = z[6] - z[4];
    double dx31 = x[3] - x[1], dy31 = y[3] - y[1], dz31 = z[3] - z[1];
    double dx72 = x[7] - x[2], dy72 = y[7] - y[2], dz72 = z[7] - z[2];
    double dx43 = x[4] - x[3], dy43 = y[4] - y[3], dz43 = z[4] - z[3];
    double dx57 = x[5] - x[7], dy57 = y[5] - y[7], dz57 = z[5] - z[7];
    double dx14 = x[1] - x[4], dy14 = y[1] - y[4], dz14 = z[1] - z[4];
    double dx25 = x[2] - x[5], dy25 = y[2] - y[5], dz25 = z[2] - z[5];
    double vol = triple(dx31 + dx72, dx63, dx20, dy31 + dy72, dy63, dy20,
                        dz31 + dz72, dz63, dz20) +
                 triple(dx43 + dx57, dx64, dx70, dy43 + dy57, dy64, dy70,
                        dz43 + dz57, dz64, dz70) +
                 triple(dx14 + dx25, dx61, dx50, dy14 + dy25, dy61, dy50,
                        dz14 + dz25, dz61, dz50);
    vol *= twelveth;
    return vol;
}

/* CalcElemShapeFunctionDerivatives, lulesh.cu:1466-1561 */
static void shape_derivs(const double *x, const double *y, const double *z,
                         double b[3][8], double *volume)
{
    double fj[3][3]; /* [coord][xi,eta,zeta] */
    const double *c[3] = {x, y, z};
    for (int k = 0; k < 3; ++k) {
        const double *a = c[k];
        double d60 = a[6] - a[0], d53 = a[5] - a[3], d71 = a[7] - a[1],
               d42 = a[4] - a[2];
        fj[k][0] = .125 * (d60 + d53 - d71 - d42);
        fj[k][1] = .125 * (d60 - d53 + d71 - d42);
        fj[k][2] = .125 * (d60 + d53 + d71 + d42);
    }
    double fjxxi = fj[0][0], fjxet = fj[0][1], fjxze = fj[0][2];
    double fjyxi = fj[1][0], fjyet = fj[1][1], fjyze = fj[1][2];
    double fjzxi = fj[2][0], fjzet = fj[2][1], fjzze = fj[2][2];
    double cj[3][3];
    cj[0][0] = (fjyet * fjzze) - (fjzet * fjyze);
    cj[0][1] = -(fjyxi * fjzze) + (fjzxi * fjyze);
    cj[0][2] = (fjyxi * fjzet) - (fjzxi * fjyet);
    cj[1][0] = -(fjxet * fjzze) + (fjzet * fjxze);
    cj[1][1] = (fjxxi * fjzze) - (fjzxi * fjxze);
    cj[1][2] = -(fjxxi * fjzet) + (fjzxi * fjxet);
    cj[2][0] = (fjxet * fjyze) - (fjyet * fjxze);
    cj[2][1] = -(fjxxi * fjyze) + (fjyxi * fjxze);
    cj[2][2] = (fjxxi * fjyet) - (fjyxi * fjxet);
    for (int k = 0; k < 3; ++k) {
        double cxi = cj[k][0], cet = cj[k][1], cze = cj[k][2];
        b[k][0] = -cxi - cet - cze;
        b[k][1] = cxi - cet - cze;
        b[k][2] = cxi + cet - cze;
        b[k][3] = -cxi + cet - cze;
        b[k][4] = -b[k][2];
        b[k][5] = -b[k][3];
        b[k][6] = -b[k][0];
        b[k][7] = -b[k][1];
    }
    *volume = 8. * (fjxet * cj[0][1] + fjyet * cj[1][1] + fjzet * cj[2][1]);
}

/* SumElemFaceNormal, lulesh.cu:1566-1599: adds the face area vector of
 * corners (n0,n1,n2,n3) to each of the four corners */
static void face_normal(double *pfx, double *pfy, double *pfz, const double *x,
                        const double *y, const double *z, int n0, int n1,
                        int n2, int n3)
{
    double bx0 = 0.5 * (x[n3] + x[n2] - x[n1] - x[n0]);
    double by0 = 0.5 * (y[n3] + y[n2] - y[n1] - y[n0]);
    double bz0 = 0.5 * (z[n3] + z[n2] - z[n1] - z[n0]);
    double bx1 = 0.5 * (x[n2] + x[n1] - x[n3] - x[n0]);
    double by1 = 0.5 * (y[n2] + y[n1] - y[n3] - y[n0]);
    double bz1 = 0.5 * (z[n2] + z[n1] - z[n3] - z[n0]);
    double ax = 0.25 * (by0 * bz1 - bz0 * by1);
    double ay = 0.25 * (bz0 * bx1 - bx0 * bz1);
    double az = 0.25 * (bx0 * by1 - by0 * bx1);
    int n[4] = {n0, n1, n2, n3};
    for (int k = 0; k < 4; ++k) {
        pfx[n[k]] += ax;
        pfy[n[k]] += ay;
        pfz[n[k]] += az;
    }
}

/* CalcElemNodeNormals, lulesh.cu:1657-1711: six faces in this order */
static const int kFaces[6][4] = {{0, 1, 2, 3}, {0, 4, 5, 1}, {1, 5, 6, 2},
                                 {2, 6, 7, 3}, {3, 7, 4, 0}, {4, 7, 6, 5}};

static void node_normals(double *pfx, double *pfy, double *pfz,
                         const double *x, const double *y, const double *z)
{
    for (int i = 0; i < 8; ++i) pfx[i] = pfy[i] = pfz[i] = 0.0;
    for (int f = 0; f < 6; ++f)
        face_normal(pfx, pfy, pfz, x, y, z, kFaces[f][0], kFaces[f][1],
                    kFaces[f][2], kFaces[f][3]);
}

/* VoluDer, lulesh.cu:1756-1784 (arguments are the six node coordinates of
 * the call site in the order it passes them) */
static void volu_der(const double *x, const double *y, const double *z,
                     const int *m, double *dvdx, double *dvdy, double *dvdz)
{
    const double twelfth = 1.0 / 12.0;
    double x0 = x[m[0]], x1 = x[m[1]], x2 = x[m[2]], x3 = x[m[3]],
           x4 = x[m[4]], x5 = x[m[5]];
    double y0 = y[m[0]], y1 = y[m[1]], y2 = y[m[2]], y3 = y[m[3]],
           y4 = y[m[4]], y5 = y[m[5]];
    double z0 = z[m[0]], z1 = z[m[1]], z2 = z[m[2]], z3 = z[m[3]],
           z4 = z[m[4]], z5 = z[m[5]];
    *dvdx = (y1 + y2) * (z0 + z1) - (y0 + y1) * (z1 + z2) +
            (y0 + y4) * (z3 + z4) - (y3 + y4) * (z0 + z4) -
            (y2 + y5) * (z3 + z5) + (y3 + y5) * (z2 + z5);
    *dvdy = -(x1 + x2) * (z0 + z1) + (x0 + x1) * (z1 + z2) -
            (x0 + x4) * (z3 + z4) + (x3 + x4) * (z0 + z4) +
            (x2 + x5) * (z3 + z5) - (x3 + x5) * (z2 + z5);
    *dvdz = -(y1 + y2) * (x0 + x1) + (y0 + y1) * (x1 + x2) -
            (y0 + y4) * (x3 + x4) + (y3 + y4) * (x0 + x4) +
            (y2 + y5) * (x3 + x5) - (y3 + y5) * (x2 + x5);
    *dvdx *= twelfth;
    *dvdy *= twelfth;
    *dvdz *= twelfth;
}

/* CalcElemVolumeDerivative, lulesh.cu:1789-1828: node permutation per
 * output corner, in the reference's call order */
static const int kVoluDer[8][7] = {
    /* out, six nodes */
    {0, 1, 2, 3, 4, 5, 7}, {3, 0, 1, 2, 7, 4, 6}, {2, 3, 0, 1, 6, 7, 5},
    {1, 2, 3, 0, 5, 6, 4}, {4, 7, 6, 5, 0, 3, 1}, {5, 4, 7, 6, 1, 0, 2},
    {6, 5, 4, 7, 2, 1, 3}, {7, 6, 5, 4, 3, 2, 0}};

static void volume_derivative(double *dvdx, double *dvdy, double *dvdz,
                              const double *x, const double *y,
                              const double *z)
{
    for (int k = 0; k < 8; ++k) {
        int o = kVoluDer[k][0];
        volu_der(x, y, z, &kVoluDer[k][1], &dvdx[o], &dvdy[o], &dvdz[o]);
    }
}

/* Hourglass base vectors (sign patterns), lulesh.cu:2023-2069 */
static const double kGamma[4][8] = {{1, 1, -1, -1, -1, -1, 1, 1},
                                    {1, -1, -1, 1, -1, 1, 1, -1},
                                    {1, -1, 1, -1, 1, -1, 1, -1},
                                    {-1, 1, -1, 1, 1, -1, 1, -1}};

/* sum_k gamma[m][k] * a[k], accumulated left to right; multiplying by +-1
 * is exact, so this equals the reference's written +/- chain */
static double gsum(int m, const double *a)
{
    double s = kGamma[m][0] * a[0];
    for (int k = 1; k < 8; ++k) s = s + kGamma[m][k] * a[k];
    return s;
}

/* CalcHourglassModes, lulesh.cu:2017-2071 */
static void hourglass_modes(const double *xn, const double *yn,
                            const double *zn, const double *dvdx,
                            const double *dvdy, const double *dvdz,
                            double hg[8][4], double volinv)
{
    for (int m = 0; m < 4; ++m) {
        double hx = gsum(m, xn), hy = gsum(m, yn), hz = gsum(m, zn);
        for (int k = 0; k < 8; ++k)
            hg[k][m] = kGamma[m][k] -
                       volinv * (dvdx[k] * hx + dvdy[k] * hy + dvdz[k] * hz);
    }
}

/* CalcElemFBHourglassForce, lulesh.cu:1833-2013, one velocity component */
static void fb_hourglass(const double *vel, double hg[8][4], double coef,
                         double *hgf)
{
    double h[4];
    for (int m = 0; m < 4; ++m) {
        double s = hg[0][m] * vel[0] + hg[1][m] * vel[1];
        for (int k = 2; k < 8; ++k) s = s + hg[k][m] * vel[k];
        h[m] = s;
    }
    for (int k = 0; k < 8; ++k)
        hgf[k] += coef * (hg[k][0] * h[0] + hg[k][1] * h[1] +
                          hg[k][2] * h[2] + hg[k][3] * h[3]);
}

/* AreaFace, lulesh.cu:3103-3122 */
static double area_face(const double *x, const double *y, const double *z,
                        int a, int b, int c, int d)
{
    double fx = (x[c] - x[a]) - (x[d] - x[b]);
    double fy = (y[c] - y[a]) - (y[d] - y[b]);
    double fz = (z[c] - z[a]) - (z[d] - z[b]);
    double gx = (x[c] - x[a]) + (x[d] - x[b]);
    double gy = (y[c] - y[a]) + (y[d] - y[b]);
    double gz = (z[c] - z[a]) + (z[d] - z[b]);
    double t = (fx * gx + fy * gy + fz * gz);
    return (fx * fx + fy * fy + fz * fz) * (gx * gx + gy * gy + gz * gz) -
           t * t;
}

/* CalcElemCharacteristicLength, lulesh.cu:3126-3166 */
static const int kLenFaces[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 1, 5, 4},
                                    {1, 2, 6, 5}, {2, 3, 7, 6}, {3, 0, 4, 7}};

static double char_length(const double *x, const double *y, const double *z,
                          double volume)
{
    double cl = 0.0;
    for (int f = 0; f < 6; ++f) {
        double a = area_face(x, y, z, kLenFaces[f][0], kLenFaces[f][1],
                             kLenFaces[f][2], kLenFaces[f][3]);
        cl = fmax(a, cl);
    }
    return 4.0 * volume / sqrt(cl);
}

/* CalcElemVelocityGradient, lulesh.cu:3171-3248 */
static void velocity_gradient(const double *xv, const double *yv,
                              const double *zv, double b[3][8], double detJ,
                              double *d)
{
    const double inv = 1.0 / detJ;
    const double *v[3] = {xv, yv, zv};
    double g[3][3]; /* g[c][k]: d(vel_c)/d(x_k) */
    for (int c = 0; c < 3; ++c) {
        double t1 = v[c][0] - v[c][6], t2 = v[c][1] - v[c][7],
               t3 = v[c][2] - v[c][4], t4 = v[c][3] - v[c][5];
        for (int k = 0; k < 3; ++k)
            g[c][k] = inv * (b[k][0] * t1 + b[k][1] * t2 + b[k][2] * t3 +
                             b[k][3] * t4);
    }
    d[0] = g[0][0];
    d[1] = g[1][1];
    d[2] = g[2][2];
    d[5] = .5 * (g[0][1] + g[1][0]);
    d[4] = .5 * (g[0][2] + g[2][0]);
    d[3] = .5 * (g[2][1] + g[1][2]);
}

/* CalcMonoGradient, lulesh.cu:3251-3334 */
static double sum4(const double *a, int i, int j, int k, int l)
{
    return a[i] + a[j] + a[k] + a[l];
}

static void mono_gradient(const double *x, const double *y, const double *z,
                          const double *xv, const double *yv, const double *zv,
                          double vol, double *dx_zeta, double *dv_zeta,
                          double *dx_xi, double *dv_xi, double *dx_eta,
                          double *dv_eta)
{
    const double ptiny = 1.e-36;
    double norm = 1.0 / (vol + ptiny);
    double dxj = -0.25 * (sum4(x, 0, 1, 5, 4) - sum4(x, 3, 2, 6, 7));
    double dyj = -0.25 * (sum4(y, 0, 1, 5, 4) - sum4(y, 3, 2, 6, 7));
    double dzj = -0.25 * (sum4(z, 0, 1, 5, 4) - sum4(z, 3, 2, 6, 7));
    double dxi = 0.25 * (sum4(x, 1, 2, 6, 5) - sum4(x, 0, 3, 7, 4));
    double dyi = 0.25 * (sum4(y, 1, 2, 6, 5) - sum4(y, 0, 3, 7, 4));
    double dzi = 0.25 * (sum4(z, 1, 2, 6, 5) - sum4(z, 0, 3, 7, 4));
    double dxk = 0.25 * (sum4(x, 4, 5, 6, 7) - sum4(x, 0, 1, 2, 3));
    double dyk = 0.25 * (sum4(y, 4, 5, 6, 7) - sum4(y, 0, 1, 2, 3));
    double dzk = 0.25 * (sum4(z, 4, 5, 6, 7) - sum4(z, 0, 1, 2, 3));
    double ax, ay, az, dxv, dyv, dzv;

    ax = dyi * dzj - dzi * dyj;
    ay = dzi * dxj - dxi * dzj;
    az = dxi * dyj - dyi * dxj;
    *dx_zeta = vol / sqrt(ax * ax + ay * ay + az * az + ptiny);
    ax *= norm;
    ay *= norm;
    az *= norm;
    dxv = 0.25 * (sum4(xv, 4, 5, 6, 7) - sum4(xv, 0, 1, 2, 3));
    dyv = 0.25 * (sum4(yv, 4, 5, 6, 7) - sum4(yv, 0, 1, 2, 3));
    dzv = 0.25 * (sum4(zv, 4, 5, 6, 7) - sum4(zv, 0, 1, 2, 3));
    *dv_zeta = ax * dxv + ay * dyv + az * dzv;

    ax = dyj * dzk - dzj * dyk;
    ay = dzj * dxk - dxj * dzk;
    az = dxj * dyk - dyj * dxk;
    *dx_xi = vol / sqrt(ax * ax + ay * ay + az * az + ptiny);
    ax *= norm;
    ay *= norm;
    az *= norm;
    dxv = 0.25 * (sum4(xv, 1, 2, 6, 5) - sum4(xv, 0, 3, 7, 4));
    dyv = 0.25 * (sum4(yv, 1, 2, 6, 5) - sum4(yv, 0, 3, 7, 4));
    dzv = 0.25 * (sum4(zv, 1, 2, 6, 5) - sum4(zv, 0, 3, 7, 4));
    *dv_xi = ax * dxv + ay * dyv + az * dzv;

    ax = dyk * dzi - dzk * dyi;
    ay = dzk * dxi - dxk * dzi;
    az = dxk * dyi - dyk * dxi;
    *dx_eta = vol / sqrt(ax * ax + ay * ay + az * az + ptiny);
    ax *= norm;
    ay *= norm;
    az *= norm;
    dxv = -0.25 * (sum4(xv, 0, 1, 5, 4) - sum4(xv, 3, 2, 6, 7));
    dyv = -0.25 * (sum4(yv, 0, 1, 5, 4) - sum4(yv, 3, 2, 6, 7));
    dzv = -0.25 * (sum4(zv, 0, 1, 5, 4) - sum4(zv, 3, 2, 6, 7));
    *dv_eta = ax * dxv + ay * dyv + az * dzv;
}

/* ------------------------------------------------------------------ */
/* setup                                                                */
/* ------------------------------------------------------------------ */

/* Domain::sortRegions, lulesh.cu:1224-1250: bubble sort by reps,
 * descending, carrying sizes and original indices */
static void sort_regions(OracleDomain *d)
{
    int n = d->numReg;
    int *idx = ZI(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    for (int i = 0; i < n - 1; ++i)
        for (int j = 0; j < n - i - 1; ++j)
            if (d->regReps[j] < d->regReps[j + 1]) {
                int t = d->regReps[j];
                d->regReps[j] = d->regReps[j + 1];
                d->regReps[j + 1] = t;
                t = d->regElemSize[j];
                d->regElemSize[j] = d->regElemSize[j + 1];
                d->regElemSize[j + 1] = t;
                t = idx[j];
                idx[j] = idx[j + 1];
                idx[j + 1] = t;
            }
    for (int i = 0; i < n; ++i) d->regSorted[idx[i]] = i;
    free(idx);
}

static int ipow(int b, int e)
{
    int r = 1;
    for (int i = 0; i < e; ++i) r *= b;
    return r;
}

/* Domain::CreateRegionIndexSets, lulesh.cu:1261-1398 (libc rand) */
static void create_regions(OracleDomain *d, int nr, int balance)
{
    int myRank = d->rank;
    srand((unsigned)myRank);
    d->numReg = nr;
    d->balance = balance;
    int E = d->numElem;
    d->regElemSize = ZI(nr);
    d->regCSR = ZI(nr);
    d->regReps = ZI(nr);
    d->regSorted = ZI(nr);
    d->regNumList = ZI(E);
    d->regElemlist = ZI(E);
    int next = 0;
    if (nr == 1) {
        while (next < E) d->regNumList[next++] = 1;
    } else {
        int lastReg = -1, costDen = 0;
        int *binEnd = ZI(nr);
        for (int i = 0; i < nr; ++i) {
            costDen += ipow(i + 1, balance);
            binEnd[i] = costDen;
        }
        while (next < E) {
            int rv = rand() % costDen, i = 0, regionNum, elements;
            while (rv >= binEnd[i]) i++;
            regionNum = ((i + myRank) % nr) + 1;
            while (regionNum == lastReg) {
                rv = rand() % costDen;
                i = 0;
                while (rv >= binEnd[i]) i++;
                regionNum = ((i + myRank) % nr) + 1;
            }
            int bin = rand() % 1000;
            if (bin < 773)
                elements = rand() % 15 + 1;
            else if (bin < 937)
                elements = rand() % 16 + 16;
            else if (bin < 970)
                elements = rand() % 32 + 32;
            else if (bin < 974)
                elements = rand() % 64 + 64;
            else if (bin < 978)
                elements = rand() % 128 + 128;
            else if (bin < 981)
                elements = rand() % 256 + 256;
            else
                elements = rand() % 1537 + 512;
            int runto = elements + next;
            while (next < runto && next < E) d->regNumList[next++] = regionNum;
            lastReg = regionNum;
        }
        free(binEnd);
    }
    for (int i = 0; i < E; ++i) d->regElemSize[d->regNumList[i] - 1]++;
    for (int r = 0; r < nr; ++r) {
        int rep;
        if (r < nr / 2)
            rep = 1;
        else if (r < (nr - (nr + 15) / 20))
            rep = 1 + d->cost;
        else
            rep = 10 * (1 + d->cost);
        d->regReps[r] = rep;
    }
    sort_regions(d);
    d->regCSR[0] = 0;
    for (int i = 1; i < nr; ++i)
        d->regCSR[i] = d->regCSR[i - 1] + d->regElemSize[i - 1];
    for (int i = 0; i < E; ++i) {
        int r = d->regSorted[d->regNumList[i] - 1];
        d->regElemlist[d->regCSR[r]] = i;
        d->regCSR[r]++;
    }
}

/* node -> corner CSR, lulesh.cu:1054-1106 (outer j, inner element) */
static void corner_csr(OracleDomain *d)
{
    const int E = d->numElem, N = d->numNode, Ep = d->Ep;
    d->nodeElemCount = ZI(N);
    d->nodeElemStart = ZI(N);
    for (int i = 0; i < E; ++i)
        for (int j = 0; j < 8; ++j) d->nodeElemCount[d->nodelist[j * Ep + i]]++;
    d->nodeElemStart[0] = 0;
    for (int i = 1; i < N; ++i)
        d->nodeElemStart[i] = d->nodeElemStart[i - 1] + d->nodeElemCount[i - 1];
    d->cornerListLen = d->nodeElemStart[N - 1] + d->nodeElemCount[N - 1];
    d->nodeElemCornerList = ZI(d->cornerListLen);
    for (int i = 0; i < N; ++i) d->nodeElemCount[i] = 0;
    for (int j = 0; j < 8; ++j)
        for (int i = 0; i < E; ++i) {
            int m = d->nodelist[Ep * j + i];
            int off = d->nodeElemStart[m] + d->nodeElemCount[m];
            d->nodeElemCornerList[off] = Ep * j + i;
            d->nodeElemCount[m]++;
        }
    d->matElemlist = ZI(E);
    for (int i = 0; i < E; ++i) d->matElemlist[i] = i;
}

static void set_params(OracleDomain *d);
static void masses(OracleDomain *d);

OracleDomain *oracle_create(int nx, int numReg, int balance, int cost,
                            int tp, int col, int row, int plane, int rank)
{
    if (nx < 1 || numReg < 1 || tp < 1) return NULL;
    OracleDomain *d = (OracleDomain *)zalloc(sizeof(OracleDomain));
    int en = nx + 1;
    d->nx = nx;
    d->tp = tp;
    d->colLoc = col;
    d->rowLoc = row;
    d->planeLoc = plane;
    d->rank = rank;
    d->cost = cost;
    d->numElem = nx * nx * nx;
    d->Ep = ((d->numElem + 31) / 32) * 32;
    d->numNode = en * en * en;
    int E = d->numElem, N = d->numNode, Ep = d->Ep;

    /* SetupCommBuffers neighbour flags, lulesh.cu:463-468 */
    d->rowMin = (row == 0) ? 0 : 1;
    d->rowMax = (row == tp - 1) ? 0 : 1;
    d->colMin = (col == 0) ? 0 : 1;
    d->colMax = (col == tp - 1) ? 0 : 1;
    d->planeMin = (plane == 0) ? 0 : 1;
    d->planeMax = (plane == tp - 1) ? 0 : 1;
    d->allElem = E + 2 * nx * nx * 3;

    d->e = ZD(E); d->p = ZD(E); d->q = ZD(E); d->ql = ZD(E); d->qq = ZD(E);
    d->v = ZD(E); d->volo = ZD(E); d->delv = ZD(E); d->vdov = ZD(E);
    d->arealg = ZD(E); d->ss = ZD(E); d->elemMass = ZD(E);
    d->x = ZD(N); d->y = ZD(N); d->z = ZD(N);
    d->xd = ZD(N); d->yd = ZD(N); d->zd = ZD(N);
    d->xdd = ZD(N); d->ydd = ZD(N); d->zdd = ZD(N);
    d->fx = ZD(N); d->fy = ZD(N); d->fz = ZD(N); d->nodalMass = ZD(N);
    d->vnew = ZD(E);
    d->delx_xi = ZD(E); d->delx_eta = ZD(E); d->delx_zeta = ZD(E);
    d->delv_xi = ZD(d->allElem); d->delv_eta = ZD(d->allElem);
    d->delv_zeta = ZD(d->allElem);
    d->fx_elem = ZD(8 * Ep); d->fy_elem = ZD(8 * Ep); d->fz_elem = ZD(8 * Ep);
    /* InitializeFields, lulesh.cu:432-451: only v is non-zero */
    for (int i = 0; i < E; ++i) d->v[i] = 1.0;

    /* BuildMesh, lulesh.cu:688-747 */
    int meshEdge = tp * nx, nidx = 0;
    for (int pl = 0; pl < en; ++pl) {
        double tz = 1.125 * (double)(plane * nx + pl) / (double)meshEdge;
        for (int r = 0; r < en; ++r) {
            double ty = 1.125 * (double)(row * nx + r) / (double)meshEdge;
            for (int c = 0; c < en; ++c) {
                double tx = 1.125 * (double)(col * nx + c) / (double)meshEdge;
                d->x[nidx] = tx;
                d->y[nidx] = ty;
                d->z[nidx] = tz;
                ++nidx;
            }
        }
    }
    d->nodelist = ZI(8 * Ep);
    {
        int zidx = 0;
        nidx = 0;
        for (int pl = 0; pl < nx; ++pl) {
            for (int r = 0; r < nx; ++r) {
                for (int c = 0; c < nx; ++c) {
                    int *nl = d->nodelist;
                    nl[0 * Ep + zidx] = nidx;
                    nl[1 * Ep + zidx] = nidx + 1;
                    nl[2 * Ep + zidx] = nidx + en + 1;
                    nl[3 * Ep + zidx] = nidx + en;
                    nl[4 * Ep + zidx] = nidx + en * en;
                    nl[5 * Ep + zidx] = nidx + en * en + 1;
                    nl[6 * Ep + zidx] = nidx + en * en + en + 1;
                    nl[7 * Ep + zidx] = nidx + en * en + en;
                    ++zidx;
                    ++nidx;
                }
                ++nidx;
            }
            nidx += en;
        }
    }

    /* symmetry node sets, lulesh.cu:809-851 */
    d->symmLen = en * en;
    d->symmX = ZI(en * en);
    d->symmY = ZI(en * en);
    d->symmZ = ZI(en * en);
    d->numSymmX = (col == 0) ? en * en : 0;
    d->numSymmY = (row == 0) ? en * en : 0;
    d->numSymmZ = (plane == 0) ? en * en : 0;
    nidx = 0;
    for (int i = 0; i < en; ++i) {
        int planeInc = i * en * en, rowInc = i * en;
        for (int j = 0; j < en; ++j) {
            if (plane == 0) d->symmZ[nidx] = rowInc + j;
            if (row == 0) d->symmY[nidx] = planeInc + j;
            if (col == 0) d->symmX[nidx] = planeInc + j * en;
            ++nidx;
        }
    }

    /* SetupConnectivityBC, lulesh.cu:537-686 */
    d->lxim = ZI(E); d->lxip = ZI(E); d->letam = ZI(E); d->letap = ZI(E);
    d->lzetam = ZI(E); d->lzetap = ZI(E); d->elemBC = ZI(E);
    d->lxim[0] = 0;
    for (int i = 1; i < E; ++i) {
        d->lxim[i] = i - 1;
        d->lxip[i - 1] = i;
    }
    d->lxip[E - 1] = E - 1;
    for (int i = 0; i < nx; ++i) {
        d->letam[i] = i;
        d->letap[E - nx + i] = E - nx + i;
    }
    for (int i = nx; i < E; ++i) {
        d->letam[i] = i - nx;
        d->letap[i - nx] = i;
    }
    for (int i = 0; i < nx * nx; ++i) {
        d->lzetam[i] = i;
        d->lzetap[E - nx * nx + i] = E - nx * nx + i;
    }
    for (int i = nx * nx; i < E; ++i) {
        d->lzetam[i] = i - nx * nx;
        d->lzetap[i - nx * nx] = i;
    }
    int ghost[6];
    for (int i = 0; i < 6; ++i) ghost[i] = INT_MIN;
    int pidx = E;
    if (d->planeMin) { ghost[0] = pidx; pidx += nx * nx; }
    if (d->planeMax) { ghost[1] = pidx; pidx += nx * nx; }
    if (d->rowMin) { ghost[2] = pidx; pidx += nx * nx; }
    if (d->rowMax) { ghost[3] = pidx; pidx += nx * nx; }
    if (d->colMin) { ghost[4] = pidx; pidx += nx * nx; }
    if (d->colMax) { ghost[5] = pidx; }
    for (int i = 0; i < 6; ++i) d->ghost[i] = ghost[i];
    for (int i = 0; i < nx; ++i) {
        int planeInc = i * nx * nx, rowInc = i * nx;
        for (int j = 0; j < nx; ++j) {
            if (plane == 0) {
                d->elemBC[rowInc + j] |= BC_ZETA_M_SYMM;
            } else {
                d->elemBC[rowInc + j] |= BC_ZETA_M_COMM;
                d->lzetam[rowInc + j] = ghost[0] + rowInc + j;
            }
            if (plane == tp - 1) {
                d->elemBC[rowInc + j + E - nx * nx] |= BC_ZETA_P_FREE;
            } else {
                d->elemBC[rowInc + j + E - nx * nx] |= BC_ZETA_P_COMM;
                d->lzetap[rowInc + j + E - nx * nx] = ghost[1] + rowInc + j;
            }
            if (row == 0) {
                d->elemBC[planeInc + j] |= BC_ETA_M_SYMM;
            } else {
                d->elemBC[planeInc + j] |= BC_ETA_M_COMM;
                d->letam[planeInc + j] = ghost[2] + rowInc + j;
            }
            if (row == tp - 1) {
                d->elemBC[planeInc + j + nx * nx - nx] |= BC_ETA_P_FREE;
            } else {
                d->elemBC[planeInc + j + nx * nx - nx] |= BC_ETA_P_COMM;
                d->letap[planeInc + j + nx * nx - nx] = ghost[3] + rowInc + j;
            }
            if (col == 0) {
                d->elemBC[planeInc + j * nx] |= BC_XI_M_SYMM;
            } else {
                d->elemBC[planeInc + j * nx] |= BC_XI_M_COMM;
                d->lxim[planeInc + j * nx] = ghost[4] + rowInc + j;
            }
            if (col == tp - 1) {
                d->elemBC[planeInc + j * nx + nx - 1] |= BC_XI_P_FREE;
            } else {
                d->elemBC[planeInc + j * nx + nx - 1] |= BC_XI_P_COMM;
                d->lxip[planeInc + j * nx + nx - 1] = ghost[5] + rowInc + j;
            }
        }
    }

    corner_csr(d);
    set_params(d);
    /* volo, elemMass, nodalMass, lulesh.cu:1165-1187 */
    masses(d);

    /* energy deposit and initial dt, lulesh.cu:1189-1205 */
    const double ebase = 3.948746e+7;
    double scale = (nx * tp) / 45.0;
    double einit = ebase * scale * scale * scale;
    if (row + col + plane == 0) d->e[0] = einit;
    d->deltatime = (.5 * cbrt(d->volo[0])) / sqrt(2 * einit);
    d->initial_deltatime = d->deltatime;

    create_regions(d, numReg, balance);
    return d;
}

/* parameters, lulesh.cu:1120-1158 */
static void set_params(OracleDomain *d)
{
    d->bad_vol = -1;
    d->bad_q = -1;
    d->dthydro = 1e20;
    d->dtcourant = 1e20;
    d->time = 0.;
    d->dtfixed = -1.0e-6;
    d->deltatimemultlb = 1.1;
    d->deltatimemultub = 1.2;
    d->stoptime = 1.0e-2;
    d->dtmax = 1.0e-2;
    d->cycle = 0;
    d->e_cut = 1.0e-7;
    d->p_cut = 1.0e-7;
    d->q_cut = 1.0e-7;
    d->u_cut = 1.0e-7;
    d->v_cut = 1.0e-10;
    d->hgcoef = 3.0;
    d->ss4o3 = 4.0 / 3.0;
    d->qstop = 1.0e+12;
    d->monoq_max_slope = 1.0;
    d->monoq_limiter_mult = 2.0;
    d->qlc_monoq = 0.5;
    d->qqc_monoq = 2.0 / 3.0;
    d->qqc = 2.0;
    d->pmin = 0.;
    d->emin = -1.0e+15;
    d->dvovmax = 0.1;
    d->eosvmax = 1.0e+9;
    d->eosvmin = 1.0e-9;
    d->refdens = 1.0;
}

/* volo, elemMass, nodalMass, lulesh.cu:1165-1187 */
static void masses(OracleDomain *d)
{
    const int E = d->numElem, Ep = d->Ep;
    for (int i = 0; i < E; ++i) {
        double xl[8], yl[8], zl[8];
        for (int k = 0; k < 8; ++k) {
            int g = d->nodelist[k * Ep + i];
            xl[k] = d->x[g];
            yl[k] = d->y[g];
            zl[k] = d->z[g];
        }
        double vol = elem_volume(xl, yl, zl);
        d->volo[i] = vol;
        d->elemMass[i] = vol;
        for (int k = 0; k < 8; ++k)
            d->nodalMass[d->nodelist[k * Ep + i]] += vol / 8.0;
    }
}

/* lmesh reader: whitespace-separated ints and doubles, 0 at a read failure */
static int rd_int(FILE *f, int *ok)
{
    int v = 0;
    if (*ok && fscanf(f, "%d", &v) != 1) *ok = 0;
    return v;
}

static double rd_real(FILE *f, int *ok)
{
    double v = 0.0;
    if (*ok && fscanf(f, "%lf", &v) != 1) *ok = 0;
    return v;
}

/* OR `bits` of the faces whose four nodes are all marked (the face tests of
 * lulesh.cu:1001-1012, 1035-1045); order zeta-, zeta+, eta-, eta+, xi-, xi+ */
static void mark_faces(OracleDomain *d, const char *mark, const int bits[6])
{
    static const int face[6] = {0x0f, 0xf0, 0x33, 0xcc, 0x99, 0x66};
    for (int z = 0; z < d->numElem; ++z) {
        int mask = 0;
        for (int k = 0; k < 8; ++k)
            if (mark[d->nodelist[k * d->Ep + z]]) mask |= 1 << k;
        for (int f = 0; f < 6; ++f)
            if ((mask & face[f]) == face[f]) d->elemBC[z] |= bits[f];
    }
}

OracleDomain *oracle_create_lmesh(const char *path, int numReg, int balance, int cost)
{
    if (!path || numReg < 1) return NULL;
    FILE *f = fopen(path, "r");
    if (!f) return NULL;
    int ok = 1;
    const int E = rd_int(f, &ok), N = rd_int(f, &ok);
    if (!ok || E < 1 || N < 8) {
        fclose(f);
        return NULL;
    }
    OracleDomain *d = (OracleDomain *)zalloc(sizeof(OracleDomain));
    d->nx = 0;
    d->tp = 1;
    d->cost = cost;
    d->numElem = E;
    d->numNode = N;
    d->Ep = ((E + 31) / 32) * 32;
    d->allElem = E;
    const int Ep = d->Ep;
    d->e = ZD(E); d->p = ZD(E); d->q = ZD(E); d->ql = ZD(E); d->qq = ZD(E);
    d->v = ZD(E); d->volo = ZD(E); d->delv = ZD(E); d->vdov = ZD(E);
    d->arealg = ZD(E); d->ss = ZD(E); d->elemMass = ZD(E);
    d->x = ZD(N); d->y = ZD(N); d->z = ZD(N);
    d->xd = ZD(N); d->yd = ZD(N); d->zd = ZD(N);
    d->xdd = ZD(N); d->ydd = ZD(N); d->zdd = ZD(N);
    d->fx = ZD(N); d->fy = ZD(N); d->fz = ZD(N); d->nodalMass = ZD(N);
    d->vnew = ZD(E);
    d->delx_xi = ZD(E); d->delx_eta = ZD(E); d->delx_zeta = ZD(E);
    d->delv_xi = ZD(E); d->delv_eta = ZD(E); d->delv_zeta = ZD(E);
    d->fx_elem = ZD(8 * Ep); d->fy_elem = ZD(8 * Ep); d->fz_elem = ZD(8 * Ep);
    for (int i = 0; i < E; ++i) d->v[i] = 1.0;

    /* the -u branch of NewDomain, lulesh.cu:855-1052 */
    for (int i = 0; i < N; ++i) {
        d->x[i] = rd_real(f, &ok);
        d->y[i] = rd_real(f, &ok);
        d->z[i] = rd_real(f, &ok);
    }
    d->nodelist = ZI(8 * Ep);
    for (int z = 0; z < E; ++z)
        for (int k = 0; k < 8; ++k) {
            int n = rd_int(f, &ok);
            if (n < 0 || n >= N) ok = 0;
            d->nodelist[k * Ep + z] = ok ? n : 0;
        }
    d->lxim = ZI(E); d->lxip = ZI(E); d->letam = ZI(E); d->letap = ZI(E);
    d->lzetam = ZI(E); d->lzetap = ZI(E); d->elemBC = ZI(E);
    int *links[6] = {d->lxim, d->lxip, d->letam, d->letap, d->lzetam, d->lzetap};
    for (int z = 0; z < E; ++z)
        for (int l = 0; l < 6; ++l) {
            int v = rd_int(f, &ok);
            if (v < 0 || v >= E) ok = 0;
            links[l][z] = ok ? v : 0;
        }
    char *symm = (char *)zalloc((size_t)N), *freesurf = (char *)zalloc((size_t)N);
    int *sets[3] = {NULL, NULL, NULL}, counts[3] = {0, 0, 0};
    for (int a = 0; a < 3; ++a) {
        int c = rd_int(f, &ok);
        if (c < 0 || c > N) ok = 0;
        counts[a] = ok ? c : 0;
        sets[a] = ZI(counts[a]);
        for (int k = 0; k < counts[a]; ++k) {
            int n = rd_int(f, &ok);
            if (n < 0 || n >= N) ok = 0;
            sets[a][k] = ok ? n : 0;
            if (ok) symm[n] = 1;
        }
    }
    int nfree = rd_int(f, &ok);
    if (nfree < 0 || nfree > N) ok = 0;
    for (int k = 0; ok && k < nfree; ++k) {
        int n = rd_int(f, &ok);
        if (n < 0 || n >= N) ok = 0;
        if (ok) freesurf[n] = 1;
    }
    fclose(f);
    int len = 1;
    for (int a = 0; a < 3; ++a) len = counts[a] > len ? counts[a] : len;
    d->symmLen = len;
    int **dst[3] = {&d->symmX, &d->symmY, &d->symmZ};
    for (int a = 0; a < 3; ++a) {
        *dst[a] = ZI(len);
        memcpy(*dst[a], sets[a], sizeof(int) * (size_t)counts[a]);
        free(sets[a]);
    }
    d->numSymmX = counts[0];
    d->numSymmY = counts[1];
    d->numSymmZ = counts[2];
    if (!ok) {
        free(symm);
        free(freesurf);
        oracle_destroy(d);
        return NULL;
    }
    /* boundary masks: symmetry faces, then free-surface faces.  Deliberate
     * difference: the reference tags free-surface faces with the *_SYMM
     * bits (lulesh.cu:1039-1044); they get the *_FREE bits here. */
    const int symm_bits[6] = {BC_ZETA_M_SYMM, BC_ZETA_P_SYMM, BC_ETA_M_SYMM,
                              BC_ETA_P_SYMM, BC_XI_M_SYMM, BC_XI_P_SYMM};
    const int free_bits[6] = {BC_ZETA_M_FREE, BC_ZETA_P_FREE, BC_ETA_M_FREE,
                              BC_ETA_P_FREE, BC_XI_M_FREE, BC_XI_P_FREE};
    mark_faces(d, symm, symm_bits);
    d->octantCorner = 0;
    for (int z = 0; z < E; ++z)
        if (d->elemBC[z] == (BC_XI_M_SYMM | BC_ETA_M_SYMM | BC_ZETA_M_SYMM)) {
            d->octantCorner = z;
            break;
        }
    mark_faces(d, freesurf, free_bits);
    free(symm);
    free(freesurf);

    corner_csr(d);
    set_params(d);
    masses(d);
    /* deposit at the octant corner (lulesh.cu:1050); the shared setup's
     * overwrite with einit(nx = 0) = 0 (lulesh.cu:1189-1205) is not kept */
    const double einit = 3.948746e+7;
    d->e[d->octantCorner] = einit;
    d->deltatime = (.5 * cbrt(d->volo[d->octantCorner])) / sqrt(2 * einit);
    d->initial_deltatime = d->deltatime;
    create_regions(d, numReg, balance);
    return d;
}

void oracle_destroy(OracleDomain *d)
{
    if (!d) return;
    void *ptrs[] = {d->nodelist, d->lxim, d->lxip, d->letam, d->letap,
                    d->lzetam, d->lzetap, d->elemBC, d->nodeElemCount,
                    d->nodeElemStart, d->nodeElemCornerList, d->symmX,
                    d->symmY, d->symmZ, d->matElemlist, d->regElemSize,
                    d->regCSR, d->regReps, d->regNumList, d->regElemlist,
                    d->regSorted, d->e, d->p, d->q, d->ql, d->qq, d->v,
                    d->volo, d->delv, d->vdov, d->arealg, d->ss, d->elemMass,
                    d->x, d->y, d->z, d->xd, d->yd, d->zd, d->xdd, d->ydd,
                    d->zdd, d->fx, d->fy, d->fz, d->nodalMass, d->vnew,
                    d->delx_xi, d->delx_eta, d->delx_zeta, d->delv_xi,
                    d->delv_eta, d->delv_zeta, d->fx_elem, d->fy_elem,
                    d->fz_elem};
    for (size_t i = 0; i < sizeof ptrs / sizeof ptrs[0]; ++i) free(ptrs[i]);
    free(d);
}

/* ------------------------------------------------------------------ */
/* one cycle                                                            */
/* ------------------------------------------------------------------ */

/* TimeIncrement, lulesh.cu:1400-1461 (one domain: no MPI_Allreduce) */
static void time_increment(OracleDomain *d)
{
    double targetdt = d->stoptime - d->time;
    if ((d->dtfixed <= 0.0) && (d->cycle != 0)) {
        double gnewdt = 1.0e+20, newdt, ratio;
        if (d->dtcourant < gnewdt) gnewdt = d->dtcourant / 2.0;
        if (d->dthydro < gnewdt) gnewdt = d->dthydro * 2.0 / 3.0;
        newdt = gnewdt;
        double olddt = d->deltatime;
        ratio = newdt / olddt;
        if (ratio >= 1.0) {
            if (ratio < d->deltatimemultlb)
                newdt = olddt;
            else if (ratio > d->deltatimemultub)
                newdt = olddt * d->deltatimemultub;
        }
        if (newdt > d->dtmax) newdt = d->dtmax;
        d->deltatime = newdt;
    }
    if ((targetdt > d->deltatime) &&
        (targetdt < (4.0 * d->deltatime / 3.0)))
        targetdt = 2.0 * d->deltatime / 3.0;
    if (targetdt < d->deltatime) d->deltatime = targetdt;
    d->time += d->deltatime;
    ++d->cycle;
}

/* CalcVolumeForceForElems_kernel<true/false>, lulesh.cu:2080-2259, then
 * AddNodeForcesFromElems_kernel, lulesh.cu:1715-1751 */
static void volume_force(OracleDomain *d)
{
    const int Ep = d->Ep;
    const double hourg = d->hgcoef;
    for (int el = 0; el < d->numElem; ++el) {
        double xn[8], yn[8], zn[8], xdn[8], ydn[8], zdn[8];
        double dvdx[8], dvdy[8], dvdz[8], hgfx[8], hgfy[8], hgfz[8];
        double hg[8][4], B[3][8];
        double volume = d->v[el];
        double det = d->volo[el] * volume;
        if (volume < 0.) d->bad_vol = el;
        double ss1 = d->ss[el], mass1 = d->elemMass[el];
        double sigxx = -d->p[el] - d->q[el];
        int n[8];
        for (int k = 0; k < 8; ++k) n[k] = d->nodelist[el + k * Ep];
        double volinv = 1.0 / det;
        for (int k = 0; k < 8; ++k) {
            xn[k] = d->x[n[k]];
            yn[k] = d->y[n[k]];
            zn[k] = d->z[n[k]];
        }
        double volume13 = cbrt(det);
        double coefficient = -hourg * 0.01 * ss1 * mass1 / volume13;
        volume_derivative(dvdx, dvdy, dvdz, xn, yn, zn);
        hourglass_modes(xn, yn, zn, dvdx, dvdy, dvdz, hg, volinv);
        shape_derivs(xn, yn, zn, B, &det);
        node_normals(B[0], B[1], B[2], xn, yn, zn);
        if (det < 0.) d->bad_vol = el;
        for (int k = 0; k < 8; ++k) {
            hgfx[k] = -(sigxx * B[0][k]);
            hgfy[k] = -(sigxx * B[1][k]);
            hgfz[k] = -(sigxx * B[2][k]);
        }
        if (hourg > 0.0) {
            for (int k = 0; k < 8; ++k) {
                xdn[k] = d->xd[n[k]];
                ydn[k] = d->yd[n[k]];
                zdn[k] = d->zd[n[k]];
            }
            fb_hourglass(xdn, hg, coefficient, hgfx);
            fb_hourglass(ydn, hg, coefficient, hgfy);
            fb_hourglass(zdn, hg, coefficient, hgfz);
        }
        for (int k = 0; k < 8; ++k) {
            d->fx_elem[el + Ep * k] = hgfx[k];
            d->fy_elem[el + Ep * k] = hgfy[k];
            d->fz_elem[el + Ep * k] = hgfz[k];
        }
    }
    for (int i = 0; i < d->numNode; ++i) {
        int cnt = d->nodeElemCount[i], st = d->nodeElemStart[i];
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int j = 0; j < cnt; ++j) {
            int pos = d->nodeElemCornerList[st + j];
            fx += d->fx_elem[pos];
            fy += d->fy_elem[pos];
            fz += d->fz_elem[pos];
        }
        d->fx[i] = fx;
        d->fy[i] = fy;
        d->fz[i] = fz;
    }
}

/* lulesh.cu:2925-3044: acceleration, symmetry BCs, velocity and position */
static void nodal_update(OracleDomain *d)
{
    for (int i = 0; i < d->numNode; ++i) {
        double inv = 1. / d->nodalMass[i];
        d->xdd[i] = d->fx[i] * inv;
        d->ydd[i] = d->fy[i] * inv;
        d->zdd[i] = d->fz[i] * inv;
    }
    for (int i = 0; i < d->numSymmX; ++i) d->xdd[d->symmX[i]] = 0.0;
    for (int i = 0; i < d->numSymmY; ++i) d->ydd[d->symmY[i]] = 0.0;
    for (int i = 0; i < d->numSymmZ; ++i) d->zdd[d->symmZ[i]] = 0.0;
    const double dt = d->deltatime, u_cut = d->u_cut;
    for (int i = 0; i < d->numNode; ++i) {
        double xt = d->xd[i] + d->xdd[i] * dt;
        double yt = d->yd[i] + d->ydd[i] * dt;
        double zt = d->zd[i] + d->zdd[i] * dt;
        if (fabs(xt) < u_cut) xt = 0.0;
        if (fabs(yt) < u_cut) yt = 0.0;
        if (fabs(zt) < u_cut) zt = 0.0;
        d->x[i] += xt * dt;
        d->y[i] += yt * dt;
        d->z[i] += zt * dt;
        d->xd[i] = xt;
        d->yd[i] = yt;
        d->zd[i] = zt;
    }
}

/* CalcKinematicsAndMonotonicQGradient_kernel, lulesh.cu:3343-3507 */
static void kinematics(OracleDomain *d)
{
    const int Ep = d->Ep;
    const double dt = d->deltatime;
    for (int k = 0; k < d->numElem; ++k) {
        double B[3][8], D[6], xl[8], yl[8], zl[8], xdl[8], ydl[8], zdl[8];
        int nodes[8];
        for (int j = 0; j < 8; ++j) nodes[j] = d->nodelist[k + j * Ep];
        for (int j = 0; j < 8; ++j) {
            xl[j] = d->x[nodes[j]];
            yl[j] = d->y[nodes[j]];
            zl[j] = d->z[nodes[j]];
        }
        double volume = elem_volume(xl, yl, zl);
        double relv = volume / d->volo[k];
        d->vnew[k] = relv;
        d->delv[k] = relv - d->v[k];
        d->arealg[k] = char_length(xl, yl, zl, volume);
        for (int j = 0; j < 8; ++j) {
            xdl[j] = d->xd[nodes[j]];
            ydl[j] = d->yd[nodes[j]];
            zdl[j] = d->zd[nodes[j]];
        }
        double dt2 = 0.5 * dt;
        for (int j = 0; j < 8; ++j) {
            xl[j] -= dt2 * xdl[j];
            yl[j] -= dt2 * ydl[j];
            zl[j] -= dt2 * zdl[j];
        }
        double detJ;
        shape_derivs(xl, yl, zl, B, &detJ);
        velocity_gradient(xdl, ydl, zdl, B, detJ, D);
        double vdovNew = D[0] + D[1] + D[2];
        d->vdov[k] = vdovNew;
        double vol = d->volo[k] * d->vnew[k];
        for (int j = 0; j < 8; ++j) {
            xl[j] += dt2 * xdl[j];
            yl[j] += dt2 * ydl[j];
            zl[j] += dt2 * zdl[j];
        }
        mono_gradient(xl, yl, zl, xdl, ydl, zdl, vol, &d->delx_zeta[k],
                      &d->delv_zeta[k], &d->delx_xi[k], &d->delv_xi[k],
                      &d->delx_eta[k], &d->delv_eta[k]);
        if (relv < 0) d->bad_vol = k;
    }
}

/* one direction of the monotonic limiter, lulesh.cu:3595-3624 */
static double limiter(const double *dv, int i, int mask, int m_symm,
                      int m_free, int p_symm, int p_free, int lm, int lp,
                      int mmask, int pmask, double mult, double maxslope,
                      double ptiny)
{
    double norm = 1. / (dv[i] + ptiny);
    double dm = 0.0, dp = 0.0;
    int mm = mask & mmask, pm = mask & pmask;
    if (mm == m_symm)
        dm = dv[i];
    else if (mm == m_free)
        dm = 0.0;
    else
        dm = dv[lm];
    if (pm == p_symm)
        dp = dv[i];
    else if (pm == p_free)
        dp = 0.0;
    else
        dp = dv[lp];
    dm = dm * norm;
    dp = dp * norm;
    double phi = .5 * (dm + dp);
    dm *= mult;
    dp *= mult;
    if (dm < phi) phi = dm;
    if (dp < phi) phi = dp;
    if (phi < 0.) phi = 0.;
    if (phi > maxslope) phi = maxslope;
    return phi;
}

/* CalcMonotonicQRegionForElems_kernel, lulesh.cu:3554-3725 */
static void monoq_region(OracleDomain *d)
{
    const double ptiny = 1.e-36, mult = d->monoq_limiter_mult,
                 maxs = d->monoq_max_slope;
    for (int ie = 0; ie < d->numElem; ++ie) {
        int i = d->regElemlist[ie];
        int bc = d->elemBC[i];
        double phixi = limiter(d->delv_xi, i, bc, BC_XI_M_SYMM, BC_XI_M_FREE,
                               BC_XI_P_SYMM, BC_XI_P_FREE, d->lxim[i],
                               d->lxip[i], BC_XI_M, BC_XI_P, mult, maxs, ptiny);
        double phieta = limiter(d->delv_eta, i, bc, BC_ETA_M_SYMM,
                                BC_ETA_M_FREE, BC_ETA_P_SYMM, BC_ETA_P_FREE,
                                d->letam[i], d->letap[i], BC_ETA_M, BC_ETA_P,
                                mult, maxs, ptiny);
        double phizeta = limiter(d->delv_zeta, i, bc, BC_ZETA_M_SYMM,
                                 BC_ZETA_M_FREE, BC_ZETA_P_SYMM,
                                 BC_ZETA_P_FREE, d->lzetam[i], d->lzetap[i],
                                 BC_ZETA_M, BC_ZETA_P, mult, maxs, ptiny);
        double qlin, qquad;
        if (d->vdov[i] > 0.) {
            qlin = 0.;
            qquad = 0.;
        } else {
            double dxi = d->delv_xi[i] * d->delx_xi[i];
            double deta = d->delv_eta[i] * d->delx_eta[i];
            double dzeta = d->delv_zeta[i] * d->delx_zeta[i];
            if (dxi > 0.) dxi = 0.;
            if (deta > 0.) deta = 0.;
            if (dzeta > 0.) dzeta = 0.;
            double rho = d->elemMass[i] / (d->volo[i] * d->vnew[i]);
            qlin = -d->qlc_monoq * rho *
                   (dxi * (1. - phixi) + deta * (1. - phieta) +
                    dzeta * (1. - phizeta));
            qquad = d->qqc_monoq * rho *
                    (dxi * dxi * (1. - phixi * phixi) +
                     deta * deta * (1. - phieta * phieta) +
                     dzeta * dzeta * (1. - phizeta * phizeta));
        }
        d->qq[i] = qquad;
        d->ql[i] = qlin;
        if (d->q[i] > d->qstop) d->bad_q = i;
    }
}

/* CalcPressureForElems_device, lulesh.cu:3764-3791 */
static void pressure(double *p_new, double *bvc, double *pbvc, double e_old,
                     double compression, double vnewc, double pmin,
                     double p_cut, double eosvmax)
{
    const double c1s = 2.0 / 3.0;
    *bvc = c1s * (compression + 1.);
    *pbvc = c1s;
    double pt = *bvc * e_old;
    if (fabs(pt) < p_cut) pt = 0.0;
    if (vnewc >= eosvmax) pt = 0.0;
    if (pt < pmin) pt = pmin;
    *p_new = pt;
}

/* CalcEnergyForElems_device, lulesh.cu:3867-3974 */
static void energy(double *p_new, double *e_new, double *q_new, double *bvc,
                   double *pbvc, double p_old, double e_old, double q_old,
                   double compression, double compHalfStep, double vnewc,
                   double work, double delvc, const OracleDomain *d,
                   double qq, double ql, double rho0)
{
    const double sixth = 1.0 / 6.0;
    const double pmin = d->pmin, p_cut = d->p_cut, e_cut = d->e_cut,
                 q_cut = d->q_cut, emin = d->emin, eosvmax = d->eosvmax;
    double pHalf;
    double en = e_old - 0.5 * delvc * (p_old + q_old) + 0.5 * work;
    if (en < emin) en = emin;
    pressure(&pHalf, bvc, pbvc, en, compHalfStep, vnewc, pmin, p_cut, eosvmax);
    double vhalf = 1. / (1. + compHalfStep);
    double qn;
    if (delvc > 0.) {
        qn = 0.;
    } else {
        double ssc = (*pbvc * en + vhalf * vhalf * *bvc * pHalf) / rho0;
        if (ssc <= .1111111e-36)
            ssc = .3333333e-18;
        else
            ssc = sqrt(ssc);
        qn = (ssc * ql + qq);
    }
    en = en + 0.5 * delvc * (3.0 * (p_old + q_old) - 4.0 * (pHalf + qn));
    en += 0.5 * work;
    if (fabs(en) < e_cut) en = 0.;
    if (en < emin) en = emin;
    pressure(p_new, bvc, pbvc, en, compression, vnewc, pmin, p_cut, eosvmax);
    double q_tilde;
    if (delvc > 0.) {
        q_tilde = 0.;
    } else {
        double ssc = (*pbvc * en + vnewc * vnewc * *bvc * *p_new) / rho0;
        if (ssc <= .1111111e-36)
            ssc = .3333333e-18;
        else
            ssc = sqrt(ssc);
        q_tilde = (ssc * ql + qq);
    }
    en = en - (7.0 * (p_old + q_old) - 8.0 * (pHalf + qn) +
               (*p_new + q_tilde)) *
                  delvc * sixth;
    if (fabs(en) < e_cut) en = 0.;
    if (en < emin) en = emin;
    pressure(p_new, bvc, pbvc, en, compression, vnewc, pmin, p_cut, eosvmax);
    if (delvc <= 0.) {
        double ssc = (*pbvc * en + vnewc * vnewc * *bvc * *p_new) / rho0;
        if (ssc <= .1111111e-36)
            ssc = .3333333e-18;
        else
            ssc = sqrt(ssc);
        qn = (ssc * ql + qq);
        if (fabs(qn) < q_cut) qn = 0.;
    }
    *e_new = en;
    *q_new = qn;
}

/* ApplyMaterialPropertiesAndUpdateVolume_kernel, lulesh.cu:3988-4097 */
static void eos(OracleDomain *d)
{
    const double eosvmin = d->eosvmin, eosvmax = d->eosvmax,
                 rho0 = d->refdens;
    for (int i = 0; i < d->numElem; ++i) {
        int z = d->regElemlist[i];
        /* ApplyMaterialPropertiesForElems_device, lulesh.cu:3814-3845 */
        double vnewc = d->vnew[z];
        if (eosvmin != 0.) {
            if (vnewc < eosvmin) vnewc = eosvmin;
        }
        if (eosvmax != 0.) {
            if (vnewc > eosvmax) vnewc = eosvmax;
        }
        double vc = d->v[z];
        if (eosvmin != 0.) {
            if (vc < eosvmin) vc = eosvmin;
        }
        if (eosvmax != 0.) {
            if (vc > eosvmax) vc = eosvmax;
        }
        if (vc <= 0.) d->bad_vol = z;
        /* giveMyRegion, lulesh.cu:3976-3984 (regCSR holds region ends) */
        int region = d->numReg - 1;
        for (int r = 0; r < d->numReg - 1; ++r)
            if (i < d->regCSR[r]) {
                region = r;
                break;
            }
        int rep = d->regReps[region];
        double e_t = d->e[z], p_t = d->p[z], q_t = d->q[z], qq_t = d->qq[z],
               ql_t = d->ql[z], dv_t = d->delv[z];
        double p_new = 0, e_new = 0, q_new = 0, bvc = 0, pbvc = 0;
        for (int r = 0; r < rep; ++r) {
            double p_old = p_t, delvc = dv_t;
            double compression = 1. / vnewc - 1.;
            double vchalf = vnewc - delvc * .5;
            double compHalf = 1. / vchalf - 1.;
            if (eosvmin != 0.) {
                if (vnewc <= eosvmin) compHalf = compression;
            }
            if (eosvmax != 0.) {
                if (vnewc >= eosvmax) {
                    p_old = 0.;
                    compression = 0.;
                    compHalf = 0.;
                }
            }
            energy(&p_new, &e_new, &q_new, &bvc, &pbvc, p_old, e_t, q_t,
                   compression, compHalf, vnewc, 0., delvc, d, qq_t, ql_t,
                   rho0);
        }
        d->p[z] = p_new;
        d->e[z] = e_new;
        d->q[z] = q_new;
        /* CalcSoundSpeedForElems_device, lulesh.cu:3795-3809 */
        double ssTmp = (pbvc * e_new + vnewc * vnewc * bvc * p_new) / rho0;
        if (ssTmp <= .1111111e-36)
            ssTmp = .3333333e-18;
        else
            ssTmp = sqrt(ssTmp);
        d->ss[z] = ssTmp;
        /* UpdateVolumesForElems_device, lulesh.cu:3850-3861 */
        double tmpV = d->vnew[z];
        if (fabs(tmpV - 1.0) < d->v_cut) tmpV = 1.0;
        d->v[z] = tmpV;
    }
}

/* CalcTimeConstraintsForElems, lulesh.cu:4216-4435 (the minimum is exact,
 * so the block/grid reduction order of the reference does not matter) */
static void time_constraints(OracleDomain *d)
{
    const double qqc2 = 64.0 * d->qqc * d->qqc, dvovmax = d->dvovmax;
    double mh = 1.0e+20, mc = 1.0e+20;
    for (int i = 0; i < d->numElem; ++i) {
        int indx = d->matElemlist[i];
        double vd = d->vdov[indx];
        if (vd != 0.) {
            double dtdvov = dvovmax / (fabs(vd) + 1.e-20);
            if (mh > dtdvov) mh = dtdvov;
        }
        double ss = d->ss[indx], area = d->arealg[indx];
        double dtf = ss * ss;
        dtf += ((vd < 0.) ? qqc2 * area * area * vd * vd : 0.);
        dtf = area / sqrt(dtf);
        if (vd != 0. && dtf < mc) mc = dtf;
    }
    d->dtcourant = mc;
    d->dthydro = mh;
}

int oracle_step(OracleDomain *d)
{
    time_increment(d);
    volume_force(d);
    nodal_update(d);
    kinematics(d);
    monoq_region(d);
    eos(d);
    time_constraints(d);
    if (d->bad_vol != -1) return -1;
    if (d->bad_q != -1) return -2;
    return 0;
}

int oracle_run(OracleDomain *d, int its, int *cycles_run)
{
    int n = 0, st = 0;
    while (d->time < d->stoptime) {
        st = oracle_step(d);
        ++n;
        if (st != 0) break;
        if (n == its) break;
    }
    if (cycles_run) *cycles_run = n;
    return st;
}

/* ------------------------------------------------------------------ */
/* decomposed stepping                                                  */
/* ------------------------------------------------------------------ */

void oracle_set_mirror(OracleDomain *d, int dir, const OracleMirror *m)
{
    if (dir < 0 || dir >= 27) return;
    d->has_mirror[dir] = m != NULL;
    if (m) d->mirror[dir] = *m;
}

/* corner forces (the first loop of volume_force) */
static void corner_forces(OracleDomain *d)
{
    const int Ep = d->Ep;
    const double hourg = d->hgcoef;
    for (int el = 0; el < d->numElem; ++el) {
        double xn[8], yn[8], zn[8], xdn[8], ydn[8], zdn[8];
        double dvdx[8], dvdy[8], dvdz[8], hgfx[8], hgfy[8], hgfz[8];
        double hg[8][4], B[3][8];
        double volume = d->v[el];
        double det = d->volo[el] * volume;
        if (volume < 0.) d->bad_vol = el;
        double ss1 = d->ss[el], mass1 = d->elemMass[el];
        double sigxx = -d->p[el] - d->q[el];
        int n[8];
        for (int k = 0; k < 8; ++k) n[k] = d->nodelist[el + k * Ep];
        double volinv = 1.0 / det;
        for (int k = 0; k < 8; ++k) {
            xn[k] = d->x[n[k]];
            yn[k] = d->y[n[k]];
            zn[k] = d->z[n[k]];
        }
        double volume13 = cbrt(det);
        double coefficient = -hourg * 0.01 * ss1 * mass1 / volume13;
        volume_derivative(dvdx, dvdy, dvdz, xn, yn, zn);
        hourglass_modes(xn, yn, zn, dvdx, dvdy, dvdz, hg, volinv);
        shape_derivs(xn, yn, zn, B, &det);
        node_normals(B[0], B[1], B[2], xn, yn, zn);
        if (det < 0.) d->bad_vol = el;
        for (int k = 0; k < 8; ++k) {
            hgfx[k] = -(sigxx * B[0][k]);
            hgfy[k] = -(sigxx * B[1][k]);
            hgfz[k] = -(sigxx * B[2][k]);
        }
        if (hourg > 0.0) {
            for (int k = 0; k < 8; ++k) {
                xdn[k] = d->xd[n[k]];
                ydn[k] = d->yd[n[k]];
                zdn[k] = d->zd[n[k]];
            }
            fb_hourglass(xdn, hg, coefficient, hgfx);
            fb_hourglass(ydn, hg, coefficient, hgfy);
            fb_hourglass(zdn, hg, coefficient, hgfz);
        }
        for (int k = 0; k < 8; ++k) {
            d->fx_elem[el + Ep * k] = hgfx[k];
            d->fy_elem[el + Ep * k] = hgfy[k];
            d->fz_elem[el + Ep * k] = hgfz[k];
        }
    }
}

static const int kCX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int kCY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
static const int kCZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};

static int axis_side(int v, int n) { return v < 0 ? -1 : (v >= n ? 1 : 0); }
static int dir_index(int sx, int sy, int sz) { return (sx + 1) + 3 * (sy + 1) + 9 * (sz + 1); }

/* Node force sums over the whole problem: every node of the subdomain adds
 * the corner forces of the elements that touch it in corner order j = 0..7
 * (the order of nodeElemCornerList on the undecomposed mesh,
 * lulesh.cu:1079-1088), taking an element of a neighbouring subdomain from
 * that neighbour's mirror; then the node update. */
static void nodal_decomposed(OracleDomain *d)
{
    const int nx = d->nx, en = nx + 1;
    for (int i = 0; i < d->numNode; ++i) {
        const int px = i % en, py = (i / en) % en, pz = i / (en * en);
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int j = 0; j < 8; ++j) {
            const int ex = px - kCX[j], ey = py - kCY[j], ez = pz - kCZ[j];
            const int sx = axis_side(ex, nx), sy = axis_side(ey, nx), sz = axis_side(ez, nx);
            const int c = j * d->Ep + ((ez - sz * nx) * nx + (ey - sy * nx)) * nx + (ex - sx * nx);
            if ((sx | sy | sz) == 0) {
                fx += d->fx_elem[c];
                fy += d->fy_elem[c];
                fz += d->fz_elem[c];
            } else {
                const int k = dir_index(sx, sy, sz);
                if (!d->has_mirror[k]) continue;
                fx += d->mirror[k].fx_elem[c];
                fy += d->mirror[k].fy_elem[c];
                fz += d->mirror[k].fz_elem[c];
            }
        }
        d->fx[i] = fx;
        d->fy[i] = fy;
        d->fz[i] = fz;
    }
    nodal_update(d);
}

/* CommSyncPosVel: a node on a max face shared with a neighbour takes
 * x..zd from the neighbour that holds it on its min faces */
static void posvel_decomposed(OracleDomain *d)
{
    const int nx = d->nx, en = nx + 1, tp = d->tp;
    for (int i = 0; i < d->numNode; ++i) {
        const int px = i % en, py = (i / en) % en, pz = i / (en * en);
        const int sx = (px == nx && d->colLoc < tp - 1);
        const int sy = (py == nx && d->rowLoc < tp - 1);
        const int sz = (pz == nx && d->planeLoc < tp - 1);
        if ((sx | sy | sz) == 0) continue;
        const int k = dir_index(sx, sy, sz);
        if (!d->has_mirror[k]) continue;
        const OracleMirror *m = &d->mirror[k];
        const int j = ((pz - sz * nx) * en + (py - sy * nx)) * en + (px - sx * nx);
        d->x[i] = m->x[j];
        d->y[i] = m->y[j];
        d->z[i] = m->z[j];
        d->xd[i] = m->xd[j];
        d->yd[i] = m->yd[j];
        d->zd[i] = m->zd[j];
    }
}

/* CommMonoQ: the delv_* ghost faces take the neighbour's boundary layer */
static void monoq_ghosts_decomposed(OracleDomain *d)
{
    const int nx = d->nx;
    static const int dirs[6][3] = {{0, 0, -1}, {0, 0, 1}, {0, -1, 0},
                                   {0, 1, 0},  {-1, 0, 0}, {1, 0, 0}};
    for (int f = 0; f < 6; ++f) {
        if (d->ghost[f] == INT_MIN) continue;
        const int k = dir_index(dirs[f][0], dirs[f][1], dirs[f][2]);
        if (!d->has_mirror[k]) continue;
        const OracleMirror *m = &d->mirror[k];
        for (int a = 0; a < nx; ++a)
            for (int b = 0; b < nx; ++b) {
                int src;
                switch (f) {
                    case 0: src = ((nx - 1) * nx + a) * nx + b; break;
                    case 1: src = (0 * nx + a) * nx + b; break;
                    case 2: src = (a * nx + (nx - 1)) * nx + b; break;
                    case 3: src = (a * nx + 0) * nx + b; break;
                    case 4: src = (a * nx + b) * nx + (nx - 1); break;
                    default: src = (a * nx + b) * nx + 0; break;
                }
                const int g = d->ghost[f] + a * nx + b;
                d->delv_xi[g] = m->delv_xi[src];
                d->delv_eta[g] = m->delv_eta[src];
                d->delv_zeta[g] = m->delv_zeta[src];
            }
    }
}

int oracle_phase(OracleDomain *d, int phase)
{
    switch (phase) {
        case ORACLE_PHASE_TIME_INCREMENT: time_increment(d); break;
        case ORACLE_PHASE_FORCE: corner_forces(d); break;
        case ORACLE_PHASE_NODAL: nodal_decomposed(d); break;
        case ORACLE_PHASE_POSVEL_SYNC: posvel_decomposed(d); break;
        case ORACLE_PHASE_KINEMATICS: kinematics(d); break;
        case ORACLE_PHASE_MONOQ_GHOST: monoq_ghosts_decomposed(d); break;
        case ORACLE_PHASE_EOS:
            monoq_region(d);
            eos(d);
            time_constraints(d);
            break;
        default: return -5;
    }
    if (d->bad_vol != -1) return -1;
    if (d->bad_q != -1) return -2;
    return 0;
}

/* nodalMass over the whole problem: the volume/8 of every element that
 * touches the node, in ascending global element index (the single-domain
 * element loop of lulesh.cu:1165-1187), neighbours' volumes from mirrors */
void oracle_nodal_mass_decomposed(OracleDomain *d)
{
    const int nx = d->nx, en = nx + 1;
    for (int i = 0; i < d->numNode; ++i) {
        const int px = i % en, py = (i / en) % en, pz = i / (en * en);
        double m = 0.0;
        for (int ez = pz - 1; ez <= pz; ++ez)
            for (int ey = py - 1; ey <= py; ++ey)
                for (int ex = px - 1; ex <= px; ++ex) {
                    const int sx = axis_side(ex, nx), sy = axis_side(ey, nx),
                              sz = axis_side(ez, nx);
                    const int e = ((ez - sz * nx) * nx + (ey - sy * nx)) * nx + (ex - sx * nx);
                    if ((sx | sy | sz) == 0) {
                        m += d->volo[e] / 8.0;
                    } else {
                        const int k = dir_index(sx, sy, sz);
                        if (!d->has_mirror[k]) continue;  /* outside the mesh */
                        m += d->mirror[k].volo[e] / 8.0;
                    }
                }
        d->nodalMass[i] = m;
    }
}

void oracle_set_dt_minima(OracleDomain *d, double dtcourant, double dthydro)
{
    d->dtcourant = dtcourant;
    d->dthydro = dthydro;
}

/* ------------------------------------------------------------------ */
/* accessors                                                            */
/* ------------------------------------------------------------------ */

double *oracle_real_field(OracleDomain *d, const char *name, int *count)
{
    struct {
        const char *n;
        double *p;
        int c;
    } t[] = {{"e", d->e, d->numElem},
             {"p", d->p, d->numElem},
             {"q", d->q, d->numElem},
             {"ql", d->ql, d->numElem},
             {"qq", d->qq, d->numElem},
             {"v", d->v, d->numElem},
             {"volo", d->volo, d->numElem},
             {"delv", d->delv, d->numElem},
             {"vdov", d->vdov, d->numElem},
             {"arealg", d->arealg, d->numElem},
             {"ss", d->ss, d->numElem},
             {"elemMass", d->elemMass, d->numElem},
             {"x", d->x, d->numNode},
             {"y", d->y, d->numNode},
             {"z", d->z, d->numNode},
             {"xd", d->xd, d->numNode},
             {"yd", d->yd, d->numNode},
             {"zd", d->zd, d->numNode},
             {"xdd", d->xdd, d->numNode},
             {"ydd", d->ydd, d->numNode},
             {"zdd", d->zdd, d->numNode},
             {"fx", d->fx, d->numNode},
             {"fy", d->fy, d->numNode},
             {"fz", d->fz, d->numNode},
             {"nodalMass", d->nodalMass, d->numNode},
             {"vnew", d->vnew, d->numElem},
             {"delx_xi", d->delx_xi, d->numElem},
             {"delx_eta", d->delx_eta, d->numElem},
             {"delx_zeta", d->delx_zeta, d->numElem},
             {"delv_xi", d->delv_xi, d->allElem},
             {"delv_eta", d->delv_eta, d->allElem},
             {"delv_zeta", d->delv_zeta, d->allElem},
             {"fx_elem", d->fx_elem, 8 * d->Ep},
             {"fy_elem", d->fy_elem, 8 * d->Ep},
             {"fz_elem", d->fz_elem, 8 * d->Ep}};
    for (size_t i = 0; i < sizeof t / sizeof t[0]; ++i)
        if (strcmp(t[i].n, name) == 0) {
            if (count) *count = t[i].c;
            return t[i].p;
        }
    if (count) *count = 0;
    return NULL;
}

int *oracle_int_field(OracleDomain *d, const char *name, int *count)
{
    struct {
        const char *n;
        int *p;
        int c;
    } t[] = {{"nodelist", d->nodelist, 8 * d->Ep},
             {"lxim", d->lxim, d->numElem},
             {"lxip", d->lxip, d->numElem},
             {"letam", d->letam, d->numElem},
             {"letap", d->letap, d->numElem},
             {"lzetam", d->lzetam, d->numElem},
             {"lzetap", d->lzetap, d->numElem},
             {"elemBC", d->elemBC, d->numElem},
             {"nodeElemCount", d->nodeElemCount, d->numNode},
             {"nodeElemStart", d->nodeElemStart, d->numNode},
             {"nodeElemCornerList", d->nodeElemCornerList, d->cornerListLen},
             {"symmX", d->symmX, d->symmLen},
             {"symmY", d->symmY, d->symmLen},
             {"symmZ", d->symmZ, d->symmLen},
             {"matElemlist", d->matElemlist, d->numElem},
             {"regElemSize", d->regElemSize, d->numReg},
             {"regCSR", d->regCSR, d->numReg},
             {"regReps", d->regReps, d->numReg},
             {"regNumList", d->regNumList, d->numElem},
             {"regElemlist", d->regElemlist, d->numElem},
             {"regSorted", d->regSorted, d->numReg}};
    for (size_t i = 0; i < sizeof t / sizeof t[0]; ++i)
        if (strcmp(t[i].n, name) == 0) {
            if (count) *count = t[i].c;
            return t[i].p;
        }
    if (count) *count = 0;
    return NULL;
}

double oracle_scalar(OracleDomain *d, const char *name)
{
    if (!strcmp(name, "time")) return d->time;
    if (!strcmp(name, "deltatime")) return d->deltatime;
    if (!strcmp(name, "dtcourant")) return d->dtcourant;
    if (!strcmp(name, "dthydro")) return d->dthydro;
    if (!strcmp(name, "cycle")) return d->cycle;
    if (!strcmp(name, "numElem")) return d->numElem;
    if (!strcmp(name, "numNode")) return d->numNode;
    if (!strcmp(name, "padded_numElem")) return d->Ep;
    if (!strcmp(name, "numReg")) return d->numReg;
    if (!strcmp(name, "bad_vol")) return d->bad_vol;
    if (!strcmp(name, "bad_q")) return d->bad_q;
    if (!strcmp(name, "numSymmX")) return d->numSymmX;
    if (!strcmp(name, "numSymmY")) return d->numSymmY;
    if (!strcmp(name, "numSymmZ")) return d->numSymmZ;
    if (!strcmp(name, "initial_deltatime")) return d->initial_deltatime;
    if (!strcmp(name, "allElem")) return d->allElem;
    return NAN;
}

void oracle_set_deltatime(OracleDomain *d, double dt) { d->deltatime = dt; }

double oracle_origin_energy(OracleDomain *d) { return d->e[d->octantCorner]; }

/* symmetry check of plane 0, lulesh.cu:4712-4736 */
void oracle_symmetry(OracleDomain *d, double *max_abs, double *total_abs,
                     double *max_rel)
{
    double ma = 0.0, ta = 0.0, mr = 0.0;
    int nx = d->nx;
    for (int j = 0; j < nx; ++j)
        for (int k = j + 1; k < nx; ++k) {
            double ad = fabs(d->e[j * nx + k] - d->e[k * nx + j]);
            ta += ad;
            if (ma < ad) ma = ad;
            double rd = ad / d->e[k * nx + j];
            if (mr < rd) mr = rd;
        }
    *max_abs = ma;
    *total_abs = ta;
    *max_rel = mr;
}
