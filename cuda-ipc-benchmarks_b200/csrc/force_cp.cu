// force_cp.cu -- corner-parallel force kernel (CalcVolumeForceForElems_kernel,
// LULESH/cuda/src/lulesh.cu:2080-2259, restructured for B200).
//
// One element per 8 threads, one thread per corner; a warp holds four
// elements.  The element's node coordinates and velocities are staged in
// shared memory, and the per-element work is split over the element's eight
// lanes with no redundancy:
//   corner k:  the volume derivative of corner k (VoluDer), its four
//              hourglass-vector entries, its face-normal sum and its three
//              corner forces;
//   lanes:     the 12 hourglass-mode sums, the 12 velocity projections and
//              the 6 face area vectors are each computed once, by one lane.
// Every value is the same expression, in the same operand order, as in the
// reference (and in elem_math.cuh), and every sum is accumulated in the
// reference's order, so results do not change.  What changes is the
// register footprint: a thread holds one corner's state instead of the
// whole element's, so far more warps stay resident to hide FP64 and gather
// latency.
#include <climits>

#include "elem_math.cuh"
#include "kernels.cuh"

namespace lulesh {

constexpr int kCpElems = kCpElemsPerBlock;
constexpr int kCpBlock = 8 * kCpElems;        // 256 threads

// per-element staging area in shared memory
struct CpElem {
    double x[8], y[8], z[8], xd[8], yd[8], zd[8];
    double hg[4][8];    // hourglass vectors, [mode][corner]
    double hm[4][3];    // hourglass-mode sums of the coordinates, [mode][x,y,z]
    double hv[4][3];    // velocity projections h, [mode][x,y,z]
    double area[6][3];  // face area vectors, [face][x,y,z]
};

// VoluDer (lulesh.cu:1756-1784) for corner `out`, with the six corners the
// reference passes for it (CalcElemVolumeDerivative, lulesh.cu:1789-1828).
__device__ __forceinline__ void cp_volu_der(const CpElem &s, int out, double &dvdx, double &dvdy,
                                            double &dvdz)
{
    int m[6];
    switch (out) {
        case 0: m[0] = 1; m[1] = 2; m[2] = 3; m[3] = 4; m[4] = 5; m[5] = 7; break;
        case 1: m[0] = 2; m[1] = 3; m[2] = 0; m[3] = 5; m[4] = 6; m[5] = 4; break;
        case 2: m[0] = 3; m[1] = 0; m[2] = 1; m[3] = 6; m[4] = 7; m[5] = 5; break;
        case 3: m[0] = 0; m[1] = 1; m[2] = 2; m[3] = 7; m[4] = 4; m[5] = 6; break;
        case 4: m[0] = 7; m[1] = 6; m[2] = 5; m[3] = 0; m[4] = 3; m[5] = 1; break;
        case 5: m[0] = 4; m[1] = 7; m[2] = 6; m[3] = 1; m[4] = 0; m[5] = 2; break;
        case 6: m[0] = 5; m[1] = 4; m[2] = 7; m[3] = 2; m[4] = 1; m[5] = 3; break;
        default: m[0] = 6; m[1] = 5; m[2] = 4; m[3] = 3; m[4] = 2; m[5] = 0; break;
    }
    const double twelfth = 1.0 / 12.0;
    const double x0 = s.x[m[0]], x1 = s.x[m[1]], x2 = s.x[m[2]], x3 = s.x[m[3]],
                 x4 = s.x[m[4]], x5 = s.x[m[5]];
    const double y0 = s.y[m[0]], y1 = s.y[m[1]], y2 = s.y[m[2]], y3 = s.y[m[3]],
                 y4 = s.y[m[4]], y5 = s.y[m[5]];
    const double z0 = s.z[m[0]], z1 = s.z[m[1]], z2 = s.z[m[2]], z3 = s.z[m[3]],
                 z4 = s.z[m[4]], z5 = s.z[m[5]];
    dvdx = (y1 + y2) * (z0 + z1) - (y0 + y1) * (z1 + z2) + (y0 + y4) * (z3 + z4) -
           (y3 + y4) * (z0 + z4) - (y2 + y5) * (z3 + z5) + (y3 + y5) * (z2 + z5);
    dvdy = -(x1 + x2) * (z0 + z1) + (x0 + x1) * (z1 + z2) - (x0 + x4) * (z3 + z4) +
           (x3 + x4) * (z0 + z4) + (x2 + x5) * (z3 + z5) - (x3 + x5) * (z2 + z5);
    dvdz = -(y1 + y2) * (x0 + x1) + (y0 + y1) * (x1 + x2) - (y0 + y4) * (x3 + x4) +
           (y3 + y4) * (x0 + x4) + (y2 + y5) * (x3 + x5) - (y3 + y5) * (x2 + x5);
    dvdx *= twelfth;
    dvdy *= twelfth;
    dvdz *= twelfth;
}

// sign of corner k in hourglass mode m (the base vectors of
// CalcHourglassModes, lulesh.cu:2023-2069): bit k of kNeg[m] set = -1
__device__ __forceinline__ bool hg_negative(int m, int k)
{
    // mode 0: + + - - - - + +   mode 1: + - - + - + + -
    // mode 2: + - + - + - + -   mode 3: - + - + + - + -
    const unsigned neg = (m == 0) ? 0x3Cu : (m == 1) ? 0x96u : (m == 2) ? 0xAAu : 0xA5u;
    return (neg >> k) & 1u;
}

// signed left-to-right sum over the eight corners of mode m, as the
// reference writes it (xn[0] + xn[1] - xn[2] ... ; mode 3 starts -xn[0])
__device__ __forceinline__ double hg_mode_sum(int m, const double a[8])
{
    double s = hg_negative(m, 0) ? -a[0] : a[0];
#pragma unroll
    for (int k = 1; k < 8; ++k) s = hg_negative(m, k) ? s - a[k] : s + a[k];
    return s;
}

// face f of CalcElemNodeNormals in the reference's corner order
__device__ __forceinline__ void cp_face(int f, int &a, int &b, int &c, int &d)
{
    switch (f) {
        case 0: a = 0; b = 1; c = 2; d = 3; break;
        case 1: a = 0; b = 4; c = 5; d = 1; break;
        case 2: a = 1; b = 5; c = 6; d = 2; break;
        case 3: a = 2; b = 6; c = 7; d = 3; break;
        case 4: a = 3; b = 7; c = 4; d = 0; break;
        default: a = 4; b = 7; c = 6; d = 5; break;
    }
}

// bit f set: face f contains corner k
__device__ __forceinline__ unsigned faces_of_corner(int k)
{
    // faces: 0 {0,1,2,3} 1 {0,4,5,1} 2 {1,5,6,2} 3 {2,6,7,3} 4 {3,7,4,0} 5 {4,7,6,5}
    switch (k) {
        case 0: return 0x13u;  // faces 0,1,4
        case 1: return 0x07u;  // 0,1,2
        case 2: return 0x0Du;  // 0,2,3
        case 3: return 0x19u;  // 0,3,4
        case 4: return 0x32u;  // 1,4,5
        case 5: return 0x26u;  // 1,2,5
        case 6: return 0x2Cu;  // 2,3,5
        default: return 0x38u; // 3,4,5
    }
}

template <bool HG>
__global__ void __launch_bounds__(kCpBlock, kForceCpMinBlocks) k_force_cp(SetArgs a, Params P)
{
    __shared__ CpElem sm[kCpElems];
    const int2 blk = a.blocks[blockIdx.x];
    const DomDev &D = a.doms[blk.x];
    TimeCtl &T = a.tcs[D.tc];
    if (!T.active) return;  // uniform per block
    const int le = threadIdx.x >> 3;   // element slot in the block
    const int k = threadIdx.x & 7;     // corner
    const int elem = blk.y + le;
    const bool valid = elem < D.numElem;
    const unsigned wmask = 0xffffffffu;
    CpElem &s = sm[le];

    // ---- stage the element's nodes (corner k loads node k)
    const int nx = D.nx, en = D.en;
    int node = 0;
    double volume = 0.0, det = 1.0, ss1 = 0.0, mass1 = 0.0, sigxx = 0.0;
    if (valid) {
        const int ix = elem % nx, t = elem / nx, iy = t % nx, iz = t / nx;
        const int cx = (0x66 >> k) & 1, cy = (0xCC >> k) & 1, cz = (0xF0 >> k) & 1;
        node = ((iz + cz) * en + (iy + cy)) * en + (ix + cx);
        s.x[k] = D.x[node];
        s.y[k] = D.y[node];
        s.z[k] = D.z[node];
        if (HG) {
            s.xd[k] = D.xd[node];
            s.yd[k] = D.yd[node];
            s.zd[k] = D.zd[node];
        }
        volume = D.v[elem];
        det = D.volo[elem] * volume;
        ss1 = D.ss[elem];
        mass1 = D.elemMass[elem];
        sigxx = -D.p[elem] - D.q[elem];
        if (k == 0 && volume < 0.) atomicMin(&T.bad_vol, elem);
    }
    __syncwarp(wmask);
    const double volinv = 1.0 / det;

    // ---- hourglass-mode coordinate sums: lanes 0-3 do modes 0-3 for x
    //      and y, lanes 4-7 modes 0-3 for z
    if (valid) {
        const int m = k & 3;
        if (k < 4) {
            s.hm[m][0] = hg_mode_sum(m, s.x);
            s.hm[m][1] = hg_mode_sum(m, s.y);
        } else {
            s.hm[m][2] = hg_mode_sum(m, s.z);
        }
    }
    __syncwarp(wmask);

    // ---- corner k: volume derivative and hourglass-vector entries
    double hgk[4] = {0, 0, 0, 0};
    if (valid) {
        double dvdx, dvdy, dvdz;
        cp_volu_der(s, k, dvdx, dvdy, dvdz);
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            const double g = hg_negative(m, k) ? -1.0 : 1.0;
            hgk[m] = g - volinv * (dvdx * s.hm[m][0] + dvdy * s.hm[m][1] + dvdz * s.hm[m][2]);
            s.hg[m][k] = hgk[m];
        }
    }
    // ---- face area vectors: lane f < 6 computes face f (SumElemFaceNormal)
    if (valid && k < 6) {
        int A, B, C, Dd;
        cp_face(k, A, B, C, Dd);
        const double bisectX0 = 0.5 * (s.x[Dd] + s.x[C] - s.x[B] - s.x[A]);
        const double bisectY0 = 0.5 * (s.y[Dd] + s.y[C] - s.y[B] - s.y[A]);
        const double bisectZ0 = 0.5 * (s.z[Dd] + s.z[C] - s.z[B] - s.z[A]);
        const double bisectX1 = 0.5 * (s.x[C] + s.x[B] - s.x[Dd] - s.x[A]);
        const double bisectY1 = 0.5 * (s.y[C] + s.y[B] - s.y[Dd] - s.y[A]);
        const double bisectZ1 = 0.5 * (s.z[C] + s.z[B] - s.z[Dd] - s.z[A]);
        s.area[k][0] = 0.25 * (bisectY0 * bisectZ1 - bisectZ0 * bisectY1);
        s.area[k][1] = 0.25 * (bisectZ0 * bisectX1 - bisectX0 * bisectZ1);
        s.area[k][2] = 0.25 * (bisectX0 * bisectY1 - bisectY0 * bisectX1);
    }
    // ---- lane 7: Jacobian determinant (volume error check only) and the
    //      hourglass coefficient
    double coefficient = 0.0;
    if (valid && k == 7) {
        double B[3][8];  // only the determinant is used (the normals replace B)
        double detJ;
        shape_function_derivatives(s.x, s.y, s.z, B, &detJ);
        if (detJ < 0.) atomicMin(&T.bad_vol, elem);
        const double hourg = P.hgcoef;
        const double volume13 = cbrt(det);
        coefficient = -hourg * 0.01 * ss1 * mass1 / volume13;
    }
    coefficient = __shfl_sync(wmask, coefficient, (threadIdx.x & 31) | 7);
    __syncwarp(wmask);

    // ---- velocity projections h[m][c] = sum_j hg[m][j] * v_c[j], j in order:
    //      lanes 0-3: modes 0-3 of xd and yd; lanes 4-7: modes 0-3 of zd
    if (HG && valid) {
        const int m = k & 3;
        const double *g = s.hg[m];
        if (k < 4) {
            s.hv[m][0] = g[0] * s.xd[0] + g[1] * s.xd[1] + g[2] * s.xd[2] + g[3] * s.xd[3] +
                         g[4] * s.xd[4] + g[5] * s.xd[5] + g[6] * s.xd[6] + g[7] * s.xd[7];
            s.hv[m][1] = g[0] * s.yd[0] + g[1] * s.yd[1] + g[2] * s.yd[2] + g[3] * s.yd[3] +
                         g[4] * s.yd[4] + g[5] * s.yd[5] + g[6] * s.yd[6] + g[7] * s.yd[7];
        } else {
            s.hv[m][2] = g[0] * s.zd[0] + g[1] * s.zd[1] + g[2] * s.zd[2] + g[3] * s.zd[3] +
                         g[4] * s.zd[4] + g[5] * s.zd[5] + g[6] * s.zd[6] + g[7] * s.zd[7];
        }
    }
    __syncwarp(wmask);
    if (!valid) return;

    // ---- corner k: node normal (faces accumulated in face order), stress
    //      force, hourglass force
    const unsigned fm = faces_of_corner(k);
    double pfx = 0.0, pfy = 0.0, pfz = 0.0;
#pragma unroll
    for (int f = 0; f < 6; ++f)
        if ((fm >> f) & 1u) {
            pfx += s.area[f][0];
            pfy += s.area[f][1];
            pfz += s.area[f][2];
        }
    double hgfx = -(sigxx * pfx);
    double hgfy = -(sigxx * pfy);
    double hgfz = -(sigxx * pfz);
    if (HG) {
        hgfx += coefficient * (hgk[0] * s.hv[0][0] + hgk[1] * s.hv[1][0] + hgk[2] * s.hv[2][0] +
                               hgk[3] * s.hv[3][0]);
        hgfy += coefficient * (hgk[0] * s.hv[0][1] + hgk[1] * s.hv[1][1] + hgk[2] * s.hv[2][1] +
                               hgk[3] * s.hv[3][1]);
        hgfz += coefficient * (hgk[0] * s.hv[0][2] + hgk[1] * s.hv[1][2] + hgk[2] * s.hv[2][2] +
                               hgk[3] * s.hv[3][2]);
    }
    const int Ep = D.Ep;
    D.fx_elem[elem + Ep * k] = hgfx;
    D.fy_elem[elem + Ep * k] = hgfy;
    D.fz_elem[elem + Ep * k] = hgfz;
}

void launch_force_cp(const SetArgs &a, int nblocks_cp, Params P, cudaStream_t s)
{
    if (P.hgcoef > 0.0)
        k_force_cp<true><<<nblocks_cp, kCpBlock, 0, s>>>(a, P);
    else
        k_force_cp<false><<<nblocks_cp, kCpBlock, 0, s>>>(a, P);
}

}  // namespace lulesh
