// elem_math.cuh -- per-element hexahedron arithmetic of the LULESH step.
//
// Each function restates one device helper of LULESH/cuda/src/lulesh.cu and
// keeps every expression in the reference's written form (same operands,
// same association), so nvcc makes the same multiply-add contractions and
// the FP64 results match the reference build.  Templated on the compute
// type T so the mixed-precision path can run the same steps in FP32.
#pragma once

namespace lulesh {

__device__ __forceinline__ double sqrt_t(double a) { return sqrt(a); }
__device__ __forceinline__ float sqrt_t(float a) { return sqrtf(a); }
__device__ __forceinline__ double cbrt_t(double a) { return cbrt(a); }
__device__ __forceinline__ float cbrt_t(float a) { return cbrtf(a); }
__device__ __forceinline__ double fmax_t(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ float fmax_t(float a, float b) { return fmaxf(a, b); }

// TRIPLE_PRODUCT of lulesh.cu:287-288, with its argument binding
template <typename T>
__device__ __forceinline__ T triple_product(T x1, T y1, T z1, T x2, T y2, T z2,
                                            T x3, T y3, T z3)
{
    return ((x1) * ((y2) * (z3) - (z2) * (y3)) + (x2) * ((z1) * (y3) - (y1) * (z3)) +
            (x3) * ((y1) * (z2) - (z1) * (y2)));
}

// CalcElemVolume, lulesh.cu:221-307
template <typename T>
__device__ __forceinline__ T elem_volume(const T x[8], const T y[8], const T z[8])
{
    const T twelveth = T(1.0) / T(12.0);
    T dx61 = x[6] - x[1], dy61 = y[6] - y[1], dz61 = z[6] - z[1];
    T dx70 = x[7] - x[0], dy70 = y[7] - y[0], dz70 = z[7] - z[0];
    T dx63 = x[6] - x[3], dy63 = y[6] - y[3], dz63 = z[6] - z[3];
    T dx20 = x[2] - x[0], dy20 = y[2] - y[0], dz20 = z[2] - z[0];
    T dx50 = x[5] - x[0], dy50 = y[5] - y[0], dz50 = z[5] - z[0];
    T dx64 = x[6] - x[4], dy64 = y[6] - y[4], dz64 = z[6] - z[4];
    T dx31 = x[3] - x[1], dy31 = y[3] - y[1], dz31 = z[3] - z[1];
    T dx72 = x[7] - x[2], dy72 = y[7] - y[2], dz72 = z[7] - z[2];
    T dx43 = x[4] - x[3], dy43 = y[4] - y[3], dz43 = z[4] - z[3];
    T dx57 = x[5] - x[7], dy57 = y[5] - y[7], dz57 = z[5] - z[7];
    T dx14 = x[1] - x[4], dy14 = y[1] - y[4], dz14 = z[1] - z[4];
    T dx25 = x[2] - x[5], dy25 = y[2] - y[5], dz25 = z[2] - z[5];
    T volume = triple_product(dx31 + dx72, dx63, dx20, dy31 + dy72, dy63, dy20,
                              dz31 + dz72, dz63, dz20) +
               triple_product(dx43 + dx57, dx64, dx70, dy43 + dy57, dy64, dy70,
                              dz43 + dz57, dz64, dz70) +
               triple_product(dx14 + dx25, dx61, dx50, dy14 + dy25, dy61, dy50,
                              dz14 + dz25, dz61, dz50);
    volume *= twelveth;
    return volume;
}

// CalcElemShapeFunctionDerivatives, lulesh.cu:1466-1561
template <typename T>
__device__ __forceinline__ void shape_function_derivatives(const T x[8], const T y[8],
                                                           const T z[8], T b[3][8],
                                                           T *volume)
{
    const T fjxxi = T(.125) * ((x[6] - x[0]) + (x[5] - x[3]) - (x[7] - x[1]) - (x[4] - x[2]));
    const T fjxet = T(.125) * ((x[6] - x[0]) - (x[5] - x[3]) + (x[7] - x[1]) - (x[4] - x[2]));
    const T fjxze = T(.125) * ((x[6] - x[0]) + (x[5] - x[3]) + (x[7] - x[1]) + (x[4] - x[2]));
    const T fjyxi = T(.125) * ((y[6] - y[0]) + (y[5] - y[3]) - (y[7] - y[1]) - (y[4] - y[2]));
    const T fjyet = T(.125) * ((y[6] - y[0]) - (y[5] - y[3]) + (y[7] - y[1]) - (y[4] - y[2]));
    const T fjyze = T(.125) * ((y[6] - y[0]) + (y[5] - y[3]) + (y[7] - y[1]) + (y[4] - y[2]));
    const T fjzxi = T(.125) * ((z[6] - z[0]) + (z[5] - z[3]) - (z[7] - z[1]) - (z[4] - z[2]));
    const T fjzet = T(.125) * ((z[6] - z[0]) - (z[5] - z[3]) + (z[7] - z[1]) - (z[4] - z[2]));
    const T fjzze = T(.125) * ((z[6] - z[0]) + (z[5] - z[3]) + (z[7] - z[1]) + (z[4] - z[2]));

    const T cjxxi = (fjyet * fjzze) - (fjzet * fjyze);
    const T cjxet = -(fjyxi * fjzze) + (fjzxi * fjyze);
    const T cjxze = (fjyxi * fjzet) - (fjzxi * fjyet);
    const T cjyxi = -(fjxet * fjzze) + (fjzet * fjxze);
    const T cjyet = (fjxxi * fjzze) - (fjzxi * fjxze);
    const T cjyze = -(fjxxi * fjzet) + (fjzxi * fjxet);
    const T cjzxi = (fjxet * fjyze) - (fjyet * fjxze);
    const T cjzet = -(fjxxi * fjyze) + (fjyxi * fjxze);
    const T cjzze = (fjxxi * fjyet) - (fjyxi * fjxet);

    // partials for corners 0-3; 4-7 are their negatives by symmetry
    b[0][0] = -cjxxi - cjxet - cjxze;
    b[0][1] = cjxxi - cjxet - cjxze;
    b[0][2] = cjxxi + cjxet - cjxze;
    b[0][3] = -cjxxi + cjxet - cjxze;
    b[1][0] = -cjyxi - cjyet - cjyze;
    b[1][1] = cjyxi - cjyet - cjyze;
    b[1][2] = cjyxi + cjyet - cjyze;
    b[1][3] = -cjyxi + cjyet - cjyze;
    b[2][0] = -cjzxi - cjzet - cjzze;
    b[2][1] = cjzxi - cjzet - cjzze;
    b[2][2] = cjzxi + cjzet - cjzze;
    b[2][3] = -cjzxi + cjzet - cjzze;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        b[c][4] = -b[c][2];
        b[c][5] = -b[c][3];
        b[c][6] = -b[c][0];
        b[c][7] = -b[c][1];
    }
    *volume = T(8.) * (fjxet * cjxet + fjyet * cjyet + fjzet * cjzet);
}

// SumElemFaceNormal, lulesh.cu:1566-1599, for the face with corners
// (a, b, c, d) in the reference's call order
template <typename T, int A, int B, int C, int D>
__device__ __forceinline__ void sum_face_normal(T pfx[8], T pfy[8], T pfz[8], const T x[8],
                                                const T y[8], const T z[8])
{
    const T bisectX0 = T(0.5) * (x[D] + x[C] - x[B] - x[A]);
    const T bisectY0 = T(0.5) * (y[D] + y[C] - y[B] - y[A]);
    const T bisectZ0 = T(0.5) * (z[D] + z[C] - z[B] - z[A]);
    const T bisectX1 = T(0.5) * (x[C] + x[B] - x[D] - x[A]);
    const T bisectY1 = T(0.5) * (y[C] + y[B] - y[D] - y[A]);
    const T bisectZ1 = T(0.5) * (z[C] + z[B] - z[D] - z[A]);
    const T areaX = T(0.25) * (bisectY0 * bisectZ1 - bisectZ0 * bisectY1);
    const T areaY = T(0.25) * (bisectZ0 * bisectX1 - bisectX0 * bisectZ1);
    const T areaZ = T(0.25) * (bisectX0 * bisectY1 - bisectY0 * bisectX1);
    pfx[A] += areaX; pfx[B] += areaX; pfx[C] += areaX; pfx[D] += areaX;
    pfy[A] += areaY; pfy[B] += areaY; pfy[C] += areaY; pfy[D] += areaY;
    pfz[A] += areaZ; pfz[B] += areaZ; pfz[C] += areaZ; pfz[D] += areaZ;
}

// CalcElemNodeNormals, lulesh.cu:1657-1711 (six faces in this order)
template <typename T>
__device__ __forceinline__ void elem_node_normals(T pfx[8], T pfy[8], T pfz[8], const T x[8],
                                                  const T y[8], const T z[8])
{
#pragma unroll
    for (int i = 0; i < 8; ++i) pfx[i] = pfy[i] = pfz[i] = T(0.0);
    sum_face_normal<T, 0, 1, 2, 3>(pfx, pfy, pfz, x, y, z);
    sum_face_normal<T, 0, 4, 5, 1>(pfx, pfy, pfz, x, y, z);
    sum_face_normal<T, 1, 5, 6, 2>(pfx, pfy, pfz, x, y, z);
    sum_face_normal<T, 2, 6, 7, 3>(pfx, pfy, pfz, x, y, z);
    sum_face_normal<T, 3, 7, 4, 0>(pfx, pfy, pfz, x, y, z);
    sum_face_normal<T, 4, 7, 6, 5>(pfx, pfy, pfz, x, y, z);
}

// VoluDer, lulesh.cu:1756-1784, over the six corners (n0..n5) the caller
// passes, writing corner OUT
template <typename T, int OUT, int N0, int N1, int N2, int N3, int N4, int N5>
__device__ __forceinline__ void volu_der(T dvdx[8], T dvdy[8], T dvdz[8], const T x[8],
                                         const T y[8], const T z[8])
{
    const T twelfth = T(1.0) / T(12.0);
    const T x0 = x[N0], x1 = x[N1], x2 = x[N2], x3 = x[N3], x4 = x[N4], x5 = x[N5];
    const T y0 = y[N0], y1 = y[N1], y2 = y[N2], y3 = y[N3], y4 = y[N4], y5 = y[N5];
    const T z0 = z[N0], z1 = z[N1], z2 = z[N2], z3 = z[N3], z4 = z[N4], z5 = z[N5];
    T ddx = (y1 + y2) * (z0 + z1) - (y0 + y1) * (z1 + z2) + (y0 + y4) * (z3 + z4) -
            (y3 + y4) * (z0 + z4) - (y2 + y5) * (z3 + z5) + (y3 + y5) * (z2 + z5);
    T ddy = -(x1 + x2) * (z0 + z1) + (x0 + x1) * (z1 + z2) - (x0 + x4) * (z3 + z4) +
            (x3 + x4) * (z0 + z4) + (x2 + x5) * (z3 + z5) - (x3 + x5) * (z2 + z5);
    T ddz = -(y1 + y2) * (x0 + x1) + (y0 + y1) * (x1 + x2) - (y0 + y4) * (x3 + x4) +
            (y3 + y4) * (x0 + x4) + (y2 + y5) * (x3 + x5) - (y3 + y5) * (x2 + x5);
    ddx *= twelfth;
    ddy *= twelfth;
    ddz *= twelfth;
    dvdx[OUT] = ddx;
    dvdy[OUT] = ddy;
    dvdz[OUT] = ddz;
}

// CalcElemVolumeDerivative, lulesh.cu:1789-1828 (same call order)
template <typename T>
__device__ __forceinline__ void elem_volume_derivative(T dvdx[8], T dvdy[8], T dvdz[8],
                                                       const T x[8], const T y[8], const T z[8])
{
    volu_der<T, 0, 1, 2, 3, 4, 5, 7>(dvdx, dvdy, dvdz, x, y, z);
    volu_der<T, 3, 0, 1, 2, 7, 4, 6>(dvdx, dvdy, dvdz, x, y, z);
    volu_der<T, 2, 3, 0, 1, 6, 7, 5>(dvdx, dvdy, dvdz, x, y, z);
    volu_der<T, 1, 2, 3, 0, 5, 6, 4>(dvdx, dvdy, dvdz, x, y, z);
    volu_der<T, 4, 7, 6, 5, 0, 3, 1>(dvdx, dvdy, dvdz, x, y, z);
    volu_der<T, 5, 4, 7, 6, 1, 0, 2>(dvdx, dvdy, dvdz, x, y, z);
    volu_der<T, 6, 5, 4, 7, 2, 1, 3>(dvdx, dvdy, dvdz, x, y, z);
    volu_der<T, 7, 6, 5, 4, 3, 2, 0>(dvdx, dvdy, dvdz, x, y, z);
}

// CalcHourglassModes, lulesh.cu:2017-2071.  The four hourglass base
// vectors are the sign patterns below; the reference writes each signed
// sum out left to right, which the S* helpers reproduce term by term.
#define LULESH_HG_SUM(a, s0, s1, s2, s3, s4, s5, s6, s7)                             \
    (s0 a[0] s1 a[1] s2 a[2] s3 a[3] s4 a[4] s5 a[5] s6 a[6] s7 a[7])

template <typename T>
__device__ __forceinline__ void hourglass_modes(const T xn[8], const T yn[8], const T zn[8],
                                                const T dvdxn[8], const T dvdyn[8],
                                                const T dvdzn[8], T hourgam[8][4], T volinv)
{
    T hx, hy, hz;
#define LULESH_HG_MODE(m, g0, g1, g2, g3, g4, g5, g6, g7)                              \
    hourgam[0][m] = T(g0) - volinv * (dvdxn[0] * hx + dvdyn[0] * hy + dvdzn[0] * hz);  \
    hourgam[1][m] = T(g1) - volinv * (dvdxn[1] * hx + dvdyn[1] * hy + dvdzn[1] * hz);  \
    hourgam[2][m] = T(g2) - volinv * (dvdxn[2] * hx + dvdyn[2] * hy + dvdzn[2] * hz);  \
    hourgam[3][m] = T(g3) - volinv * (dvdxn[3] * hx + dvdyn[3] * hy + dvdzn[3] * hz);  \
    hourgam[4][m] = T(g4) - volinv * (dvdxn[4] * hx + dvdyn[4] * hy + dvdzn[4] * hz);  \
    hourgam[5][m] = T(g5) - volinv * (dvdxn[5] * hx + dvdyn[5] * hy + dvdzn[5] * hz);  \
    hourgam[6][m] = T(g6) - volinv * (dvdxn[6] * hx + dvdyn[6] * hy + dvdzn[6] * hz);  \
    hourgam[7][m] = T(g7) - volinv * (dvdxn[7] * hx + dvdyn[7] * hy + dvdzn[7] * hz);

    hx = LULESH_HG_SUM(xn, +, +, -, -, -, -, +, +);
    hy = LULESH_HG_SUM(yn, +, +, -, -, -, -, +, +);
    hz = LULESH_HG_SUM(zn, +, +, -, -, -, -, +, +);
    LULESH_HG_MODE(0, 1.0, 1.0, -1.0, -1.0, -1.0, -1.0, 1.0, 1.0)
    hx = LULESH_HG_SUM(xn, +, -, -, +, -, +, +, -);
    hy = LULESH_HG_SUM(yn, +, -, -, +, -, +, +, -);
    hz = LULESH_HG_SUM(zn, +, -, -, +, -, +, +, -);
    LULESH_HG_MODE(1, 1.0, -1.0, -1.0, 1.0, -1.0, 1.0, 1.0, -1.0)
    hx = LULESH_HG_SUM(xn, +, -, +, -, +, -, +, -);
    hy = LULESH_HG_SUM(yn, +, -, +, -, +, -, +, -);
    hz = LULESH_HG_SUM(zn, +, -, +, -, +, -, +, -);
    LULESH_HG_MODE(2, 1.0, -1.0, 1.0, -1.0, 1.0, -1.0, 1.0, -1.0)
    hx = LULESH_HG_SUM(xn, -, +, -, +, +, -, +, -);
    hy = LULESH_HG_SUM(yn, -, +, -, +, +, -, +, -);
    hz = LULESH_HG_SUM(zn, -, +, -, +, +, -, +, -);
    LULESH_HG_MODE(3, -1.0, 1.0, -1.0, 1.0, 1.0, -1.0, 1.0, -1.0)
#undef LULESH_HG_MODE
}
#undef LULESH_HG_SUM

// CalcElemFBHourglassForce, lulesh.cu:1833-2013, for one velocity
// component: hgf[k] += coefficient * sum_m hourgam[k][m] * (hourgam[:,m] . vel)
template <typename T>
__device__ __forceinline__ void fb_hourglass_component(const T vel[8], const T hourgam[8][4],
                                                       T coefficient, T hgf[8])
{
    T h[4];
#pragma unroll
    for (int m = 0; m < 4; ++m)
        h[m] = hourgam[0][m] * vel[0] + hourgam[1][m] * vel[1] + hourgam[2][m] * vel[2] +
               hourgam[3][m] * vel[3] + hourgam[4][m] * vel[4] + hourgam[5][m] * vel[5] +
               hourgam[6][m] * vel[6] + hourgam[7][m] * vel[7];
#pragma unroll
    for (int k = 0; k < 8; ++k)
        hgf[k] += coefficient * (hourgam[k][0] * h[0] + hourgam[k][1] * h[1] +
                                 hourgam[k][2] * h[2] + hourgam[k][3] * h[3]);
}

// AreaFace, lulesh.cu:3103-3122, for corners (a,b,c,d) in call order
template <typename T, int A, int B, int C, int D>
__device__ __forceinline__ T area_face(const T x[8], const T y[8], const T z[8])
{
    const T fx = (x[C] - x[A]) - (x[D] - x[B]);
    const T fy = (y[C] - y[A]) - (y[D] - y[B]);
    const T fz = (z[C] - z[A]) - (z[D] - z[B]);
    const T gx = (x[C] - x[A]) + (x[D] - x[B]);
    const T gy = (y[C] - y[A]) + (y[D] - y[B]);
    const T gz = (z[C] - z[A]) + (z[D] - z[B]);
    const T temp = (fx * gx + fy * gy + fz * gz);
    return (fx * fx + fy * fy + fz * fz) * (gx * gx + gy * gy + gz * gz) - temp * temp;
}

// CalcElemCharacteristicLength, lulesh.cu:3126-3166
template <typename T>
__device__ __forceinline__ T elem_characteristic_length(const T x[8], const T y[8],
                                                        const T z[8], T volume)
{
    T charLength = T(0.0);
    charLength = fmax_t(area_face<T, 0, 1, 2, 3>(x, y, z), charLength);
    charLength = fmax_t(area_face<T, 4, 5, 6, 7>(x, y, z), charLength);
    charLength = fmax_t(area_face<T, 0, 1, 5, 4>(x, y, z), charLength);
    charLength = fmax_t(area_face<T, 1, 2, 6, 5>(x, y, z), charLength);
    charLength = fmax_t(area_face<T, 2, 3, 7, 6>(x, y, z), charLength);
    charLength = fmax_t(area_face<T, 3, 0, 4, 7>(x, y, z), charLength);
    charLength = T(4.0) * volume / sqrt_t(charLength);
    return charLength;
}

// CalcElemVelocityGradient, lulesh.cu:3171-3248; only d[0..2] feed the
// step (the deviatoric d[3..5] and dxx/dyy/dzz are dead in the reference)
template <typename T>
__device__ __forceinline__ void elem_velocity_divergence(const T xvel[8], const T yvel[8],
                                                         const T zvel[8], const T b[3][8],
                                                         const T detJ, T d[3])
{
    const T inv_detJ = T(1.0) / detJ;
    T tmp1 = (xvel[0] - xvel[6]), tmp2 = (xvel[1] - xvel[7]);
    T tmp3 = (xvel[2] - xvel[4]), tmp4 = (xvel[3] - xvel[5]);
    d[0] = inv_detJ * (b[0][0] * tmp1 + b[0][1] * tmp2 + b[0][2] * tmp3 + b[0][3] * tmp4);
    tmp1 = (yvel[0] - yvel[6]);
    tmp2 = (yvel[1] - yvel[7]);
    tmp3 = (yvel[2] - yvel[4]);
    tmp4 = (yvel[3] - yvel[5]);
    d[1] = inv_detJ * (b[1][0] * tmp1 + b[1][1] * tmp2 + b[1][2] * tmp3 + b[1][3] * tmp4);
    tmp1 = (zvel[0] - zvel[6]);
    tmp2 = (zvel[1] - zvel[7]);
    tmp3 = (zvel[2] - zvel[4]);
    tmp4 = (zvel[3] - zvel[5]);
    d[2] = inv_detJ * (b[2][0] * tmp1 + b[2][1] * tmp2 + b[2][2] * tmp3 + b[2][3] * tmp4);
}

// CalcMonoGradient, lulesh.cu:3251-3334
template <typename T>
__device__ __forceinline__ void mono_gradient(const T x[8], const T y[8], const T z[8],
                                              const T xv[8], const T yv[8], const T zv[8],
                                              T vol, T *delx_zeta, T *delv_zeta, T *delx_xi,
                                              T *delv_xi, T *delx_eta, T *delv_eta)
{
#define LULESH_SUM4(a, b, c, d) (a + b + c + d)
    const T ptiny = T(1.e-36);
    T ax, ay, az, dxv, dyv, dzv;
    const T norm = T(1.0) / (vol + ptiny);
    const T dxj = T(-0.25) * (LULESH_SUM4(x[0], x[1], x[5], x[4]) - LULESH_SUM4(x[3], x[2], x[6], x[7]));
    const T dyj = T(-0.25) * (LULESH_SUM4(y[0], y[1], y[5], y[4]) - LULESH_SUM4(y[3], y[2], y[6], y[7]));
    const T dzj = T(-0.25) * (LULESH_SUM4(z[0], z[1], z[5], z[4]) - LULESH_SUM4(z[3], z[2], z[6], z[7]));
    const T dxi = T(0.25) * (LULESH_SUM4(x[1], x[2], x[6], x[5]) - LULESH_SUM4(x[0], x[3], x[7], x[4]));
    const T dyi = T(0.25) * (LULESH_SUM4(y[1], y[2], y[6], y[5]) - LULESH_SUM4(y[0], y[3], y[7], y[4]));
    const T dzi = T(0.25) * (LULESH_SUM4(z[1], z[2], z[6], z[5]) - LULESH_SUM4(z[0], z[3], z[7], z[4]));
    const T dxk = T(0.25) * (LULESH_SUM4(x[4], x[5], x[6], x[7]) - LULESH_SUM4(x[0], x[1], x[2], x[3]));
    const T dyk = T(0.25) * (LULESH_SUM4(y[4], y[5], y[6], y[7]) - LULESH_SUM4(y[0], y[1], y[2], y[3]));
    const T dzk = T(0.25) * (LULESH_SUM4(z[4], z[5], z[6], z[7]) - LULESH_SUM4(z[0], z[1], z[2], z[3]));

    // zeta: i cross j
    ax = dyi * dzj - dzi * dyj;
    ay = dzi * dxj - dxi * dzj;
    az = dxi * dyj - dyi * dxj;
    *delx_zeta = vol / sqrt_t(ax * ax + ay * ay + az * az + ptiny);
    ax *= norm;
    ay *= norm;
    az *= norm;
    dxv = T(0.25) * (LULESH_SUM4(xv[4], xv[5], xv[6], xv[7]) - LULESH_SUM4(xv[0], xv[1], xv[2], xv[3]));
    dyv = T(0.25) * (LULESH_SUM4(yv[4], yv[5], yv[6], yv[7]) - LULESH_SUM4(yv[0], yv[1], yv[2], yv[3]));
    dzv = T(0.25) * (LULESH_SUM4(zv[4], zv[5], zv[6], zv[7]) - LULESH_SUM4(zv[0], zv[1], zv[2], zv[3]));
    *delv_zeta = ax * dxv + ay * dyv + az * dzv;

    // xi: j cross k
    ax = dyj * dzk - dzj * dyk;
    ay = dzj * dxk - dxj * dzk;
    az = dxj * dyk - dyj * dxk;
    *delx_xi = vol / sqrt_t(ax * ax + ay * ay + az * az + ptiny);
    ax *= norm;
    ay *= norm;
    az *= norm;
    dxv = T(0.25) * (LULESH_SUM4(xv[1], xv[2], xv[6], xv[5]) - LULESH_SUM4(xv[0], xv[3], xv[7], xv[4]));
    dyv = T(0.25) * (LULESH_SUM4(yv[1], yv[2], yv[6], yv[5]) - LULESH_SUM4(yv[0], yv[3], yv[7], yv[4]));
    dzv = T(0.25) * (LULESH_SUM4(zv[1], zv[2], zv[6], zv[5]) - LULESH_SUM4(zv[0], zv[3], zv[7], zv[4]));
    *delv_xi = ax * dxv + ay * dyv + az * dzv;

    // eta: k cross i
    ax = dyk * dzi - dzk * dyi;
    ay = dzk * dxi - dxk * dzi;
    az = dxk * dyi - dyk * dxi;
    *delx_eta = vol / sqrt_t(ax * ax + ay * ay + az * az + ptiny);
    ax *= norm;
    ay *= norm;
    az *= norm;
    dxv = T(-0.25) * (LULESH_SUM4(xv[0], xv[1], xv[5], xv[4]) - LULESH_SUM4(xv[3], xv[2], xv[6], xv[7]));
    dyv = T(-0.25) * (LULESH_SUM4(yv[0], yv[1], yv[5], yv[4]) - LULESH_SUM4(yv[3], yv[2], yv[6], yv[7]));
    dzv = T(-0.25) * (LULESH_SUM4(zv[0], zv[1], zv[5], zv[4]) - LULESH_SUM4(zv[3], zv[2], zv[6], zv[7]));
    *delv_eta = ax * dxv + ay * dyv + az * dzv;
#undef LULESH_SUM4
}

}  // namespace lulesh
