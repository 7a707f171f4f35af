// setup.cu -- the geometry and connectivity of a single structured domain,
// generated on the device.
//
// NewDomain (LULESH/cuda/src/lulesh.cu:750-1221) builds these arrays on the
// host and copies them to the GPU: about 600 bytes per element.  For a
// single domain (tp = 1) every one of them is a closed-form function of the
// element or node position, so two kernels write them in place.  The
// region sets are drawn from glibc rand on the host, but only as runs of
// elements (region_runs.hpp); a third kernel writes regNumList,
// regElemlist and the EOS order from them.  The values are those of the
// host builder, bit for bit:
//   * this file is compiled with -fmad=false: the volume and coordinate
//     arithmetic is not contracted into FMAs, like the reference's host code;
//   * every expression keeps the host builder's operand order;
//   * the nodal mass adds its elements' volume/8 in ascending element index,
//     the order of the reference's element loop.
#include "domain_dev.hpp"
#include "set.hpp"

namespace lulesh {

namespace {

__device__ __forceinline__ double lattice_d(int g, int edge)
{
    return 1.125 * (double)g / (double)edge;  // BuildMesh, lulesh.cu:698-715
}

__device__ __forceinline__ double triple_d(double a1, double b1, double c1, double a2,
                                           double b2, double c2, double a3, double b3,
                                           double c3)
{
    return a1 * (b2 * c3 - c2 * b3) + a2 * (c1 * b3 - b1 * c3) + a3 * (b1 * c2 - c1 * b2);
}

// CalcElemVolume (lulesh.cu:221-307), the expression of elem_volume_host
__device__ double elem_volume_d(const double *x, const double *y, const double *z)
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
    double vol = triple_d(dx31 + dx72, dx63, dx20, dy31 + dy72, dy63, dy20, dz31 + dz72, dz63,
                          dz20) +
                 triple_d(dx43 + dx57, dx64, dx70, dy43 + dy57, dy64, dy70, dz43 + dz57, dz64,
                          dz70) +
                 triple_d(dx14 + dx25, dx61, dx50, dy14 + dy25, dy61, dy50, dz14 + dz25, dz61,
                          dz50);
    vol *= twelveth;
    return vol;
}

// corner k of an element sits at (x: bit k of 0x66, y: 0xCC, z: 0xF0)
__device__ __forceinline__ int cx(int k) { return (0x66 >> k) & 1; }
__device__ __forceinline__ int cy(int k) { return (0xCC >> k) & 1; }
__device__ __forceinline__ int cz(int k) { return (0xF0 >> k) & 1; }

// elements adjacent to lattice coordinate p along one axis, and their
// prefix sum over coordinates below k (nodeElemStart in closed form)
__device__ __forceinline__ int adj(int p, int nx) { return (p > 0) + (p < nx); }
__device__ __forceinline__ int adj_below(int k) { return k == 0 ? 0 : 2 * k - 1; }

// Per element: nodelist, face links, boundary mask, material list, volume,
// mass, relative volume 1, and the energy deposit (lulesh.cu:537-686,
// 722-744, 1108-1205).
__global__ void k_setup_elems(DomDev D, double einit)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = D.nx, en = D.en, E = D.numElem, Ep = D.Ep, nn = nx * nx;
    if (i >= E) return;
    const int ix = i % nx, t = i / nx, iy = t % nx, iz = t / nx;
    const int n0 = (iz * en + iy) * en + ix;
    double xl[8], yl[8], zl[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        D.nodelist[(size_t)k * Ep + i] = n0 + cx(k) + cy(k) * en + cz(k) * en * en;
        xl[k] = lattice_d(ix + cx(k), nx);
        yl[k] = lattice_d(iy + cy(k), nx);
        zl[k] = lattice_d(iz + cz(k), nx);
    }
    // the host builder's links: the linear neighbour, the element itself at
    // the mesh's first/last index (overwritten only for comm faces, none here)
    D.lxim[i] = (i == 0) ? 0 : i - 1;
    D.lxip[i] = (i == E - 1) ? E - 1 : i + 1;
    D.letam[i] = (i < nx) ? i : i - nx;
    D.letap[i] = (i >= E - nx) ? i : i + nx;
    D.lzetam[i] = (i < nn) ? i : i - nn;
    D.lzetap[i] = (i >= E - nn) ? i : i + nn;
    int bc = 0;
    if (iz == 0) bc |= ZETA_M_SYMM;
    if (iz == nx - 1) bc |= ZETA_P_FREE;
    if (iy == 0) bc |= ETA_M_SYMM;
    if (iy == nx - 1) bc |= ETA_P_FREE;
    if (ix == 0) bc |= XI_M_SYMM;
    if (ix == nx - 1) bc |= XI_P_FREE;
    D.elemBC[i] = bc;
    D.matElemlist[i] = i;
    const double vol = elem_volume_d(xl, yl, zl);
    D.volo[i] = vol;
    D.elemMass[i] = vol;
    D.v[i] = 1.0;
    if (i == 0) D.e[0] = einit;
}

// Per node: coordinates, corner CSR (outer corner j, as lulesh.cu:1079-1088
// orders it), nodal mass, and the symmetry node sets (lulesh.cu:809-851).
// Runs after k_setup_elems (it reads volo).
__global__ void k_setup_nodes(DomDev D)
{
    const int n = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx = D.nx, en = D.en, Ep = D.Ep;
    if (n >= D.numNode) return;
    const int px = n % en, t = n / en, py = t % en, pz = t / en;
    D.x[n] = lattice_d(px, nx);
    D.y[n] = lattice_d(py, nx);
    D.z[n] = lattice_d(pz, nx);
    const int A = 2 * nx;  // elements along one axis summed over all coordinates
    const int start = adj_below(pz) * A * A + adj(pz, nx) * adj_below(py) * A +
                      adj(pz, nx) * adj(py, nx) * adj_below(px);
    D.nodeElemStart[n] = start;
    D.nodeElemCount[n] = adj(px, nx) * adj(py, nx) * adj(pz, nx);
    int r = 0;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int ex = px - cx(j), ey = py - cy(j), ez = pz - cz(j);
        if (ex >= 0 && ey >= 0 && ez >= 0 && ex < nx && ey < nx && ez < nx)
            D.nodeElemCornerList[start + r++] = Ep * j + (ez * nx + ey) * nx + ex;
    }
    double m = 0.0;
    for (int ez = pz - 1; ez <= pz; ++ez)
        for (int ey = py - 1; ey <= py; ++ey)
            for (int ex = px - 1; ex <= px; ++ex)
                if (ex >= 0 && ey >= 0 && ez >= 0 && ex < nx && ey < nx && ez < nx)
                    m += D.volo[(ez * nx + ey) * nx + ex] / 8.0;
    D.nodalMass[n] = m;
    if (n < en * en) {
        const int i = n / en, j = n % en;
        D.symmZ[n] = n;
        D.symmY[n] = i * en * en + j;
        D.symmX[n] = i * en * en + j * en;
    }
}

// The init-time nodal mass exchange of a decomposed problem (CommRecv/
// CommSend/CommSBN of nodalMass, lulesh.cu:4811-4831) as a gather: every
// node of every subdomain adds volume/8 of the elements touching it over
// the whole problem, in ascending global element index (the single-domain
// element loop of lulesh.cu:1165-1187), reading an element of a
// neighbouring subdomain from that subdomain (or its proxy, whose volo the
// MASS messages filled).  The sum then equals the single-domain nodal mass
// bit for bit, where the reference's exchange of partial sums differs in
// the last bits.  An element outside the mesh has no neighbour (nbr -1).
__global__ void k_nodal_mass(const DomDev *doms, const int2 *blocks)
{
    const int2 blk = blocks[blockIdx.x];
    const DomDev &D = doms[blk.x];
    const int n = blk.y + threadIdx.x;
    if (n >= D.numNode) return;
    const int nx = D.nx, en = D.en;
    const int px = n % en, t = n / en, py = t % en, pz = t / en;
    double m = 0.0;
    for (int ez = pz - 1; ez <= pz; ++ez)
        for (int ey = py - 1; ey <= py; ++ey)
            for (int ex = px - 1; ex <= px; ++ex) {
                const int sx = ex < 0 ? -1 : (ex >= nx ? 1 : 0);
                const int sy = ey < 0 ? -1 : (ey >= nx ? 1 : 0);
                const int sz = ez < 0 ? -1 : (ez >= nx ? 1 : 0);
                const double *volo = D.volo;
                if (sx | sy | sz) {
                    const int nb = D.nbr[(sx + 1) + 3 * (sy + 1) + 9 * (sz + 1)];
                    if (nb < 0) continue;
                    volo = doms[nb].volo;
                }
                m += volo[((ez - sz * nx) * nx + (ey - sy * nx)) * nx + (ex - sx * nx)] / 8.0;
            }
    D.nodalMass[n] = m;
}

// regNumList, regElemlist and the EOS order of a single domain from its
// region runs (CreateRegionIndexSets' fill, lulesh.cu:1343-1395): one
// thread per element.
__global__ void k_region_sets(const RegionRun *runs, int nruns, int E, int *regNumList,
                              int *regElemlist, int *eosOrder)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= E) return;
    expand_region_element(runs, nruns, i, regNumList, regElemlist, eosOrder);
}

}  // namespace

int setup_regions_on_device(const DomDev &D, const std::vector<RegionRun> &runs,
                            cudaStream_t st)
{
    // the runs are staged in fx_elem, which set-up zeroes and the first
    // force pass overwrites: every run holds at least one element, so the
    // table (16 B per run) fits in that array's 64 B per element
    const size_t bytes = sizeof(RegionRun) * runs.size();
    if (runs.size() > (size_t)D.numElem ||
        !region_runs_valid(runs.data(), (int)runs.size(), D.numElem)) {
        set_error("region runs do not cover the domain");
        return LULESH_INVALID_ARG;
    }
    RegionRun *staged = reinterpret_cast<RegionRun *>(D.fx_elem);
    cudaError_t e = cudaMemcpyAsync(staged, runs.data(), bytes, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_status(e, "region runs upload");
    const int b = 128;
    k_region_sets<<<(D.numElem + b - 1) / b, b, 0, st>>>(staged, (int)runs.size(), D.numElem,
                                                         D.regNumList, D.regElemlist,
                                                         D.eosOrder);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_status(e, "region sets kernel");
    return cuda_status(cudaMemsetAsync(staged, 0, bytes, st), "region runs clear");
}

int nodal_mass_on_device(lulesh_set *s)
{
    if (s->n_node_blocks == 0) return LULESH_OK;
    k_nodal_mass<<<s->n_node_blocks, s->nb, 0, s->stream>>>(s->ddoms, s->node_blocks);
    return cuda_status(cudaGetLastError(), "nodal mass");
}

int setup_geometry_on_device(const DomDev &D, double einit, cudaStream_t st)
{
    const int b = 128;
    // padding slots of nodelist (elements E..Ep) are zero on the host too
    cudaError_t e = cudaMemsetAsync(D.nodelist, 0, sizeof(int) * 8 * (size_t)D.Ep, st);
    if (e != cudaSuccess) return cuda_status(e, "setup memset");
    k_setup_elems<<<(D.numElem + b - 1) / b, b, 0, st>>>(D, einit);
    k_setup_nodes<<<(D.numNode + b - 1) / b, b, 0, st>>>(D);
    return cuda_status(cudaGetLastError(), "setup kernels");
}

}  // namespace lulesh
