// domain_dev.cu -- device memory of one domain: sizing, carving, upload.
#include <climits>
#include <cstring>
#include <vector>

#include "domain_dev.hpp"
#include "set.hpp"

namespace lulesh {

DomSizes sizes_of(int nx, int numReg, long comm_doubles)
{
    DomSizes s;
    s.E = (size_t)nx * nx * nx;
    s.N = (size_t)(nx + 1) * (nx + 1) * (nx + 1);
    s.Ep = ((s.E + 31) / 32) * 32;
    s.allElem = s.E + 6 * (size_t)nx * nx;
    s.corner = 8 * s.E;
    s.en2 = (size_t)(nx + 1) * (nx + 1);
    s.nr = (size_t)numReg;
    s.comm = (size_t)comm_doubles;
    return s;
}

DomSizes sizes_of(const HostDomain &h, long comm_doubles)
{
    if (!h.unstructured) return sizes_of(h.nx, h.numReg, comm_doubles);
    DomSizes s;
    s.E = (size_t)h.numElem;
    s.N = (size_t)h.numNode;
    s.Ep = (size_t)h.Ep;
    s.allElem = s.E;
    s.corner = 8 * s.E;
    s.en2 = h.symmX.size();
    s.nr = (size_t)h.numReg;
    s.comm = 0;
    s.unstructured = true;
    s.ell = !h.nodeCornerEll.empty();
    return s;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t domain_bytes(const DomSizes &s, bool mixed)
{
    size_t b = 0;
    b += 16 * align256(8 * s.E);        // element doubles incl. vnew, delx_*
    b += 3 * align256(8 * s.allElem);   // delv_* with ghost faces
    b += 13 * align256(8 * s.N);        // node doubles
    b += 3 * align256(8 * 8 * s.Ep);    // corner forces
    b += align256(4 * 8 * s.Ep);        // nodelist
    b += 11 * align256(4 * s.E);        // l*, elemBC, matElemlist, regNumList, regElemlist, eosOrder
    b += 2 * align256(4 * s.N);         // nodeElemCount/Start
    b += align256(4 * s.corner);        // nodeElemCornerList
    b += 3 * align256(4 * s.en2);       // symm*
    b += 3 * align256(4 * s.nr);        // regCSR, regReps, regSorted
    if (s.comm) b += align256(8 * s.comm);
    if (mixed) b += 3 * align256(4 * 8 * s.Ep);
    if (s.unstructured) b += align256(4 * s.N);  // nodeBC
    if (s.ell) b += align256(4 * 8 * s.N);       // nodeCornerEll
    return b;
}

// receive-buffer capacity of SetupCommBuffers, lulesh.cu:457-510, for a
// domain with all 26 neighbours (the worst case every rank is sized for)
long comm_buffer_doubles(int nx, int tp)
{
    if (tp <= 1) return 0;
    const long pad = 16;  // CACHE_COHERENCE_PAD_REAL for doubles
    const long edge = nx + 1;
    const long maxPlane = ((edge * edge + pad - 1) / pad) * pad;
    return 6 * maxPlane * 6 + 12 * maxPlane * 6 + 8 * pad;
}

template <typename T>
static int upload(T *dst, const std::vector<T> &src, cudaStream_t s)
{
    if (src.empty()) return LULESH_OK;
    return cuda_status(cudaMemcpyAsync(dst, src.data(), sizeof(T) * src.size(),
                                       cudaMemcpyHostToDevice, s),
                       "upload");
}

#define DCHECK(call)                                            \
    do {                                                        \
        int _st = cuda_status((call), #call);                   \
        if (_st != LULESH_OK) return _st;                       \
    } while (0)

size_t node_region_bytes(size_t numNode) { return 6 * align256(8 * numNode); }

int upload_domain(const HostDomain &h, int tc, long comm_doubles, bool mixed, Carver &cv,
                  cudaStream_t st, DomDev *out, CornerF32 *c32, Carver *node_cv)
{
    const DomSizes z = sizes_of(h, comm_doubles);
    DomDev D{};
    D.nx = h.nx;
    D.en = h.nx + 1;
    D.numElem = h.numElem;
    D.numNode = h.numNode;
    D.Ep = h.Ep;
    D.allElem = h.allElem;
    D.col = h.col;
    D.row = h.row;
    D.plane = h.plane;
    D.tp = h.tp;
    D.tc = tc;
    D.numReg = h.numReg;
    D.numSymmX = h.numSymmX;
    D.numSymmY = h.numSymmY;
    D.numSymmZ = h.numSymmZ;
    for (int f = 0; f < 6; ++f) D.ghost[f] = h.ghost[f];
    for (int k = 0; k < 27; ++k) D.nbr[k] = -1;
    // element doubles
    D.e = cv.take<double>(z.E); D.p = cv.take<double>(z.E); D.q = cv.take<double>(z.E);
    D.ql = cv.take<double>(z.E); D.qq = cv.take<double>(z.E); D.v = cv.take<double>(z.E);
    D.volo = cv.take<double>(z.E); D.delv = cv.take<double>(z.E);
    D.vdov = cv.take<double>(z.E); D.arealg = cv.take<double>(z.E);
    D.ss = cv.take<double>(z.E); D.elemMass = cv.take<double>(z.E);
    D.vnew = cv.take<double>(z.E); D.delx_xi = cv.take<double>(z.E);
    D.delx_eta = cv.take<double>(z.E); D.delx_zeta = cv.take<double>(z.E);
    D.delv_xi = cv.take<double>(z.allElem); D.delv_eta = cv.take<double>(z.allElem);
    D.delv_zeta = cv.take<double>(z.allElem);
    // node doubles
    Carver &ncv = node_cv ? *node_cv : cv;
    D.x = ncv.take<double>(z.N); D.y = ncv.take<double>(z.N); D.z = ncv.take<double>(z.N);
    D.xd = ncv.take<double>(z.N); D.yd = ncv.take<double>(z.N); D.zd = ncv.take<double>(z.N);
    D.xdd = cv.take<double>(z.N); D.ydd = cv.take<double>(z.N); D.zdd = cv.take<double>(z.N);
    D.fx = cv.take<double>(z.N); D.fy = cv.take<double>(z.N); D.fz = cv.take<double>(z.N);
    D.nodalMass = cv.take<double>(z.N);
    D.fx_elem = cv.take<double>(8 * z.Ep); D.fy_elem = cv.take<double>(8 * z.Ep);
    D.fz_elem = cv.take<double>(8 * z.Ep);
    // ints
    D.nodelist = cv.take<int>(8 * z.Ep);
    D.lxim = cv.take<int>(z.E); D.lxip = cv.take<int>(z.E); D.letam = cv.take<int>(z.E);
    D.letap = cv.take<int>(z.E); D.lzetam = cv.take<int>(z.E); D.lzetap = cv.take<int>(z.E);
    D.elemBC = cv.take<int>(z.E); D.matElemlist = cv.take<int>(z.E);
    D.regNumList = cv.take<int>(z.E); D.regElemlist = cv.take<int>(z.E);
    D.eosOrder = cv.take<int>(z.E);
    D.eosNumClass = h.eosNumClass;
    for (int c = 0; c < kMaxRepClasses; ++c) {
        D.eosClassEnd[c] = h.eosClassEnd[c];
        D.eosClassRep[c] = h.eosClassRep[c];
    }
    D.nodeElemCount = cv.take<int>(z.N); D.nodeElemStart = cv.take<int>(z.N);
    D.nodeElemCornerList = cv.take<int>(z.corner);
    D.symmX = cv.take<int>(z.en2); D.symmY = cv.take<int>(z.en2); D.symmZ = cv.take<int>(z.en2);
    D.regCSR = cv.take<int>(z.nr); D.regReps = cv.take<int>(z.nr); D.regSorted = cv.take<int>(z.nr);
    if (z.comm) {
        D.commRecv = cv.take<double>(z.comm);
        D.commRecvLen = (long)z.comm;
    }
    D.unstructured = h.unstructured ? 1 : 0;
    D.octant = h.octantCorner;
    if (h.unstructured) D.nodeBC = cv.take<int>(z.N);
    if (z.ell) D.nodeCornerEll = cv.take<int>(8 * z.N);
    if (mixed && c32) {
        c32->fx = cv.take<float>(8 * z.Ep);
        c32->fy = cv.take<float>(8 * z.Ep);
        c32->fz = cv.take<float>(8 * z.Ep);
    }

    // InitializeFields (lulesh.cu:432-451): zeros except v = 1
    const size_t E = z.E, N = z.N;
    double *edbl[16] = {D.e, D.p, D.q, D.ql, D.qq, D.v, D.volo, D.delv, D.vdov,
                        D.arealg, D.ss, D.elemMass, D.vnew, D.delx_xi, D.delx_eta,
                        D.delx_zeta};
    for (double *p : edbl) DCHECK(cudaMemsetAsync(p, 0, 8 * E, st));
    double *ndbl[13] = {D.x, D.y, D.z, D.xd, D.yd, D.zd, D.xdd, D.ydd, D.zdd,
                        D.fx, D.fy, D.fz, D.nodalMass};
    for (double *p : ndbl) DCHECK(cudaMemsetAsync(p, 0, 8 * N, st));
    DCHECK(cudaMemsetAsync(D.delv_xi, 0, 8 * z.allElem, st));
    DCHECK(cudaMemsetAsync(D.delv_eta, 0, 8 * z.allElem, st));
    DCHECK(cudaMemsetAsync(D.delv_zeta, 0, 8 * z.allElem, st));
    DCHECK(cudaMemsetAsync(D.fx_elem, 0, 8 * 8 * z.Ep, st));
    DCHECK(cudaMemsetAsync(D.fy_elem, 0, 8 * 8 * z.Ep, st));
    DCHECK(cudaMemsetAsync(D.fz_elem, 0, 8 * 8 * z.Ep, st));
    if (z.comm) DCHECK(cudaMemsetAsync(D.commRecv, 0, 8 * z.comm, st));
    int su;
    if (h.device_geometry) {
        // single domain: geometry and the per-element region arrays on the
        // device, the region tables from the host
        if ((su = setup_geometry_on_device(D, h.einit, st)) != LULESH_OK) return su;
        if ((su = setup_regions_on_device(D, h.regionRuns, st)) != LULESH_OK) return su;
        const std::vector<int> *rv[] = {&h.regCSR, &h.regReps, &h.regSorted};
        int *rp[] = {D.regCSR, D.regReps, D.regSorted};
        for (size_t k = 0; k < sizeof(rp) / sizeof(rp[0]); ++k)
            if ((su = upload(rp[k], *rv[k], st)) != LULESH_OK) return su;
        DCHECK(cudaStreamSynchronize(st));
        *out = D;
        return LULESH_OK;
    }
    std::vector<double> ones(E, 1.0);
    if ((su = upload(D.v, ones, st)) != LULESH_OK) return su;
    if ((su = upload(D.e, h.e, st)) != LULESH_OK) return su;
    if ((su = upload(D.volo, h.volo, st)) != LULESH_OK) return su;
    if ((su = upload(D.elemMass, h.elemMass, st)) != LULESH_OK) return su;
    if ((su = upload(D.x, h.x, st)) != LULESH_OK) return su;
    if ((su = upload(D.y, h.y, st)) != LULESH_OK) return su;
    if ((su = upload(D.z, h.z, st)) != LULESH_OK) return su;
    if ((su = upload(D.nodalMass, h.nodalMass, st)) != LULESH_OK) return su;
    if ((su = upload(D.nodelist, h.nodelist, st)) != LULESH_OK) return su;
    const std::vector<int> *iv[] = {&h.lxim, &h.lxip, &h.letam, &h.letap, &h.lzetam,
                                    &h.lzetap, &h.elemBC, &h.matElemlist, &h.regNumList,
                                    &h.regElemlist, &h.nodeElemCount, &h.nodeElemStart,
                                    &h.nodeElemCornerList, &h.symmX, &h.symmY, &h.symmZ,
                                    &h.regCSR, &h.regReps, &h.regSorted, &h.eosOrder};
    int *ip[] = {D.lxim, D.lxip, D.letam, D.letap, D.lzetam, D.lzetap, D.elemBC,
                 D.matElemlist, D.regNumList, D.regElemlist, D.nodeElemCount,
                 D.nodeElemStart, D.nodeElemCornerList, D.symmX, D.symmY, D.symmZ,
                 D.regCSR, D.regReps, D.regSorted, D.eosOrder};
    for (size_t k = 0; k < sizeof(ip) / sizeof(ip[0]); ++k)
        if ((su = upload(ip[k], *iv[k], st)) != LULESH_OK) return su;
    if (h.unstructured && (su = upload(D.nodeBC, h.nodeBC, st)) != LULESH_OK) return su;
    if (z.ell && (su = upload(D.nodeCornerEll, h.nodeCornerEll, st)) != LULESH_OK) return su;
    // the host vectors must outlive the asynchronous copies
    DCHECK(cudaStreamSynchronize(st));
    *out = D;
    return LULESH_OK;
}

TimeCtl initial_timectl(double deltatime, int its_cap)
{
    TimeCtl T;
    std::memset(&T, 0, sizeof T);
    T.time = 0.0;
    T.deltatime = deltatime;
    T.dtcourant = 1.0e+20;
    T.dthydro = 1.0e+20;
    const double big = 1.0e+20;
    std::memcpy(&T.min_courant, &big, sizeof big);
    std::memcpy(&T.min_hydro, &big, sizeof big);
    T.cycle = 0;
    T.its_cap = its_cap;
    T.bad_vol = INT_MAX;
    T.bad_q = INT_MAX;
    return T;
}

}  // namespace lulesh
