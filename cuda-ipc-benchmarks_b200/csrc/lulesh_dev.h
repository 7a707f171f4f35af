// lulesh_dev.h -- device-side layout of a set of LULESH domains on one B200.
//
// Every domain keeps the reference Domain's SoA fields (LULESH/cuda/src/
// lulesh.h:40-298) as plain device arrays carved out of one arena; kernels
// see a table of DomDev records (one per domain) plus a table of TimeCtl
// records (one per independent problem: a single domain, the tp^3
// subdomains of one decomposed problem, or one job of a batch).
#pragma once

#include <cstdint>

namespace lulesh {

// element-face boundary-condition bits, lulesh.cu:151-181
enum : int {
    XI_M = 0x00007, XI_M_SYMM = 0x00001, XI_M_FREE = 0x00002, XI_M_COMM = 0x00004,
    XI_P = 0x00038, XI_P_SYMM = 0x00008, XI_P_FREE = 0x00010, XI_P_COMM = 0x00020,
    ETA_M = 0x001c0, ETA_M_SYMM = 0x00040, ETA_M_FREE = 0x00080, ETA_M_COMM = 0x00100,
    ETA_P = 0x00e00, ETA_P_SYMM = 0x00200, ETA_P_FREE = 0x00400, ETA_P_COMM = 0x00800,
    ZETA_M = 0x07000, ZETA_M_SYMM = 0x01000, ZETA_M_FREE = 0x02000, ZETA_M_COMM = 0x04000,
    ZETA_P = 0x38000, ZETA_P_SYMM = 0x08000, ZETA_P_FREE = 0x10000, ZETA_P_COMM = 0x20000
};

// Distinct EOS rep counts a domain can have: 1, 1+cost, 10*(1+cost)
// (CreateRegionIndexSets, lulesh.cu:1364-1374).
constexpr int kMaxRepClasses = 4;

// Material / control parameters of NewDomain, lulesh.cu:1125-1158.
struct Params {
    double dtfixed, deltatimemultlb, deltatimemultub, stoptime, dtmax;
    double e_cut, p_cut, q_cut, u_cut, v_cut;
    double hgcoef, ss4o3, qstop, monoq_max_slope, monoq_limiter_mult;
    double qlc_monoq, qqc_monoq, qqc, pmin, emin, dvovmax, eosvmax, eosvmin,
        refdens;
};

// Device-resident time state of one problem (replaces the host scalars
// time_h/deltatime_h/cycle and the pinned dtcourant_h/dthydro_h/bad_*_h of
// lulesh.h:171-187).  Written only by the time-increment kernel and by
// atomics of the element kernels; read by every kernel.
struct TimeCtl {
    double time, deltatime, dtcourant, dthydro;
    unsigned long long min_courant;  // bit pattern of the running minimum
    unsigned long long min_hydro;    // (positive doubles order like uint64)
    int cycle;       // cycles started
    int its_cap;     // -i; <= 0 means none
    int active;      // 1 while this cycle's kernels must run
    int done;        // 1 once the job stopped (time, its, or error)
    int bad_vol;     // smallest element index with a volume error, INT_MAX
    int bad_q;       // smallest element index with q > qstop, INT_MAX
    int status;      // lulesh_status of the job
    int chk;         // checked builds: code of the first index out of range, 0 none
};

// One domain.  Sizes follow lulesh.cu:783-798; node (px,py,pz) has index
// (pz*en + py)*en + px and element (ix,iy,iz) index (iz*nx + iy)*nx + ix,
// exactly the order BuildMesh (lulesh.cu:688-747) produces.
struct DomDev {
    int nx, en, numElem, numNode, Ep, allElem;
    int col, row, plane, tp;
    int tc;        // TimeCtl index
    int numReg;
    int nbr[27];   // domain index of the neighbour at (dx,dy,dz)+1 (x fastest), -1 none
    int ghost[6];  // ghost-face offsets into delv_* (SetupConnectivityBC order), -1 none
    // element fields
    double *e, *p, *q, *ql, *qq, *v, *volo, *delv, *vdov, *arealg, *ss, *elemMass;
    // node fields
    double *x, *y, *z, *xd, *yd, *zd, *xdd, *ydd, *zdd, *fx, *fy, *fz, *nodalMass;
    // per-cycle temporaries
    double *vnew, *delx_xi, *delx_eta, *delx_zeta, *delv_xi, *delv_eta, *delv_zeta;
    double *fx_elem, *fy_elem, *fz_elem;  // corner forces [8][Ep]
    // connectivity (reference layout)
    int *nodelist, *lxim, *lxip, *letam, *letap, *lzetam, *lzetap, *elemBC;
    int *nodeElemCount, *nodeElemStart, *nodeElemCornerList;
    int *symmX, *symmY, *symmZ, *matElemlist;
    int *regCSR, *regReps, *regNumList, *regElemlist, *regSorted;
    int numSymmX, numSymmY, numSymmZ;
    // EOS work order (see HostDomain::eosOrder)
    int *eosOrder;
    int eosNumClass;
    int eosClassEnd[kMaxRepClasses];
    int eosClassRep[kMaxRepClasses];
    // comm message buffers (staged exchange): receive buffer of this rank
    double *commRecv;
    long commRecvLen;
    // unstructured (lmesh) domains: kernels read nodelist, the corner CSR,
    // the face links and elemBC instead of computing them from the element
    // position; nodeBC[n] has bit 0/1/2 set when node n is in symmX/Y/Z
    int unstructured;
    int octant;  // element holding the energy deposit (0 on -s meshes)
    int *nodeBC;
    // slot j of node i's corner run at [j * numNode + i], -1 past the run;
    // null when some node has more than 8 corners (the kernel then reads the
    // run from nodeElemCornerList)
    int *nodeCornerEll;
};

// Mixed-precision corner forces, FP32, layout of fx_elem ([8][Ep]).
struct CornerF32 {
    float *fx, *fy, *fz;
};

}  // namespace lulesh
