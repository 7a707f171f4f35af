// host_setup.hpp -- host-side construction of LULESH domains.
//
// Builds, on the host, every array NewDomain (LULESH/cuda/src/lulesh.cu:
// 750-1221) builds for the structured (-s) mesh, in the same order and with
// the same arithmetic, so the device arena can be filled with one copy per
// array.  Compiled without FMA contraction, like the reference's host code.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "lulesh_dev.h"
#include "region_runs.hpp"

namespace lulesh {

// glibc's rand()/srand() (TYPE_3 additive feedback generator, 31 words of
// state), restated so region sets match the reference's srand(rank)/rand()
// without touching the process-wide libc state.
class GlibcRand {
  public:
    explicit GlibcRand(unsigned seed);
    int next();  // same sequence as rand() after srand(seed)

  private:
    int32_t r_[34];
    int idx_;
};

struct HostDomain {
    int nx = 0, en = 0, numElem = 0, numNode = 0, Ep = 0, allElem = 0;
    int tp = 1, col = 0, row = 0, plane = 0, rank = 0;
    int rowMin = 0, rowMax = 0, colMin = 0, colMax = 0, planeMin = 0, planeMax = 0;
    int numReg = 0, balance = 1, cost = 1;
    int numSymmX = 0, numSymmY = 0, numSymmZ = 0;
    int ghost[6] = {-1, -1, -1, -1, -1, -1};
    std::vector<int> nodelist, lxim, lxip, letam, letap, lzetam, lzetap, elemBC;
    std::vector<int> nodeElemCount, nodeElemStart, nodeElemCornerList;
    std::vector<int> symmX, symmY, symmZ, matElemlist;
    std::vector<int> regElemSize, regCSR, regReps, regNumList, regElemlist, regSorted;
    // EOS work order: elements grouped by their rep count (heaviest class
    // first), ascending element index inside a class; class c covers
    // positions [eosClassEnd[c-1], eosClassEnd[c]) and runs eosClassRep[c]
    std::vector<int> eosOrder;
    int eosNumClass = 0;
    int eosClassEnd[kMaxRepClasses] = {0};
    int eosClassRep[kMaxRepClasses] = {0};
    std::vector<double> x, y, z, volo, elemMass, nodalMass, e;
    double einit = 0.0;
    double deltatime = 0.0;  // initial dt of this domain, lulesh.cu:1205
    // geometry and connectivity left to the device (build_domain_light):
    // the vectors from nodelist to nodalMass above are empty, and so are
    // regNumList, regElemlist and eosOrder, which the device writes from
    // the region runs (region_runs.hpp); the other region tables are full
    bool device_geometry = false;
    std::vector<RegionRun> regionRuns;
    // read from an lmesh file (build_domain_lmesh)
    bool unstructured = false;
    int octantCorner = 0;
    std::vector<int> nodeBC;  // per node: bit 0/1/2 = in symmX/Y/Z
    // when no node has more than 8 corners: slot j of node i's corner run at
    // [j * numNode + i], -1 past the run (empty otherwise)
    std::vector<int> nodeCornerEll;
};

// Reference parameter block, lulesh.cu:1125-1158.
Params default_params();

// Build one domain of a tp^3 decomposition at (col,row,plane).
// `global_mass` computes nodalMass as the single-domain sum over the
// problem's elements in ascending global index (what the reference's
// single-rank run produces); otherwise only this domain's elements
// contribute (what each rank holds before the init-time CommSBN).
void build_domain(HostDomain &d, int nx, int tp, int col, int row, int plane,
                  int rank, int numReg, int balance, int cost, bool global_mass);

// A single (tp = 1) domain with only what must come from the host: the
// scalars, the energy deposit and initial dt, and the region sets drawn
// from glibc rand, as runs (regionRuns) with the per-region and per-class
// tables.  The geometry, the connectivity and the per-element region
// arrays are generated on the device (setup.cu) with the same values
// build_domain computes.
void build_domain_light(HostDomain &d, int nx, int numReg, int balance, int cost);

// An unstructured domain from an lmesh file, the format the reference reads
// with -u (lulesh.cu:855-1052): "numElem numNode", the node coordinates, 8
// node ids per element, 6 face neighbours per element (xi-, xi+, eta-,
// eta+, zeta-, zeta+), then the X, Y, Z symmetry node sets and the free
// surface node set, each as a count followed by the ids.  Boundary masks
// follow the reference's face tests on those sets, with one correction:
// faces on the free surface get the *_FREE bits (the reference's reader
// marks them *_SYMM, lulesh.cu:1039-1044).  The energy 3.948746e7 goes to
// the octant corner (the first element with all three minimum faces on
// symmetry planes, lulesh.cu:1015-1022) and the initial dt follows from
// that element's volume.  Returns false with *err set on a malformed file.
bool build_domain_lmesh(HostDomain &d, const char *path, int numReg, int balance, int cost,
                        std::string *err);

// The initial dt of a tp^3 problem of nx^3 subdomains: that of the domain
// holding the origin (lulesh.cu:1189-1205), which every subdomain starts
// from.
double origin_deltatime(int nx, int tp);

// CalcElemVolume (lulesh.cu:221-307), host copy used at setup.
double elem_volume_host(const double *x, const double *y, const double *z);

}  // namespace lulesh
