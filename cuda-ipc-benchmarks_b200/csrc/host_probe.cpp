// host_probe.cpp -- host-only entry points into the domain setup, built as
// liblulesh_host.so (no CUDA) so the CPU test suite can check the setup
// arithmetic and index layout against the oracle without a GPU.  Not part
// of the drop-in ABI (include/lulesh_b200.h).
#include <cstring>
#include <vector>

#include "host_setup.hpp"

extern "C" {

// The first n values of rand() after srand(seed).
void lulesh_host_rand(unsigned seed, int n, int *out)
{
    lulesh::GlibcRand r(seed);
    for (int i = 0; i < n; ++i) out[i] = r.next();
}

// Copy the named array of a built domain into out (capacity `cap` elements
// of the array's type); returns the array length, -1 if unknown.
static long copy_field(const lulesh::HostDomain &d, const char *name, void *out, long cap)
{
    struct I {
        const char *n;
        const std::vector<int> *v;
    } ints[] = {{"nodelist", &d.nodelist}, {"lxim", &d.lxim}, {"lxip", &d.lxip},
                {"letam", &d.letam}, {"letap", &d.letap}, {"lzetam", &d.lzetam},
                {"lzetap", &d.lzetap}, {"elemBC", &d.elemBC},
                {"nodeElemCount", &d.nodeElemCount}, {"nodeElemStart", &d.nodeElemStart},
                {"nodeElemCornerList", &d.nodeElemCornerList}, {"symmX", &d.symmX},
                {"symmY", &d.symmY}, {"symmZ", &d.symmZ}, {"matElemlist", &d.matElemlist},
                {"regElemSize", &d.regElemSize}, {"regCSR", &d.regCSR},
                {"regReps", &d.regReps}, {"regNumList", &d.regNumList},
                {"regElemlist", &d.regElemlist}, {"regSorted", &d.regSorted},
                {"nodeBC", &d.nodeBC}, {"nodeCornerEll", &d.nodeCornerEll},
                {"eosOrder", &d.eosOrder}};
    struct R {
        const char *n;
        const std::vector<double> *v;
    } reals[] = {{"x", &d.x}, {"y", &d.y}, {"z", &d.z}, {"volo", &d.volo},
                 {"elemMass", &d.elemMass}, {"nodalMass", &d.nodalMass}, {"e", &d.e}};
    for (const I &i : ints)
        if (!std::strcmp(i.n, name)) {
            long n = (long)i.v->size();
            if (out && cap >= n) std::memcpy(out, i.v->data(), sizeof(int) * n);
            return n;
        }
    for (const R &r : reals)
        if (!std::strcmp(r.n, name)) {
            long n = (long)r.v->size();
            if (out && cap >= n) std::memcpy(out, r.v->data(), sizeof(double) * n);
            return n;
        }
    if (!std::strcmp(name, "deltatime")) {
        if (out && cap >= 1) *(double *)out = d.deltatime;
        return 1;
    }
    if (!std::strcmp(name, "octant")) {
        if (out && cap >= 1) *(int *)out = d.octantCorner;
        return 1;
    }
    // the EOS rep classes: end position and rep count of each
    const int *cls = !std::strcmp(name, "eosClassEnd")   ? d.eosClassEnd
                     : !std::strcmp(name, "eosClassRep") ? d.eosClassRep
                                                         : nullptr;
    if (cls) {
        if (out && cap >= d.eosNumClass) std::memcpy(out, cls, sizeof(int) * d.eosNumClass);
        return d.eosNumClass;
    }
    return -1;
}

// Build one structured domain and copy the named array (copy_field).
long lulesh_host_domain_field(int nx, int tp, int col, int row, int plane, int rank,
                              int numReg, int balance, int cost, int global_mass,
                              const char *name, void *out, long cap)
{
    lulesh::HostDomain d;
    lulesh::build_domain(d, nx, tp, col, row, plane, rank, numReg, balance, cost,
                         global_mass != 0);
    return copy_field(d, name, out, cap);
}

// The light single-domain builder (build_domain_light: the region sets as
// runs), with regNumList, regElemlist and eosOrder then written from the
// runs on the host by expand_region_element, the function the device
// set-up kernel runs per element; "nruns" gives the number of runs.  Copies
// the named array as copy_field does.
long lulesh_host_light_field(int nx, int numReg, int balance, int cost, const char *name,
                             void *out, long cap)
{
    lulesh::HostDomain d;
    lulesh::build_domain_light(d, nx, numReg, balance, cost);
    if (!std::strcmp(name, "nruns")) {
        if (out && cap >= 1) *(long *)out = (long)d.regionRuns.size();
        return 1;
    }
    if (!std::strcmp(name, "runs")) {  // start, region, list_at, eos_at per run
        const long n = 4 * (long)d.regionRuns.size();
        if (out && cap >= n) std::memcpy(out, d.regionRuns.data(), sizeof(int) * n);
        return n;
    }
    const int E = d.numElem;
    d.regNumList.assign(E, -1);
    d.regElemlist.assign(E, -1);
    d.eosOrder.assign(E, -1);
    for (int i = 0; i < E; ++i)
        lulesh::expand_region_element(d.regionRuns.data(), (int)d.regionRuns.size(), i,
                                      d.regNumList.data(), d.regElemlist.data(),
                                      d.eosOrder.data());
    return copy_field(d, name, out, cap);
}

// region_runs_valid on a caller's table of nruns runs, four ints each
// (start, region, list_at, eos_at), over E elements: 1 valid, 0 not.
int lulesh_host_region_runs_valid(const int *runs4, int nruns, int E)
{
    std::vector<lulesh::RegionRun> runs(nruns > 0 ? nruns : 0);
    for (int k = 0; k < nruns; ++k)
        runs[k] = {runs4[4 * k], runs4[4 * k + 1], runs4[4 * k + 2], runs4[4 * k + 3]};
    return lulesh::region_runs_valid(runs.data(), nruns, E) ? 1 : 0;
}

// Read one domain from an lmesh file (lulesh_create_from_mesh's reader) and
// copy the named array; -2 if the file is unreadable or malformed.
long lulesh_host_lmesh_field(const char *path, int numReg, int balance, int cost,
                             const char *name, void *out, long cap)
{
    lulesh::HostDomain d;
    if (!lulesh::build_domain_lmesh(d, path, numReg, balance, cost, nullptr)) return -2;
    return copy_field(d, name, out, cap);
}

}  // extern "C"
