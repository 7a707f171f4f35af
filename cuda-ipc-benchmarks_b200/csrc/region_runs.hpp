// region_runs.hpp -- a domain's region sets from the runs that
// CreateRegionIndexSets draws.
//
// CreateRegionIndexSets (LULESH/cuda/src/lulesh.cu:1259-1398) draws from
// glibc rand() a sequence of runs: consecutive elements that all get one
// region number.  Every per-element array it builds follows from those
// runs.  regNumList holds the run's region number; regElemlist lists the
// elements of each region (in sorted-region order) in ascending index; and
// the EOS work order lists the elements of each rep class in ascending
// index.  Once a run knows where its first element goes in regElemlist and
// in the EOS order, its k-th element goes k places further on in both.  So
// the host draws only the runs (about one per 38 elements), and the
// per-element arrays are written from them on the device (setup.cu) or on
// the host (the CPU tests), by the same function below.
#pragma once

#ifdef __CUDACC__
#define LULESH_HD __host__ __device__
#else
#define LULESH_HD
#endif

namespace lulesh {

struct RegionRun {
    int start;    // first element of the run
    int region;   // region number, 1-based (the regNumList value)
    int list_at;  // position of element `start` in regElemlist
    int eos_at;   // position of element `start` in the EOS order
};
static_assert(sizeof(RegionRun) == 16, "four ints per run");

// Element i's entries of regNumList, regElemlist and the EOS order.  The
// runs are sorted by start, runs[0].start == 0, and together they cover
// [0, E), so every element has exactly one run: the last one that starts
// at or before it.
LULESH_HD inline void expand_region_element(const RegionRun *runs, int nruns, int i,
                                            int *regNumList, int *regElemlist, int *eosOrder)
{
    int lo = 0, hi = nruns - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (runs[mid].start <= i)
            lo = mid;
        else
            hi = mid - 1;
    }
    const RegionRun r = runs[lo];
    const int k = i - r.start;
    regNumList[i] = r.region;
    regElemlist[r.list_at + k] = i;
    eosOrder[r.eos_at + k] = i;
}

// True when runs[0..nruns) cover [0, E) as expand_region_element expects
// and every write it makes stays inside the three E-element arrays: starts
// strictly increasing from 0, at most E runs, and each run's elements
// fitting in regElemlist and the EOS order from its two positions.  Checked
// on the host before the runs go to the device.
inline bool region_runs_valid(const RegionRun *runs, int nruns, int E)
{
    if (!runs || nruns < 1 || nruns > E || runs[0].start != 0) return false;
    for (int k = 0; k < nruns; ++k) {
        const int end = k + 1 < nruns ? runs[k + 1].start : E;
        if (end <= runs[k].start || end > E) return false;
        const int len = end - runs[k].start;
        if (runs[k].list_at < 0 || runs[k].list_at > E - len) return false;
        if (runs[k].eos_at < 0 || runs[k].eos_at > E - len) return false;
    }
    return true;
}

}  // namespace lulesh
