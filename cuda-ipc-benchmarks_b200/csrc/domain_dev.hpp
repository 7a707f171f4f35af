// domain_dev.hpp -- device memory of one domain: sizing, carving, upload.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "host_setup.hpp"
#include "lulesh_b200.h"
#include "lulesh_dev.h"

namespace lulesh {

struct DomSizes {
    size_t E, N, Ep, allElem, corner, en2, nr, comm;
    bool unstructured = false;  // adds the per-node boundary mask
    bool ell = false;           // adds the slot-major corner runs (8 per node)
};

DomSizes sizes_of(int nx, int numReg, long comm_doubles);
// sizes of a host-built domain (structured or read from an lmesh file)
DomSizes sizes_of(const HostDomain &h, long comm_doubles);
size_t align256(size_t b);
// device bytes of one domain (all of its arrays at 256-byte alignment)
size_t domain_bytes(const DomSizes &s, bool mixed);
// receive-buffer doubles of a rank in a tp^3 decomposition (0 for tp = 1)
long comm_buffer_doubles(int nx, int tp);

// Hands out consecutive 256-byte-aligned pieces of one allocation.
struct Carver {
    char *base;
    size_t off = 0;
    template <typename T> T *take(size_t count)
    {
        T *p = reinterpret_cast<T *>(base + off);
        off += align256(sizeof(T) * count);
        return p;
    }
};

// Carve every array of host domain `h` from `cv`, initialise and upload it
// on `st`, and fill the device record *D (and *c32 when mixed).  `tc` is
// the TimeCtl slot of the domain's job.  Synchronises `st` before
// returning, so `h` may be released afterwards.
// With node_cv, x, y, z, xd, yd and zd come from node_cv (a set's node
// region: every domain's six arrays one after the other) and cv carves the
// rest; cv then advances by node_region_bytes(...) less than domain_bytes.
int upload_domain(const HostDomain &h, int tc, long comm_doubles, bool mixed, Carver &cv,
                  cudaStream_t st, DomDev *D, CornerF32 *c32, Carver *node_cv = nullptr);

// bytes of x, y, z, xd, yd, zd of a domain of `numNode` nodes, as carved
size_t node_region_bytes(size_t numNode);

// Write the geometry and connectivity arrays of single domain D (tp = 1) on
// the device (setup.cu), with the values build_domain computes on the
// host; e[0] = einit.  Asynchronous on `st`.
int setup_geometry_on_device(const DomDev &D, double einit, cudaStream_t st);

// Write regNumList, regElemlist and eosOrder of single domain D from its
// region runs (region_runs.hpp), staging the runs in D.fx_elem and zeroing
// them there again afterwards.  Asynchronous on `st`: `runs` must live until
// the stream has passed the upload.
int setup_regions_on_device(const DomDev &D, const std::vector<RegionRun> &runs,
                            cudaStream_t st);

// The time state of a job before its first cycle (lulesh.cu:1120-1132).
TimeCtl initial_timectl(double deltatime, int its_cap);

}  // namespace lulesh
