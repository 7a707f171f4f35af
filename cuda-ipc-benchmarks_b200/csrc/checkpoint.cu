// checkpoint.cu -- save and load the whole state of a set.
//
// All state a cycle reads or writes lives in two device allocations: the
// arena (every field of every domain, carved at fixed offsets from the
// set's jobs, tp and flags) and the array of per-job TimeCtl records.  A
// checkpoint is a header, the arena bytes and the TimeCtl bytes.  Loading
// it into a set built from the same description restores the state
// exactly, because the carving is deterministic.
#include <cstring>

#include "set.hpp"

namespace lulesh {

namespace {

constexpr unsigned kMagic = 0x4c554c43u;  // "LULC"
constexpr unsigned kVersion = 3;  // 3: subdomain sets carve x..zd first

struct CkptHeader {
    unsigned magic, version;
    int njobs, ndom, tp, flags;
    unsigned long long arena_bytes, tc_bytes;
    unsigned long long jobs_hash;  // FNV-1a of the job descriptions
    unsigned long long mesh_hash;  // an lmesh set's mesh (lulesh_set::mesh_hash)
    int nparts, part;              // a part of a problem split over GPUs
};

unsigned long long jobs_hash(const lulesh_set *s)
{
    unsigned long long h = 1469598103934665603ull;
    for (const lulesh_job &j : s->jobs) {
        const int v[5] = {j.nx, j.numReg, j.balance, j.cost, j.its};
        const unsigned char *p = reinterpret_cast<const unsigned char *>(v);
        for (size_t i = 0; i < sizeof v; ++i) h = (h ^ p[i]) * 1099511628211ull;
    }
    return h;
}

CkptHeader header_of(const lulesh_set *s)
{
    CkptHeader h{};
    h.magic = kMagic;
    h.version = kVersion;
    h.njobs = s->njobs;
    h.ndom = s->ndom;
    h.tp = s->tp;
    h.flags = s->flags;
    h.arena_bytes = s->arena_bytes;
    h.tc_bytes = sizeof(TimeCtl) * s->njobs;
    h.jobs_hash = jobs_hash(s);
    h.mesh_hash = s->mesh_hash;
    h.nparts = s->nparts;
    h.part = s->part;
    return h;
}

#define CCHECK(call)                                            \
    do {                                                        \
        int _st = cuda_status((call), #call);                   \
        if (_st != LULESH_OK) return _st;                       \
    } while (0)

}  // namespace
}  // namespace lulesh

using namespace lulesh;

extern "C" {

size_t lulesh_checkpoint_bytes(const lulesh_set *s)
{
    if (!s) return 0;
    return sizeof(CkptHeader) + s->arena_bytes + sizeof(TimeCtl) * s->njobs;
}

int lulesh_checkpoint_save(lulesh_set *s, void *buf, size_t bytes)
{
    if (!s || !buf || bytes < lulesh_checkpoint_bytes(s)) {
        set_error("lulesh_checkpoint_save: buffer smaller than lulesh_checkpoint_bytes");
        return LULESH_INVALID_ARG;
    }
    const CkptHeader h = header_of(s);
    char *p = static_cast<char *>(buf);
    std::memcpy(p, &h, sizeof h);
    CCHECK(cudaMemcpyAsync(p + sizeof h, s->arena, s->arena_bytes, cudaMemcpyDeviceToHost,
                           s->stream));
    CCHECK(cudaMemcpyAsync(p + sizeof h + s->arena_bytes, s->dtc, h.tc_bytes,
                           cudaMemcpyDeviceToHost, s->stream));
    CCHECK(cudaStreamSynchronize(s->stream));
    return LULESH_OK;
}

int lulesh_checkpoint_load(lulesh_set *s, const void *buf, size_t bytes)
{
    if (!s || !buf || bytes < sizeof(CkptHeader)) {
        set_error("lulesh_checkpoint_load: not a checkpoint");
        return LULESH_INVALID_ARG;
    }
    CkptHeader h;
    std::memcpy(&h, buf, sizeof h);
    const CkptHeader mine = header_of(s);
    if (h.magic != kMagic || h.version != kVersion) {
        set_error("lulesh_checkpoint_load: not a checkpoint of this library version");
        return LULESH_INVALID_ARG;
    }
    if (h.njobs != mine.njobs || h.ndom != mine.ndom || h.tp != mine.tp ||
        h.flags != mine.flags || h.arena_bytes != mine.arena_bytes ||
        h.tc_bytes != mine.tc_bytes || h.jobs_hash != mine.jobs_hash ||
        h.mesh_hash != mine.mesh_hash || h.nparts != mine.nparts || h.part != mine.part) {
        set_error("lulesh_checkpoint_load: checkpoint of a different set (jobs, mesh, tp, "
                  "part or flags)");
        return LULESH_INVALID_ARG;
    }
    if (bytes < lulesh_checkpoint_bytes(s)) {
        set_error("lulesh_checkpoint_load: truncated checkpoint");
        return LULESH_INVALID_ARG;
    }
    const char *p = static_cast<const char *>(buf);
    CCHECK(cudaStreamSynchronize(s->stream));  // no cycle may still use the state
    CCHECK(cudaMemcpyAsync(s->arena, p + sizeof h, s->arena_bytes, cudaMemcpyHostToDevice,
                           s->stream));
    CCHECK(cudaMemcpyAsync(s->dtc, p + sizeof h + s->arena_bytes, h.tc_bytes,
                           cudaMemcpyHostToDevice, s->stream));
    CCHECK(cudaStreamSynchronize(s->stream));
    return LULESH_OK;
}

}  // extern "C"
