// kernels.cuh -- launch interface of the per-cycle kernels.
#pragma once

#include <cuda_runtime.h>

#include "lulesh_dev.h"

namespace lulesh {

constexpr int kElemBlock = 128;  // threads per block, element kernels
constexpr int kNodeBlock = 128;  // threads per block, node kernels

// A kernel launch over all domains of a set: block b works on domain
// blocks[b].x starting at item blocks[b].y (element, node or region slot).
struct SetArgs {
    const DomDev *doms;
    TimeCtl *tcs;
    const int2 *blocks;
    int materialize;  // also write the per-cycle transients
};

void launch_time_increment(TimeCtl *tcs, int ntc, Params P, cudaStream_t s);
void launch_force(const SetArgs &a, int nblocks, Params P, cudaStream_t s);
void launch_nodal(const SetArgs &a, int nblocks, Params P, cudaStream_t s);
// staged comm path: own-corner partial sums, then the update from fx/fy/fz
void launch_nodal_gather_local(const SetArgs &a, int nblocks, cudaStream_t s);
void launch_nodal_update(const SetArgs &a, int nblocks, Params P, cudaStream_t s);
void launch_kinematics(const SetArgs &a, int nblocks, Params P, cudaStream_t s);
void launch_eos(const SetArgs &a, int nblocks, Params P, cudaStream_t s);
// fused halo kernels of a subdomain set (direct reads of neighbour memory)
void launch_posvel_sync(const SetArgs &a, int nblocks, cudaStream_t s);
void launch_monoq_ghost(const SetArgs &a, int nblocks, cudaStream_t s);

// mixed precision variants of the element kernels
void launch_force_mixed(const SetArgs &a, int nblocks, Params P, const CornerF32 *cf,
                        cudaStream_t s);
void launch_nodal_mixed(const SetArgs &a, int nblocks, Params P, const CornerF32 *cf,
                        cudaStream_t s);
void launch_kinematics_mixed(const SetArgs &a, int nblocks, Params P, cudaStream_t s);

}  // namespace lulesh
