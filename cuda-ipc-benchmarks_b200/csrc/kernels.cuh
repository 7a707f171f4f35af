// kernels.cuh -- launch interface of the per-cycle kernels.
#pragma once

#include <cuda_runtime.h>

#include "lulesh_dev.h"

// Block order of the kinematics and EOS launches.  Kinematics walks its
// block table last to first: its last outputs are then those of the first
// elements, where each rep class of the EOS walk starts, and they are still
// in L2 (measured on B200 at -s 100: EOS 91 -> 86 us, cycle 329 -> 325 us,
// the same results).  Reversing the EOS walk instead gained nothing.
#ifndef LULESH_KIN_REVERSE
#define LULESH_KIN_REVERSE 1
#endif
#ifndef LULESH_FORCE_REVERSE
#define LULESH_FORCE_REVERSE 0
#endif
#ifndef LULESH_EOS_REVERSE
#define LULESH_EOS_REVERSE 0
#endif

namespace lulesh {

constexpr int kElemBlock = 128;  // threads per block, element kernels
constexpr int kNodeBlock = 128;  // threads per block, node kernels

// Resident blocks per SM asked of the compiler (the register budget of the
// element kernels), chosen by measurement on B200 at -s 100: kinematics 3
// (<= 170 registers, 118 -> 92 us), EOS 12 (40 registers with small spills;
// 134 us unbounded, 97 us at 8 blocks, 86 us at 12, 88 us at 16).
#ifndef LULESH_FORCE_MINB
#define LULESH_FORCE_MINB 1
#endif
#ifndef LULESH_KIN_MINB
#define LULESH_KIN_MINB 3
#endif
#ifndef LULESH_EOS_MINB
#define LULESH_EOS_MINB 12
#endif
// nodal: 16 blocks (32 registers, every warp slot of the SM) for the
// streaming corner gather, 60.2 -> 56.7 us
#ifndef LULESH_NODAL_MINB
#define LULESH_NODAL_MINB 16
#endif
constexpr int kNodalMinBlocks = LULESH_NODAL_MINB;
// unstructured nodal kernel: four corners x 3 components in flight
#ifndef LULESH_NODAL_U_MINB
#define LULESH_NODAL_U_MINB 12
#endif
constexpr int kNodalUMinBlocks = LULESH_NODAL_U_MINB;
constexpr int kForceMinBlocks = LULESH_FORCE_MINB;
constexpr int kKinMinBlocks = LULESH_KIN_MINB;
constexpr int kEosMinBlocks = LULESH_EOS_MINB;

// Minimum resident blocks of a kernel launched with BS threads per block
// that keeps the per-SM thread target of `minb` blocks of 128 threads.
constexpr int min_blocks(int minb, int bs)
{
    return (minb * 128 / bs) > 0 ? (minb * 128 / bs) : 1;
}

// Block shapes the FP64 element kernels (force, kinematics, EOS) and the
// nodal kernel are compiled for; a set's block tables use one of each.
constexpr bool valid_elem_block(int bs) { return bs == 64 || bs == 128 || bs == 256; }
constexpr bool valid_node_block(int bs) { return bs == 128 || bs == 256 || bs == 512; }

// A kernel launch over all domains of a set: block b works on domain
// blocks[b].x starting at item blocks[b].y (element, node or region slot).
struct SetArgs {
    const DomDev *doms;
    TimeCtl *tcs;
    const int2 *blocks;
    int materialize;  // also write the per-cycle transients
    // launch with programmatic stream serialisation (host side only; the
    // kernels launched this way wait for the previous grid first)
    int pdl = 0;
};

// ---------------------------------------------------------------------------
// checked builds
//
// With -DLULESH_CHECKED=1 the FP64 cycle kernels range-check every index
// they compute or load before using it: node indices, corner indices,
// corner-list runs, EOS slots and face links.  An index out of range is
// replaced by 0, which every array holds, so no access leaves its array and
// no thread leaves the kernel's control flow.  The first failing check's
// code is kept in TimeCtl::chk, and the next time increment ends the job
// with LULESH_BOUNDS_ERROR.  This build stands in for a memory checker.
#ifndef LULESH_CHECKED
#define LULESH_CHECKED 0
#endif
enum CheckCode { kChkNode = 1, kChkCorner = 2, kChkCornerRun = 3, kChkSlot = 4, kChkLink = 5 };

__device__ __forceinline__ int chk_index(long long i, long long n, TimeCtl *T, int code)
{
#if LULESH_CHECKED
    if (i < 0 || i >= n) {
        atomicCAS(&T->chk, 0, code);
        return 0;
    }
#else
    (void)n;
    (void)T;
    (void)code;
#endif
    return (int)i;
}

// ---------------------------------------------------------------------------
// programmatic dependent launch
//
// The cycle kernels may be launched with programmatic stream serialisation
// (SetArgs::pdl): the next kernel's blocks are then scheduled while this
// one's last wave drains.  Every kernel launched that way starts with
// pdl_enter(): it waits until the previous grid has completed and its
// writes are visible, before touching any memory, then lets its own
// dependents be scheduled.  Without the attribute both pass at once.

__device__ __forceinline__ void pdl_enter()
{
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), int grid, int block, cudaStream_t s, bool pdl,
                     Args... args)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = pdl ? attr : nullptr;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, args...);  // errors: cudaGetLastError
}

void launch_time_increment(TimeCtl *tcs, int ntc, Params P, cudaStream_t s, bool pdl = false);
// u: the set's domains are unstructured (lmesh): 128-wide blocks, mesh
// arrays read instead of structured indexing
void launch_force(const SetArgs &a, int nblocks, Params P, cudaStream_t s,
                  int bs = kElemBlock, bool u = false);
void launch_nodal(const SetArgs &a, int nblocks, Params P, cudaStream_t s,
                  int bs = kNodeBlock, bool u = false);
// staged comm path: own-corner partial sums, then the update from fx/fy/fz
void launch_nodal_gather_local(const SetArgs &a, int nblocks, cudaStream_t s);
void launch_nodal_update(const SetArgs &a, int nblocks, Params P, cudaStream_t s);
void launch_kinematics(const SetArgs &a, int nblocks, Params P, cudaStream_t s,
                       int bs = kElemBlock, bool u = false);
// sub: a subdomain set's fused cycle, comm-face neighbours read in the
// neighbouring subdomain (k_monoq_ghost not needed)
void launch_eos(const SetArgs &a, int nblocks, Params P, cudaStream_t s, int bs = kElemBlock,
                bool u = false, bool sub = false);
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
