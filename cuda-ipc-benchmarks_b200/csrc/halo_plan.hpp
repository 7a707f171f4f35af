// halo_plan.hpp -- which values cross between the GPUs (parts) of a
// decomposed problem, and in which order.
//
// A problem of tp^3 subdomains (ranks r = col + tp*(row + tp*plane), as
// InitMeshDecomp places them, lulesh.cu:4606-4668) is split over `nparts`
// GPUs: rank r belongs to part r * nparts / tp^3, so each part holds a run
// of consecutive ranks, which for a cube decomposition is a compact slab or
// block.  A subdomain whose neighbour lives on another part keeps a proxy of
// that neighbour: arrays in the neighbour's own layout of which only the
// layers the local kernels read are filled, by the messages planned here.
// The kernels then read the proxy exactly as they read an in-device
// neighbour, so a decomposed run gives the single-domain bits.
//
// One message per (kind, sender part, receiver part): the concatenation, in
// ascending (receiver rank, sender rank) order, of the items each adjacent
// pair (S on the sender part, R on the receiver part) needs, where an item
// is S.field[index] and lands at the same index of R's proxy of S.  What R
// reads from S, by kind, with d = R's position minus S's:
//   CORNERS  (the fused CommSBN: each node sums its corners in corner order,
//            lulesh.cu:1715-1751) fx/fy/fz_elem of S's elements in the layer
//            facing R, only the corners j on the shared nodes (4 on a face,
//            2 on an edge, 1 at a corner)
//   POSVEL   (CommSyncPosVel, lulesh-comms-gpu.cu:1231-1661: a shared node
//            takes x..zd from its "+side owner") x,y,z,xd,yd,zd of S's node
//            layer facing R, only when R lies on S's minus sides
//   MONOQ    (CommMonoQ, lulesh-comms-gpu.cu:1665-1806) delv_xi/eta/zeta of
//            S's element layer facing R, faces only
//   MASS     (the init-time nodalMass CommSBN, lulesh.cu:4811-4831) volo of
//            S's element layer facing R, all 26 directions
#pragma once

#include <vector>

namespace lulesh {

enum HaloKind { HALO_CORNERS = 0, HALO_POSVEL = 1, HALO_MONOQ = 2, HALO_MASS = 3, HALO_KINDS = 4 };

// one planned value: field `field` (lulesh_field_id) of subdomain `rank`
// at array index `index`
struct HaloItem {
    int rank;
    int field;
    long long index;
};

// part of rank r; -1 for arguments out of range
int halo_part_of(int r, int tp, int nparts);

// the other parts that part `part` exchanges with (ascending)
std::vector<int> halo_peers(int tp, int nparts, int part);

// the message of `kind` from part `from` to part `to` (empty when the two
// parts share no boundary or from == to); nx = subdomain edge
void halo_plan(int nx, int tp, int nparts, int from, int to, int kind,
               std::vector<HaloItem> &out);

}  // namespace lulesh
