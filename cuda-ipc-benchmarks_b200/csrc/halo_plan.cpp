// halo_plan.cpp -- the message plan of a decomposed problem split over
// several GPUs (halo_plan.hpp).  Host code only: the GPU build turns the
// plan into pointer tables for its pack/unpack kernels (part.cu), and the
// CPU test suite calls the same functions through liblulesh_host.so.
#include "halo_plan.hpp"

#include <set>

#include "lulesh_b200.h"

namespace lulesh {

namespace {

void rank_pos(int r, int tp, int &c, int &w, int &p)
{
    c = r % tp;
    w = (r / tp) % tp;
    p = r / (tp * tp);
}

// corner j of an element sits at lattice offset (bit j of 0x66, 0xCC, 0xF0)
inline int cx(int j) { return (0x66 >> j) & 1; }
inline int cy(int j) { return (0xCC >> j) & 1; }
inline int cz(int j) { return (0xF0 >> j) & 1; }

// the coordinate range [lo, hi) along one axis of the layer of S that faces
// a neighbour at offset d along that axis; `ext` is the axis length
inline void layer(int d, int ext, int &lo, int &hi)
{
    if (d > 0) {
        lo = ext - 1;
        hi = ext;
    } else if (d < 0) {
        lo = 0;
        hi = 1;
    } else {
        lo = 0;
        hi = ext;
    }
}

// items S -> R for R at offset (dx,dy,dz) from S
void pair_items(int nx, int S, int dx, int dy, int dz, int kind, std::vector<HaloItem> &out)
{
    const long long E = (long long)nx * nx * nx;
    const long long Ep = ((E + 31) / 32) * 32;
    const int en = nx + 1;
    const int nonzero = (dx != 0) + (dy != 0) + (dz != 0);
    int x0, x1, y0, y1, z0, z1;
    switch (kind) {
        case HALO_CORNERS: {
            layer(dx, nx, x0, x1);
            layer(dy, nx, y0, y1);
            layer(dz, nx, z0, z1);
            const int fields[3] = {LULESH_F_FX_ELEM, LULESH_F_FY_ELEM, LULESH_F_FZ_ELEM};
            for (int f : fields)
                for (int j = 0; j < 8; ++j) {
                    // corner j touches the shared nodes when it sits on R's
                    // side along every axis where R is offset
                    if ((dx != 0 && cx(j) != (dx > 0)) || (dy != 0 && cy(j) != (dy > 0)) ||
                        (dz != 0 && cz(j) != (dz > 0)))
                        continue;
                    for (int iz = z0; iz < z1; ++iz)
                        for (int iy = y0; iy < y1; ++iy)
                            for (int ix = x0; ix < x1; ++ix)
                                out.push_back(HaloItem{S, f, j * Ep + ((long long)iz * nx + iy) * nx + ix});
                }
            break;
        }
        case HALO_POSVEL: {
            // R takes a shared node from S only when S lies on R's plus
            // sides (S is the node's "+side owner"), i.e. R on S's minus sides
            if (dx > 0 || dy > 0 || dz > 0) return;
            layer(dx, en, x0, x1);
            layer(dy, en, y0, y1);
            layer(dz, en, z0, z1);
            const int fields[6] = {LULESH_F_X,  LULESH_F_Y,  LULESH_F_Z,
                                   LULESH_F_XD, LULESH_F_YD, LULESH_F_ZD};
            for (int f : fields)
                for (int pz = z0; pz < z1; ++pz)
                    for (int py = y0; py < y1; ++py)
                        for (int px = x0; px < x1; ++px)
                            out.push_back(HaloItem{S, f, ((long long)pz * en + py) * en + px});
            break;
        }
        case HALO_MONOQ: {
            if (nonzero != 1) return;  // ghost faces only
            layer(dx, nx, x0, x1);
            layer(dy, nx, y0, y1);
            layer(dz, nx, z0, z1);
            const int fields[3] = {LULESH_F_DELV_XI, LULESH_F_DELV_ETA, LULESH_F_DELV_ZETA};
            for (int f : fields)
                for (int iz = z0; iz < z1; ++iz)
                    for (int iy = y0; iy < y1; ++iy)
                        for (int ix = x0; ix < x1; ++ix)
                            out.push_back(HaloItem{S, f, ((long long)iz * nx + iy) * nx + ix});
            break;
        }
        case HALO_MASS: {
            layer(dx, nx, x0, x1);
            layer(dy, nx, y0, y1);
            layer(dz, nx, z0, z1);
            for (int iz = z0; iz < z1; ++iz)
                for (int iy = y0; iy < y1; ++iy)
                    for (int ix = x0; ix < x1; ++ix)
                        out.push_back(HaloItem{S, LULESH_F_VOLO, ((long long)iz * nx + iy) * nx + ix});
            break;
        }
        default: break;
    }
}

}  // namespace

int halo_part_of(int r, int tp, int nparts)
{
    if (tp < 1 || nparts < 1) return -1;
    const long long T = (long long)tp * tp * tp;
    if (nparts > T || r < 0 || r >= T) return -1;
    return (int)((long long)r * nparts / T);
}

std::vector<int> halo_peers(int tp, int nparts, int part)
{
    std::set<int> peers;
    const int T = tp * tp * tp;
    for (int r = 0; r < T; ++r) {
        if (halo_part_of(r, tp, nparts) != part) continue;
        int c, w, p;
        rank_pos(r, tp, c, w, p);
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const int nc = c + dx, nw = w + dy, np = p + dz;
                    if ((dx | dy | dz) == 0 || nc < 0 || nw < 0 || np < 0 || nc >= tp ||
                        nw >= tp || np >= tp)
                        continue;
                    const int q = halo_part_of(nc + tp * (nw + tp * np), tp, nparts);
                    if (q != part) peers.insert(q);
                }
    }
    return std::vector<int>(peers.begin(), peers.end());
}

void halo_plan(int nx, int tp, int nparts, int from, int to, int kind,
               std::vector<HaloItem> &out)
{
    out.clear();
    if (from == to || nx < 1 || kind < 0 || kind >= HALO_KINDS) return;
    const int T = tp * tp * tp;
    for (int R = 0; R < T; ++R) {
        if (halo_part_of(R, tp, nparts) != to) continue;
        int rc, rw, rp;
        rank_pos(R, tp, rc, rw, rp);
        for (int S = 0; S < T; ++S) {
            if (halo_part_of(S, tp, nparts) != from) continue;
            int sc, sw, sp;
            rank_pos(S, tp, sc, sw, sp);
            const int dx = rc - sc, dy = rw - sw, dz = rp - sp;
            if ((dx | dy | dz) == 0 || dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 ||
                dz > 1)
                continue;
            pair_items(nx, S, dx, dy, dz, kind, out);
        }
    }
}

}  // namespace lulesh

using namespace lulesh;

extern "C" {

int lulesh_part_of(int rank, int tp, int nparts) { return halo_part_of(rank, tp, nparts); }

int lulesh_halo_peers(int tp, int nparts, int part, int *peers, int max_peers)
{
    if (tp < 1 || nparts < 1 || part < 0 || part >= nparts ||
        (long long)nparts > (long long)tp * tp * tp)
        return LULESH_INVALID_ARG;
    const std::vector<int> p = halo_peers(tp, nparts, part);
    for (int i = 0; i < (int)p.size() && i < max_peers; ++i)
        if (peers) peers[i] = p[i];
    return (int)p.size();
}

long long lulesh_halo_plan(int nx, int tp, int nparts, int from_part, int to_part, int kind,
                           int *rank, int *field, long long *index, long long max_items)
{
    if (nx < 1 || nx > LULESH_MAX_NX || tp < 1 || nparts < 1 ||
        (long long)nparts > (long long)tp * tp * tp || from_part < 0 || from_part >= nparts ||
        to_part < 0 || to_part >= nparts || kind < 0 || kind >= HALO_KINDS)
        return LULESH_INVALID_ARG;
    std::vector<HaloItem> items;
    halo_plan(nx, tp, nparts, from_part, to_part, kind, items);
    for (long long i = 0; i < (long long)items.size() && i < max_items; ++i) {
        if (rank) rank[i] = items[i].rank;
        if (field) field[i] = items[i].field;
        if (index) index[i] = items[i].index;
    }
    return (long long)items.size();
}

}  // extern "C"
