// host_setup.cpp -- host-side construction of LULESH domains (see header).
#include "host_setup.hpp"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <string>

namespace lulesh {

// ---- glibc rand ----------------------------------------------------------
// Published description of glibc's default generator: state r[0] = seed
// (0 becomes 1), r[i] = 16807 * r[i-1] mod (2^31 - 1) for i < 31 (Schrage's
// method), r[31..33] = r[0..2], then r[i] = r[i-31] + r[i-3] (mod 2^32);
// the first 310 outputs are discarded and each output is r[i] >> 1.
GlibcRand::GlibcRand(unsigned seed)
{
    int32_t s = (seed == 0) ? 1 : (int32_t)seed;
    int32_t st[31];
    st[0] = s;
    for (int i = 1; i < 31; ++i) {
        int64_t hi = st[i - 1] / 127773, lo = st[i - 1] % 127773;
        int64_t w = 16807 * lo - 2836 * hi;
        if (w < 0) w += 2147483647;
        st[i] = (int32_t)w;
    }
    // ring of the last 34 words, kept as unsigned arithmetic
    uint32_t ring[344];
    for (int i = 0; i < 31; ++i) ring[i] = (uint32_t)st[i];
    for (int i = 31; i < 34; ++i) ring[i] = ring[i - 31];
    for (int i = 34; i < 344; ++i) ring[i] = ring[i - 31] + ring[i - 3];
    for (int i = 0; i < 34; ++i) r_[i] = (int32_t)ring[344 - 34 + i];
    idx_ = 0;  // r_[idx_] is the oldest of the last 34 words
}

int GlibcRand::next()
{
    // newest = word[-31] + word[-3]; r_ holds words[-34..-1] starting at idx_
    uint32_t a = (uint32_t)r_[(idx_ + 34 - 31) % 34];
    uint32_t b = (uint32_t)r_[(idx_ + 34 - 3) % 34];
    uint32_t w = a + b;
    r_[idx_] = (int32_t)w;
    idx_ = (idx_ + 1) % 34;
    return (int)(w >> 1);
}

// ---- element volume --------------------------------------------------------

static inline double triple(double a1, double b1, double c1, double a2,
                            double b2, double c2, double a3, double b3,
                            double c3)
{
    return a1 * (b2 * c3 - c2 * b3) + a2 * (c1 * b3 - b1 * c3) +
           a3 * (b1 * c2 - c1 * b2);
}

double elem_volume_host(const double *x, const double *y, const double *z)
{
    const double twelveth = 1.0 / 12.0;
    double dx61 = x[6] - x[1], dy61 = y[6] - y[1], dz61 = z[6] - z[1];
    double dx70 = x[7] - x[0], dy70 = y[7] - y[0], dz70 = z[7] - z[0];
    double dx63 = x[6] - x[3], dy63 = y[6] - y[3], dz63 = z[6] - z[3];
    double dx20 = x[2] - x[0], dy20 = y[2] - y[0], dz20 = z[2] - z[0];
    double dx50 = x[5] - x[0], dy50 = y[5] - y[0], dz50 = z[5] - z[0];
    double dx64 = x[6] - x[4], dy64 = y[6] - y[4], dz64 = z[6] - z[4];
    double dx31 = x[3] - x[1], dy31 = y[3] - y[1], dz31 = z[3] - z[1];
    double dx72 = x[7] - x[2], dy72 = y[7] - y[2], dz72 = z[7] - z[2];
    double dx43 = x[4] - x[3], dy43 = y[4] - y[3], dz43 = z[4] - z[3];
    double dx57 = x[5] - x[7], dy57 = y[5] - y[7], dz57 = z[5] - z[7];
    double dx14 = x[1] - x[4], dy14 = y[1] - y[4], dz14 = z[1] - z[4];
    double dx25 = x[2] - x[5], dy25 = y[2] - y[5], dz25 = z[2] - z[5];
    double vol = triple(dx31 + dx72, dx63, dx20, dy31 + dy72, dy63, dy20,
                        dz31 + dz72, dz63, dz20) +
                 triple(dx43 + dx57, dx64, dx70, dy43 + dy57, dy64, dy70,
                        dz43 + dz57, dz64, dz70) +
                 triple(dx14 + dx25, dx61, dx50, dy14 + dy25, dy61, dy50,
                        dz14 + dz25, dz61, dz50);
    vol *= twelveth;
    return vol;
}

Params default_params()
{
    Params p;
    p.dtfixed = -1.0e-6;
    p.deltatimemultlb = 1.1;
    p.deltatimemultub = 1.2;
    p.stoptime = 1.0e-2;
    p.dtmax = 1.0e-2;
    p.e_cut = 1.0e-7;
    p.p_cut = 1.0e-7;
    p.q_cut = 1.0e-7;
    p.u_cut = 1.0e-7;
    p.v_cut = 1.0e-10;
    p.hgcoef = 3.0;
    p.ss4o3 = 4.0 / 3.0;
    p.qstop = 1.0e+12;
    p.monoq_max_slope = 1.0;
    p.monoq_limiter_mult = 2.0;
    p.qlc_monoq = 0.5;
    p.qqc_monoq = 2.0 / 3.0;
    p.qqc = 2.0;
    p.pmin = 0.;
    p.emin = -1.0e+15;
    p.dvovmax = 0.1;
    p.eosvmax = 1.0e+9;
    p.eosvmin = 1.0e-9;
    p.refdens = 1.0;
    return p;
}

// coordinate of global lattice index g on a mesh of `edge` elements
// (BuildMesh, lulesh.cu:698-715)
static inline double lattice(int g, int edge)
{
    return 1.125 * (double)g / (double)edge;
}

// node -> corner CSR from the nodelist, outer corner j, inner element
// (lulesh.cu:1054-1106)
static void build_corner_csr(HostDomain &d)
{
    const int E = d.numElem, N = d.numNode, Ep = d.Ep;
    d.nodeElemCount.assign(N, 0);
    d.nodeElemStart.assign(N, 0);
    for (int i = 0; i < E; ++i)
        for (int j = 0; j < 8; ++j) d.nodeElemCount[d.nodelist[(size_t)j * Ep + i]]++;
    for (int i = 1; i < N; ++i)
        d.nodeElemStart[i] = d.nodeElemStart[i - 1] + d.nodeElemCount[i - 1];
    d.nodeElemCornerList.assign((size_t)d.nodeElemStart[N - 1] + d.nodeElemCount[N - 1], 0);
    std::vector<int> fill(N, 0);
    for (int j = 0; j < 8; ++j)
        for (int i = 0; i < E; ++i) {
            int m = d.nodelist[(size_t)j * Ep + i];
            d.nodeElemCornerList[d.nodeElemStart[m] + fill[m]] = Ep * j + i;
            fill[m]++;
        }
}

// ---- regions: CreateRegionIndexSets + sortRegions, lulesh.cu:1224-1398 ----

// The draw of CreateRegionIndexSets (lulesh.cu:1296-1351): run k covers the
// elements from runs[k].start up to the next run's start (the last run up to
// E) and gives them region number runs[k].region.  Only start and region
// are filled.  A single region takes no draw.
static std::vector<RegionRun> draw_region_runs(int rank, int E, int nr, int balance)
{
    std::vector<RegionRun> runs;
    if (nr == 1) {
        runs.push_back({0, 1, 0, 0});
        return runs;
    }
    GlibcRand rng((unsigned)rank);
    std::vector<int> binEnd(nr);
    int costDen = 0;
    for (int i = 0; i < nr; ++i) {
        int w = 1;
        for (int k = 0; k < balance; ++k) w *= (i + 1);
        costDen += w;
        binEnd[i] = costDen;
    }
    auto pick = [&]() {
        int v = rng.next() % costDen, i = 0;
        while (v >= binEnd[i]) ++i;
        return ((i + rank) % nr) + 1;
    };
    int lastReg = -1, next = 0;
    while (next < E) {
        int regionNum = pick();
        while (regionNum == lastReg) regionNum = pick();
        int bin = rng.next() % 1000, elements;
        if (bin < 773)
            elements = rng.next() % 15 + 1;
        else if (bin < 937)
            elements = rng.next() % 16 + 16;
        else if (bin < 970)
            elements = rng.next() % 32 + 32;
        else if (bin < 974)
            elements = rng.next() % 64 + 64;
        else if (bin < 978)
            elements = rng.next() % 128 + 128;
        else if (bin < 981)
            elements = rng.next() % 256 + 256;
        else
            elements = rng.next() % 1537 + 512;
        runs.push_back({next, regionNum, 0, 0});
        next = std::min(next + elements, E);
        lastReg = regionNum;
    }
    return runs;
}

// Rep counts per region, the stable descending bubble sort by reps that
// carries the sizes and indices along (sortRegions), regSorted, and the
// region starts in regCSR.  Expects d.regElemSize to hold each region's
// element count by region index.
static void sort_regions(HostDomain &d, int nr)
{
    for (int r = 0; r < nr; ++r) {
        int rep;
        if (r < nr / 2)
            rep = 1;
        else if (r < (nr - (nr + 15) / 20))
            rep = 1 + d.cost;
        else
            rep = 10 * (1 + d.cost);
        d.regReps[r] = rep;
    }
    std::vector<int> idx(nr);
    for (int i = 0; i < nr; ++i) idx[i] = i;
    for (int i = 0; i < nr - 1; ++i)
        for (int j = 0; j < nr - i - 1; ++j)
            if (d.regReps[j] < d.regReps[j + 1]) {
                std::swap(d.regReps[j], d.regReps[j + 1]);
                std::swap(d.regElemSize[j], d.regElemSize[j + 1]);
                std::swap(idx[j], idx[j + 1]);
            }
    for (int i = 0; i < nr; ++i) d.regSorted[idx[i]] = i;
    d.regCSR[0] = 0;
    for (int i = 1; i < nr; ++i) d.regCSR[i] = d.regCSR[i - 1] + d.regElemSize[i - 1];
}

static void build_regions(HostDomain &d, int nr, int balance)
{
    const int E = d.numElem;
    d.numReg = nr;
    d.balance = balance;
    d.regElemSize.assign(nr, 0);
    d.regCSR.assign(nr, 0);
    d.regReps.assign(nr, 0);
    d.regSorted.assign(nr, 0);
    d.regNumList.assign(E, 0);
    d.regElemlist.assign(E, 0);
    const std::vector<RegionRun> runs = draw_region_runs(d.rank, E, nr, balance);
    for (size_t k = 0; k < runs.size(); ++k) {
        const int end = k + 1 < runs.size() ? runs[k + 1].start : E;
        for (int i = runs[k].start; i < end; ++i) d.regNumList[i] = runs[k].region;
    }
    for (int i = 0; i < E; ++i) d.regElemSize[d.regNumList[i] - 1]++;
    sort_regions(d, nr);
    // fill; afterwards regCSR[r] is the END of region r, which is what the
    // EOS region lookup (giveMyRegion, lulesh.cu:3976-3984) searches
    for (int i = 0; i < E; ++i) {
        int r = d.regSorted[d.regNumList[i] - 1];
        d.regElemlist[d.regCSR[r]] = i;
        d.regCSR[r]++;
    }

    // EOS work order.  Each element's rep count is that of its region
    // (regReps is sorted with the regions); the EOS of an element depends
    // only on that element, so the order elements are visited in is free.
    // Grouping by rep count keeps a warp's trip count uniform, like the
    // reference's per-region order, while the classes (at most three) are
    // far denser than single regions, so a warp's loads share cache lines.
    std::vector<int> rep_of(E);
    std::vector<int> distinct;
    for (int i = 0; i < E; ++i) {
        rep_of[i] = d.regReps[d.regSorted[d.regNumList[i] - 1]];
        bool seen = false;
        for (int v : distinct) seen = seen || (v == rep_of[i]);
        if (!seen) distinct.push_back(rep_of[i]);
    }
    std::sort(distinct.begin(), distinct.end(), [](int a, int b) { return a > b; });
    d.eosOrder.clear();
    d.eosOrder.reserve(E);
    d.eosNumClass = (int)distinct.size();
    for (int c = 0; c < d.eosNumClass; ++c) {
        for (int i = 0; i < E; ++i)
            if (rep_of[i] == distinct[c]) d.eosOrder.push_back(i);
        d.eosClassEnd[c] = (int)d.eosOrder.size();
        d.eosClassRep[c] = distinct[c];
    }
}

// The same region sets as build_regions, kept as runs: the per-region and
// per-class tables are complete, regNumList, regElemlist and eosOrder stay
// empty, and each run carries where its elements go in the last two
// (expand_region_element writes them).  A region's runs come in ascending
// element order, and so do a rep class's, which is the order both lists
// hold their elements in.
static void build_region_runs(HostDomain &d, int nr, int balance)
{
    const int E = d.numElem;
    d.numReg = nr;
    d.balance = balance;
    d.regElemSize.assign(nr, 0);
    d.regCSR.assign(nr, 0);
    d.regReps.assign(nr, 0);
    d.regSorted.assign(nr, 0);
    d.regNumList.clear();
    d.regElemlist.clear();
    d.eosOrder.clear();
    d.regionRuns = draw_region_runs(d.rank, E, nr, balance);
    std::vector<RegionRun> &runs = d.regionRuns;
    auto run_len = [&](size_t k) {
        return (k + 1 < runs.size() ? runs[k + 1].start : E) - runs[k].start;
    };
    for (size_t k = 0; k < runs.size(); ++k) d.regElemSize[runs[k].region - 1] += run_len(k);
    // element counts by region index, before the sort permutes them
    const std::vector<int> count = d.regElemSize;
    sort_regions(d, nr);
    // rep classes: the distinct rep counts of the regions that hold
    // elements, heaviest first, each class's elements one after the other
    std::vector<int> distinct;
    for (int r = 0; r < nr; ++r) {
        if (count[r] == 0) continue;
        const int rep = d.regReps[d.regSorted[r]];
        if (std::find(distinct.begin(), distinct.end(), rep) == distinct.end())
            distinct.push_back(rep);
    }
    std::sort(distinct.begin(), distinct.end(), [](int a, int b) { return a > b; });
    d.eosNumClass = (int)distinct.size();
    std::vector<int> class_at(d.eosNumClass, 0);
    int total = 0;
    for (int c = 0; c < d.eosNumClass; ++c) {
        class_at[c] = total;
        for (int r = 0; r < nr; ++r)
            if (count[r] > 0 && d.regReps[d.regSorted[r]] == distinct[c]) total += count[r];
        d.eosClassEnd[c] = total;
        d.eosClassRep[c] = distinct[c];
    }
    for (size_t k = 0; k < runs.size(); ++k) {
        const int r = runs[k].region - 1, s = d.regSorted[r];
        const int c = (int)(std::find(distinct.begin(), distinct.end(), d.regReps[s]) -
                            distinct.begin());
        runs[k].list_at = d.regCSR[s];
        runs[k].eos_at = class_at[c];
        d.regCSR[s] += run_len(k);
        class_at[c] += run_len(k);
    }
    // regCSR now holds each region's END, as after build_regions' fill
}

void build_domain(HostDomain &d, int nx, int tp, int col, int row, int plane,
                  int rank, int numReg, int balance, int cost, bool global_mass)
{
    const int en = nx + 1;
    d.nx = nx;
    d.en = en;
    d.tp = tp;
    d.col = col;
    d.row = row;
    d.plane = plane;
    d.rank = rank;
    d.cost = cost;
    d.numElem = nx * nx * nx;
    d.Ep = ((d.numElem + 31) / 32) * 32;  // PAD(numElem, 32), lulesh.cu:791
    d.numNode = en * en * en;
    const int E = d.numElem, N = d.numNode, Ep = d.Ep;

    // neighbour flags, lulesh.cu:463-468
    d.rowMin = (row == 0) ? 0 : 1;
    d.rowMax = (row == tp - 1) ? 0 : 1;
    d.colMin = (col == 0) ? 0 : 1;
    d.colMax = (col == tp - 1) ? 0 : 1;
    d.planeMin = (plane == 0) ? 0 : 1;
    d.planeMax = (plane == tp - 1) ? 0 : 1;
    // local elements + ghost faces, lulesh.cu:4146-4149
    d.allElem = E + 2 * nx * nx + 2 * nx * nx + 2 * nx * nx;

    // coordinates, lulesh.cu:696-716
    const int meshEdge = tp * nx;
    d.x.resize(N);
    d.y.resize(N);
    d.z.resize(N);
    for (int pl = 0, n = 0; pl < en; ++pl)
        for (int r = 0; r < en; ++r)
            for (int c = 0; c < en; ++c, ++n) {
                d.x[n] = lattice(col * nx + c, meshEdge);
                d.y[n] = lattice(row * nx + r, meshEdge);
                d.z[n] = lattice(plane * nx + pl, meshEdge);
            }

    // node-major nodelist with stride Ep, lulesh.cu:722-744
    d.nodelist.assign(8 * (size_t)Ep, 0);
    for (int iz = 0, zidx = 0; iz < nx; ++iz)
        for (int iy = 0; iy < nx; ++iy)
            for (int ix = 0; ix < nx; ++ix, ++zidx) {
                int n0 = (iz * en + iy) * en + ix;
                const int off[8] = {0, 1, en + 1, en, en * en, en * en + 1,
                                    en * en + en + 1, en * en + en};
                for (int k = 0; k < 8; ++k) d.nodelist[(size_t)k * Ep + zidx] = n0 + off[k];
            }

    // symmetry planes, lulesh.cu:809-851
    d.numSymmX = (col == 0) ? en * en : 0;
    d.numSymmY = (row == 0) ? en * en : 0;
    d.numSymmZ = (plane == 0) ? en * en : 0;
    d.symmX.assign(en * en, 0);
    d.symmY.assign(en * en, 0);
    d.symmZ.assign(en * en, 0);
    for (int i = 0, k = 0; i < en; ++i)
        for (int j = 0; j < en; ++j, ++k) {
            if (plane == 0) d.symmZ[k] = i * en + j;
            if (row == 0) d.symmY[k] = i * en * en + j;
            if (col == 0) d.symmX[k] = i * en * en + j * en;
        }

    // face connectivity and element BCs, lulesh.cu:537-686
    d.lxim.resize(E);
    d.lxip.resize(E);
    d.letam.resize(E);
    d.letap.resize(E);
    d.lzetam.resize(E);
    d.lzetap.resize(E);
    d.elemBC.assign(E, 0);
    d.lxim[0] = 0;
    for (int i = 1; i < E; ++i) {
        d.lxim[i] = i - 1;
        d.lxip[i - 1] = i;
    }
    d.lxip[E - 1] = E - 1;
    for (int i = 0; i < nx; ++i) {
        d.letam[i] = i;
        d.letap[E - nx + i] = E - nx + i;
    }
    for (int i = nx; i < E; ++i) {
        d.letam[i] = i - nx;
        d.letap[i - nx] = i;
    }
    for (int i = 0; i < nx * nx; ++i) {
        d.lzetam[i] = i;
        d.lzetap[E - nx * nx + i] = E - nx * nx + i;
    }
    for (int i = nx * nx; i < E; ++i) {
        d.lzetam[i] = i - nx * nx;
        d.lzetap[i - nx * nx] = i;
    }
    int gidx[6];
    for (int i = 0; i < 6; ++i) gidx[i] = INT_MIN;
    {
        int pidx = E;
        const int face = nx * nx;
        const int present[6] = {d.planeMin, d.planeMax, d.rowMin, d.rowMax, d.colMin, d.colMax};
        for (int f = 0; f < 6; ++f)
            if (present[f]) {
                gidx[f] = pidx;
                pidx += face;
            }
    }
    for (int f = 0; f < 6; ++f) d.ghost[f] = (gidx[f] == INT_MIN) ? -1 : gidx[f];
    for (int i = 0; i < nx; ++i) {
        const int planeInc = i * nx * nx, rowInc = i * nx;
        for (int j = 0; j < nx; ++j) {
            int a;
            a = rowInc + j;  // zeta-minus face
            if (plane == 0) {
                d.elemBC[a] |= ZETA_M_SYMM;
            } else {
                d.elemBC[a] |= ZETA_M_COMM;
                d.lzetam[a] = gidx[0] + rowInc + j;
            }
            a = rowInc + j + E - nx * nx;  // zeta-plus face
            if (plane == tp - 1) {
                d.elemBC[a] |= ZETA_P_FREE;
            } else {
                d.elemBC[a] |= ZETA_P_COMM;
                d.lzetap[a] = gidx[1] + rowInc + j;
            }
            a = planeInc + j;  // eta-minus face
            if (row == 0) {
                d.elemBC[a] |= ETA_M_SYMM;
            } else {
                d.elemBC[a] |= ETA_M_COMM;
                d.letam[a] = gidx[2] + rowInc + j;
            }
            a = planeInc + j + nx * nx - nx;  // eta-plus face
            if (row == tp - 1) {
                d.elemBC[a] |= ETA_P_FREE;
            } else {
                d.elemBC[a] |= ETA_P_COMM;
                d.letap[a] = gidx[3] + rowInc + j;
            }
            a = planeInc + j * nx;  // xi-minus face
            if (col == 0) {
                d.elemBC[a] |= XI_M_SYMM;
            } else {
                d.elemBC[a] |= XI_M_COMM;
                d.lxim[a] = gidx[4] + rowInc + j;
            }
            a = planeInc + j * nx + nx - 1;  // xi-plus face
            if (col == tp - 1) {
                d.elemBC[a] |= XI_P_FREE;
            } else {
                d.elemBC[a] |= XI_P_COMM;
                d.lxip[a] = gidx[5] + rowInc + j;
            }
        }
    }

    build_corner_csr(d);
    d.matElemlist.resize(E);
    for (int i = 0; i < E; ++i) d.matElemlist[i] = i;

    // volo, elemMass, nodalMass, lulesh.cu:1160-1187
    d.volo.resize(E);
    d.elemMass.resize(E);
    d.nodalMass.assign(N, 0.0);
    auto volume_of = [&](int gx, int gy, int gz) {
        // element with global lattice origin (gx,gy,gz), corner order of
        // the nodelist above
        const int dx[8] = {0, 1, 1, 0, 0, 1, 1, 0};
        const int dy[8] = {0, 0, 1, 1, 0, 0, 1, 1};
        const int dz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
        double xl[8], yl[8], zl[8];
        for (int k = 0; k < 8; ++k) {
            xl[k] = lattice(gx + dx[k], meshEdge);
            yl[k] = lattice(gy + dy[k], meshEdge);
            zl[k] = lattice(gz + dz[k], meshEdge);
        }
        return elem_volume_host(xl, yl, zl);
    };
    for (int i = 0; i < E; ++i) {
        double xl[8], yl[8], zl[8];
        for (int k = 0; k < 8; ++k) {
            int g = d.nodelist[(size_t)k * Ep + i];
            xl[k] = d.x[g];
            yl[k] = d.y[g];
            zl[k] = d.z[g];
        }
        double vol = elem_volume_host(xl, yl, zl);
        d.volo[i] = vol;
        d.elemMass[i] = vol;
        if (!global_mass)
            for (int k = 0; k < 8; ++k) d.nodalMass[d.nodelist[(size_t)k * Ep + i]] += vol / 8.0;
    }
    if (global_mass) {
        // Sum, for every node, the elements of the whole tp^3 problem that
        // touch it, in ascending global element index: the order the
        // single-rank loop above produces for the undecomposed mesh.
        for (int pz = 0, n = 0; pz < en; ++pz)
            for (int py = 0; py < en; ++py)
                for (int px = 0; px < en; ++px, ++n) {
                    const int gx = col * nx + px, gy = row * nx + py, gz = plane * nx + pz;
                    double m = 0.0;
                    for (int ez = gz - 1; ez <= gz; ++ez)
                        for (int ey = gy - 1; ey <= gy; ++ey)
                            for (int ex = gx - 1; ex <= gx; ++ex) {
                                if (ex < 0 || ey < 0 || ez < 0 || ex >= meshEdge ||
                                    ey >= meshEdge || ez >= meshEdge)
                                    continue;
                                m += volume_of(ex, ey, ez) / 8.0;
                            }
                    d.nodalMass[n] = m;
                }
    }

    // energy deposit and initial dt, lulesh.cu:1189-1205
    d.e.assign(E, 0.0);
    const double ebase = 3.948746e+7;
    double scale = (nx * tp) / 45.0;
    d.einit = ebase * scale * scale * scale;
    if (row + col + plane == 0) d.e[0] = d.einit;
    d.deltatime = (.5 * cbrt(d.volo[0])) / sqrt(2 * d.einit);

    build_regions(d, numReg, balance);
}

// ---- unstructured input (lmesh) --------------------------------------------

namespace {

// whitespace-separated integers and doubles of an lmesh file
struct LmeshReader {
    std::FILE *f = nullptr;
    bool ok = true;
    ~LmeshReader()
    {
        if (f) std::fclose(f);
    }
    int i()
    {
        int v = 0;
        if (ok && std::fscanf(f, "%d", &v) != 1) ok = false;
        return v;
    }
    double r()
    {
        double v = 0;
        if (ok && std::fscanf(f, "%lf", &v) != 1) ok = false;
        return v;
    }
};

// boundary bits of every element whose whole face lies in the node set
// (the face tests of lulesh.cu:1001-1012); m/p = bits of the min/max faces
void mark_faces(const HostDomain &d, const std::vector<char> &in_set, int zm, int zp, int em,
                int ep, int xm, int xp, std::vector<int> &bc)
{
    for (int z = 0; z < d.numElem; ++z) {
        int mask = 0;
        for (int k = 0; k < 8; ++k)
            mask |= (in_set[d.nodelist[(size_t)k * d.Ep + z]] ? 1 : 0) << k;
        if ((mask & 0x0f) == 0x0f) bc[z] |= zm;
        if ((mask & 0xf0) == 0xf0) bc[z] |= zp;
        if ((mask & 0x33) == 0x33) bc[z] |= em;
        if ((mask & 0xcc) == 0xcc) bc[z] |= ep;
        if ((mask & 0x99) == 0x99) bc[z] |= xm;
        if ((mask & 0x66) == 0x66) bc[z] |= xp;
    }
}

}  // namespace

bool build_domain_lmesh(HostDomain &d, const char *path, int numReg, int balance, int cost,
                        std::string *err)
{
    auto fail = [&](const std::string &m) {
        if (err) *err = std::string("lmesh ") + path + ": " + m;
        return false;
    };
    LmeshReader in;
    in.f = std::fopen(path, "r");
    if (!in.f) return fail("cannot open");
    const int E = in.i(), N = in.i();
    if (!in.ok || E < 1 || N < 8 || E > (1 << 27) || N > (1 << 28))
        return fail("bad element/node counts");
    d = HostDomain{};
    d.unstructured = true;
    d.nx = 0;
    d.en = 0;
    d.tp = 1;
    d.cost = cost;
    d.numElem = E;
    d.numNode = N;
    d.Ep = ((E + 31) / 32) * 32;
    d.allElem = E;
    for (int f = 0; f < 6; ++f) d.ghost[f] = -1;
    d.x.resize(N);
    d.y.resize(N);
    d.z.resize(N);
    for (int n = 0; n < N; ++n) {
        d.x[n] = in.r();
        d.y[n] = in.r();
        d.z[n] = in.r();
    }
    d.nodelist.assign(8 * (size_t)d.Ep, 0);
    for (int z = 0; z < E; ++z)
        for (int k = 0; k < 8; ++k) {
            const int n = in.i();
            if (n < 0 || n >= N) return fail("node id out of range in element " + std::to_string(z));
            d.nodelist[(size_t)k * d.Ep + z] = n;
        }
    std::vector<int> *links[6] = {&d.lxim, &d.lxip, &d.letam, &d.letap, &d.lzetam, &d.lzetap};
    for (auto *l : links) l->resize(E);
    for (int z = 0; z < E; ++z)
        for (auto *l : links) {
            const int v = in.i();
            if (v < 0 || v >= E) return fail("face neighbour out of range in element " +
                                             std::to_string(z));
            (*l)[z] = v;
        }
    std::vector<int> *sets[3] = {&d.symmX, &d.symmY, &d.symmZ};
    int *counts[3] = {&d.numSymmX, &d.numSymmY, &d.numSymmZ};
    d.nodeBC.assign(N, 0);
    std::vector<char> symm(N, 0), freesurf(N, 0);
    for (int a = 0; a < 3; ++a) {
        const int c = in.i();
        if (!in.ok || c < 0 || c > N) return fail("bad symmetry set size");
        *counts[a] = c;
        sets[a]->resize(c);
        for (int k = 0; k < c; ++k) {
            const int n = in.i();
            if (n < 0 || n >= N) return fail("symmetry node out of range");
            (*sets[a])[k] = n;
            symm[n] = 1;
            d.nodeBC[n] |= 1 << a;
        }
    }
    const int nfree = in.i();
    if (!in.ok || nfree < 0 || nfree > N) return fail("bad free-surface set size");
    for (int k = 0; k < nfree; ++k) {
        const int n = in.i();
        if (n < 0 || n >= N) return fail("free-surface node out of range");
        freesurf[n] = 1;
    }
    if (!in.ok) return fail("truncated");
    // device arrays of the symmetry sets share one size
    int en2 = 1;
    for (int a = 0; a < 3; ++a) en2 = std::max(en2, *counts[a]);
    for (auto *v : sets) v->resize(en2, 0);

    d.elemBC.assign(E, 0);
    mark_faces(d, symm, ZETA_M_SYMM, ZETA_P_SYMM, ETA_M_SYMM, ETA_P_SYMM, XI_M_SYMM, XI_P_SYMM,
               d.elemBC);
    d.octantCorner = 0;
    for (int z = 0; z < E; ++z)
        if (d.elemBC[z] == (XI_M_SYMM | ETA_M_SYMM | ZETA_M_SYMM)) {
            d.octantCorner = z;
            break;
        }
    mark_faces(d, freesurf, ZETA_M_FREE, ZETA_P_FREE, ETA_M_FREE, ETA_P_FREE, XI_M_FREE,
               XI_P_FREE, d.elemBC);

    build_corner_csr(d);
    // the corner runs again, slot-major, for the nodal kernel's coalesced
    // reads (meshes where no node has more than 8 corners)
    if (*std::max_element(d.nodeElemCount.begin(), d.nodeElemCount.end()) <= 8) {
        d.nodeCornerEll.assign((size_t)8 * N, -1);
        for (int n = 0; n < N; ++n)
            for (int j = 0; j < d.nodeElemCount[n]; ++j)
                d.nodeCornerEll[(size_t)j * N + n] = d.nodeElemCornerList[d.nodeElemStart[n] + j];
    }
    d.matElemlist.resize(E);
    for (int z = 0; z < E; ++z) d.matElemlist[z] = z;
    d.volo.resize(E);
    d.elemMass.resize(E);
    d.nodalMass.assign(N, 0.0);
    for (int z = 0; z < E; ++z) {
        double xl[8], yl[8], zl[8];
        for (int k = 0; k < 8; ++k) {
            const int g = d.nodelist[(size_t)k * d.Ep + z];
            xl[k] = d.x[g];
            yl[k] = d.y[g];
            zl[k] = d.z[g];
        }
        const double vol = elem_volume_host(xl, yl, zl);
        d.volo[z] = vol;
        d.elemMass[z] = vol;
        for (int k = 0; k < 8; ++k) d.nodalMass[d.nodelist[(size_t)k * d.Ep + z]] += vol / 8.0;
    }
    d.e.assign(E, 0.0);
    d.einit = 3.948746e+7;
    d.e[d.octantCorner] = d.einit;
    d.deltatime = (.5 * cbrt(d.volo[d.octantCorner])) / sqrt(2 * d.einit);
    build_regions(d, numReg, balance);
    return true;
}

void build_domain_light(HostDomain &d, int nx, int numReg, int balance, int cost)
{
    const int en = nx + 1;
    d.nx = nx;
    d.en = en;
    d.tp = 1;
    d.col = d.row = d.plane = d.rank = 0;
    d.cost = cost;
    d.numElem = nx * nx * nx;
    d.Ep = ((d.numElem + 31) / 32) * 32;
    d.numNode = en * en * en;
    d.rowMin = d.rowMax = d.colMin = d.colMax = d.planeMin = d.planeMax = 0;
    d.allElem = d.numElem + 6 * nx * nx;
    d.numSymmX = d.numSymmY = d.numSymmZ = en * en;
    for (int f = 0; f < 6; ++f) d.ghost[f] = -1;
    d.device_geometry = true;
    // volume of element 0 for the initial dt (the corner at the origin)
    double xl[8], yl[8], zl[8];
    const int dx[8] = {0, 1, 1, 0, 0, 1, 1, 0};
    const int dy[8] = {0, 0, 1, 1, 0, 0, 1, 1};
    const int dz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    for (int k = 0; k < 8; ++k) {
        xl[k] = lattice(dx[k], nx);
        yl[k] = lattice(dy[k], nx);
        zl[k] = lattice(dz[k], nx);
    }
    const double volo0 = elem_volume_host(xl, yl, zl);
    const double ebase = 3.948746e+7;
    double scale = nx / 45.0;
    d.einit = ebase * scale * scale * scale;
    d.deltatime = (.5 * cbrt(volo0)) / sqrt(2 * d.einit);
    build_region_runs(d, numReg, balance);
}

double origin_deltatime(int nx, int tp)
{
    // the origin domain's volo[0] and einit, as build_domain computes them
    const int meshEdge = nx * tp;
    double xl[8], yl[8], zl[8];
    const int dx[8] = {0, 1, 1, 0, 0, 1, 1, 0};
    const int dy[8] = {0, 0, 1, 1, 0, 0, 1, 1};
    const int dz[8] = {0, 0, 0, 0, 1, 1, 1, 1};
    for (int k = 0; k < 8; ++k) {
        xl[k] = lattice(dx[k], meshEdge);
        yl[k] = lattice(dy[k], meshEdge);
        zl[k] = lattice(dz[k], meshEdge);
    }
    const double volo0 = elem_volume_host(xl, yl, zl);
    const double ebase = 3.948746e+7;
    double scale = (nx * tp) / 45.0;
    const double einit = ebase * scale * scale * scale;
    return (.5 * cbrt(volo0)) / sqrt(2 * einit);
}

}  // namespace lulesh
