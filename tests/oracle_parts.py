"""A part of a decomposed problem stepped by the CPU oracle (test helper).

`OraclePart` offers the interface distributed.Engine drives (phase, pack,
unpack, dt_pack, dt_unpack, finish_setup, send/recv buffers), with the
oracle's subdomains (oracle_create with tp, col, row, plane) in place of the
GPU set: each subdomain steps phase by phase and reads its neighbours
through mirrors -- a local neighbour's own arrays, or a proxy that the
messages fill.  What the tests check is the product's exchange layer (the
message plan of lulesh_halo_plan and the engine/transports of
distributed.py): with it, the decomposed oracle run must equal the
single-domain oracle run bit for bit, as the GPU's decomposed run does.
"""
from __future__ import annotations

import numpy as np
import torch

import distributed as D
import lulesh_b200 as L
import oracle

INT_MAX = 2**31 - 1
PROXY_SIZES = {"x": "N", "y": "N", "z": "N", "xd": "N", "yd": "N", "zd": "N",
               "fx_elem": "C", "fy_elem": "C", "fz_elem": "C",
               "delv_xi": "E", "delv_eta": "E", "delv_zeta": "E", "volo": "E"}


def rank_pos(r: int, tp: int) -> tuple[int, int, int]:
    return r % tp, (r // tp) % tp, r // (tp * tp)


def direction(dx: int, dy: int, dz: int) -> int:
    return (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1)


class OraclePart:
    def __init__(self, nx: int, tp: int, nparts: int, part: int, numReg: int = 11):
        self.nx, self.tp, self.nparts, self.part = nx, tp, nparts, part
        T = tp ** 3
        self.ranks = [r for r in range(T) if D.part_of(r, tp, nparts) == part]
        self.doms = {r: oracle.Oracle(nx, numReg, 1, 1, tp, *rank_pos(r, tp), r)
                     for r in self.ranks}
        self.arrays = {r: {f: self.doms[r].view(f) for f in PROXY_SIZES} for r in self.ranks}
        E, N = nx ** 3, (nx + 1) ** 3
        Ep = (E + 31) // 32 * 32
        size = {"N": N, "E": E, "C": 8 * Ep}
        self.proxies = {}
        for r in self.ranks:
            c, w, p = rank_pos(r, tp)
            for dz in (-1, 0, 1):
                for dy in (-1, 0, 1):
                    for dx in (-1, 0, 1):
                        nc, nw, npl = c + dx, w + dy, p + dz
                        if (dx, dy, dz) == (0, 0, 0) or not (0 <= nc < tp and 0 <= nw < tp
                                                            and 0 <= npl < tp):
                            continue
                        n = nc + tp * (nw + tp * npl)
                        if n in self.doms:
                            arrays = self.arrays[n]
                        else:
                            if n not in self.proxies:
                                self.proxies[n] = {f: np.zeros(size[k])
                                                   for f, k in PROXY_SIZES.items()}
                            arrays = self.proxies[n]
                        self.doms[r].set_mirror(direction(dx, dy, dz), arrays)
        # every subdomain starts from the origin domain's dt
        dt0 = oracle.Oracle(nx, numReg, 1, 1, tp, 0, 0, 0, 0).scalar("initial_deltatime")
        for d in self.doms.values():
            d.set_deltatime(dt0)
        self.peers = D.peers(tp, nparts, part)
        self.plans, self.send, self.recv = {}, {}, {}
        for k in D.KINDS:
            self.send[k], self.recv[k] = {}, {}
            for q in self.peers:
                self.plans[(k, q, "send")] = D.plan(nx, tp, nparts, part, q, k)
                self.plans[(k, q, "recv")] = D.plan(nx, tp, nparts, q, part, k)
                self.send[k][q] = torch.zeros(len(self.plans[(k, q, "send")][0]),
                                              dtype=torch.float64)
                self.recv[k][q] = torch.zeros(len(self.plans[(k, q, "recv")][0]),
                                              dtype=torch.float64)
        self.dt = torch.zeros(4, dtype=torch.int64)

    def phase(self, ph: int) -> None:
        for r in self.ranks:
            st = self.doms[r].phase(ph)
            if st != 0:
                raise RuntimeError(f"oracle phase {ph} of rank {r}: status {st}")

    def pack(self, kind: int) -> None:
        for q in self.peers:
            ranks, fields, idx = self.plans[(kind, q, "send")]
            out = self.send[kind][q].numpy()
            for r in np.unique(ranks):
                for f in np.unique(fields[ranks == r]):
                    m = (ranks == r) & (fields == f)
                    out[m] = self.arrays[int(r)][L.FIELD_NAMES[int(f)]][idx[m]]

    def unpack(self, kind: int) -> None:
        for q in self.peers:
            ranks, fields, idx = self.plans[(kind, q, "recv")]
            buf = self.recv[kind][q].numpy()
            for r in np.unique(ranks):
                for f in np.unique(fields[ranks == r]):
                    m = (ranks == r) & (fields == f)
                    self.proxies[int(r)][L.FIELD_NAMES[int(f)]][idx[m]] = buf[m]

    def dt_pack(self):
        dtc = min(d.scalar("dtcourant") for d in self.doms.values())
        dth = min(d.scalar("dthydro") for d in self.doms.values())
        bad = [int(d.scalar("bad_vol")) for d in self.doms.values()]
        badq = [int(d.scalar("bad_q")) for d in self.doms.values()]
        bv = min([b for b in bad if b >= 0], default=INT_MAX)
        bq = min([b for b in badq if b >= 0], default=INT_MAX)
        bits = np.array([dtc, dth], dtype=np.float64).view(np.int64)
        self.dt.copy_(torch.tensor([int(bits[0]), int(bits[1]), bv, bq], dtype=torch.int64))
        return self.dt

    def dt_unpack(self, buf) -> None:
        v = buf.numpy()
        dtc, dth = np.array(v[:2], dtype=np.int64).view(np.float64)
        if v[2] != INT_MAX or v[3] != INT_MAX:
            raise RuntimeError(f"a part reported an error: {v.tolist()}")
        for d in self.doms.values():
            d.set_dt_minima(float(dtc), float(dth))

    def finish_setup(self) -> None:
        for d in self.doms.values():
            d.nodal_mass_decomposed()


def compare_with_single(part: OraclePart, single: oracle.Oracle) -> list[str]:
    """Fields of every subdomain of `part` against the single-domain run's
    region they cover; returns the fields that differ in any bit."""
    nx, tp = part.nx, part.tp
    G, en = nx * tp, nx + 1
    bad = []
    elem = ["e", "p", "q", "v", "ss", "delv", "vdov", "arealg", "volo", "elemMass"]
    node = ["x", "y", "z", "xd", "yd", "zd", "nodalMass"]
    ref = {f: single.field(f) for f in elem + node}
    ie = np.arange(nx)
    ine = np.arange(en)
    for r, d in part.doms.items():
        c, w, p = rank_pos(r, tp)
        ge = (((p * nx + ie[:, None, None]) * G + (w * nx + ie[None, :, None])) * G
              + (c * nx + ie[None, None, :])).ravel()
        gn = (((p * nx + ine[:, None, None]) * (G + 1) + (w * nx + ine[None, :, None])) * (G + 1)
              + (c * nx + ine[None, None, :])).ravel()
        for f in elem:
            if not np.array_equal(d.field(f)[:nx ** 3], ref[f][ge]):
                bad.append(f"rank {r} {f}")
        for f in node:
            if not np.array_equal(d.field(f), ref[f][gn]):
                bad.append(f"rank {r} {f}")
    return bad
