"""lmesh files: the unstructured mesh format of the reference's `-u` input.

Layout, as the reference's reader consumes it (LULESH/cuda/src/lulesh.cu:855-1052),
all whitespace-separated:

    numElem numNode
    x y z                      numNode lines of node coordinates
    n0 n1 ... n7               numElem lines of node ids (local corner order)
    xi- xi+ eta- eta+ zeta- zeta+   numElem lines of face-neighbour elements
    nX  id ...                 the X symmetry node set (count, then ids)
    nY  id ...                 the Y symmetry node set
    nZ  id ...                 the Z symmetry node set
    nF  id ...                 the free-surface node set

`box(nx)` writes the structured Sedov cube the `-s nx` run builds, with the
same numbering (BuildMesh, lulesh.cu:690-746; the face links of
lulesh.cu:540-571), so a `-u` run of it can be compared with the `-s` run
value for value.  `renumber` relabels nodes and elements of a mesh without
changing its geometry.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass
class LMesh:
    xyz: np.ndarray        # (numNode, 3) float64
    nodelist: np.ndarray   # (numElem, 8) int64, local corner order
    links: np.ndarray      # (numElem, 6) int64: xi-, xi+, eta-, eta+, zeta-, zeta+
    symm: tuple            # three int64 arrays of node ids (X, Y, Z planes)
    free: np.ndarray       # int64 node ids of the free surface

    @property
    def num_elem(self) -> int:
        return int(self.nodelist.shape[0])

    @property
    def num_node(self) -> int:
        return int(self.xyz.shape[0])


def box(nx: int) -> LMesh:
    """The -s nx Sedov cube: nodes at 1.125*g/nx, symmetry planes at 0, the
    free surface at 1.125."""
    en = nx + 1
    g = np.arange(en, dtype=np.float64)
    c = 1.125 * g / float(nx)
    pz, py, px = np.meshgrid(np.arange(en), np.arange(en), np.arange(en), indexing="ij")
    px, py, pz = px.ravel(), py.ravel(), pz.ravel()
    xyz = np.stack([c[px], c[py], c[pz]], axis=1)

    ez, ey, ex = np.meshgrid(np.arange(nx), np.arange(nx), np.arange(nx), indexing="ij")
    n0 = (ex + en * (ey + en * ez)).ravel().astype(np.int64)
    s, p = en, en * en
    nodelist = np.stack([n0, n0 + 1, n0 + s + 1, n0 + s,
                         n0 + p, n0 + p + 1, n0 + p + s + 1, n0 + p + s], axis=1)

    E = nx * nx * nx
    i = np.arange(E, dtype=np.int64)
    lxim = np.maximum(i - 1, 0)
    lxip = np.minimum(i + 1, E - 1)
    letam = np.where(i < nx, i, i - nx)
    letap = np.where(i >= E - nx, i, i + nx)
    a = nx * nx
    lzetam = np.where(i < a, i, i - a)
    lzetap = np.where(i >= E - a, i, i + a)
    links = np.stack([lxim, lxip, letam, letap, lzetam, lzetap], axis=1)

    ids = np.arange(en ** 3, dtype=np.int64)
    symm = (ids[px == 0], ids[py == 0], ids[pz == 0])
    free = ids[(px == nx) | (py == nx) | (pz == nx)]
    return LMesh(xyz, nodelist, links, symm, free)


def renumber(m: LMesh, node_perm: np.ndarray | None = None,
             elem_perm: np.ndarray | None = None) -> LMesh:
    """Relabel: old node n becomes node_perm[n], old element z becomes
    elem_perm[z].  Each element keeps its local corner order."""
    N, E = m.num_node, m.num_elem
    npm = np.arange(N) if node_perm is None else np.asarray(node_perm, dtype=np.int64)
    epm = np.arange(E) if elem_perm is None else np.asarray(elem_perm, dtype=np.int64)
    xyz = np.empty_like(m.xyz)
    xyz[npm] = m.xyz
    nodelist = np.empty_like(m.nodelist)
    nodelist[epm] = npm[m.nodelist]
    links = np.empty_like(m.links)
    links[epm] = epm[m.links]
    symm = tuple(np.sort(npm[s]) for s in m.symm)
    free = np.sort(npm[m.free])
    return LMesh(xyz, nodelist, links, symm, free)


def warp(m: LMesh, amp: float = 0.05) -> LMesh:
    """A curvilinear copy of a box mesh: every node moves by a smooth
    displacement that vanishes on the planes x, y, z = 0 and = max, so the
    symmetry planes and the free surface stay where they were."""
    lo, hi = m.xyz.min(axis=0), m.xyz.max(axis=0)
    u = (m.xyz - lo) / (hi - lo)  # 0..1 per axis
    bump = np.sin(np.pi * u)      # 0 on both end planes
    xyz = m.xyz.copy()
    for a in range(3):
        b, c = (a + 1) % 3, (a + 2) % 3
        xyz[:, a] += amp * (hi[a] - lo[a]) * bump[:, a] * np.sin(2 * np.pi * u[:, b]) * \
            np.cos(np.pi * u[:, c])
    return LMesh(xyz, m.nodelist.copy(), m.links.copy(), m.symm, m.free)


def write(path, m: LMesh) -> None:
    with open(path, "w") as f:
        f.write(f"{m.num_elem} {m.num_node}\n")
        np.savetxt(f, m.xyz, fmt="%.17g")
        np.savetxt(f, m.nodelist, fmt="%d")
        np.savetxt(f, m.links, fmt="%d")
        for ids in (*m.symm, m.free):
            f.write(f"{len(ids)}\n")
            if len(ids):
                np.savetxt(f, np.asarray(ids).reshape(1, -1), fmt="%d")


def read(path) -> LMesh:
    with open(path) as f:
        tok = f.read().split()
    E, N = int(tok[0]), int(tok[1])
    k = 2
    xyz = np.array(tok[k:k + 3 * N], dtype=np.float64).reshape(N, 3)
    k += 3 * N
    nodelist = np.array(tok[k:k + 8 * E], dtype=np.int64).reshape(E, 8)
    k += 8 * E
    links = np.array(tok[k:k + 6 * E], dtype=np.int64).reshape(E, 6)
    k += 6 * E
    sets = []
    for _ in range(4):
        c = int(tok[k])
        sets.append(np.array(tok[k + 1:k + 1 + c], dtype=np.int64))
        k += 1 + c
    return LMesh(xyz, nodelist, links, tuple(sets[:3]), sets[3])
