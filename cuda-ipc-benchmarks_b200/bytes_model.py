"""Bytes per zone-cycle of the LULESH Lagrange step, array by array.

`ALGORITHMIC` is the compulsory FP64 traffic of one cycle: the state that
crosses each of the four grid-wide dependency boundaries (force | node
update | kinematics + monotonic-Q gradient | monotonic-Q region + EOS +
volume + dt), each array read or written once per phase, with nodes counted
one per element (N/E = 1.03 at -s 100).  It is the numerator of the HBM
roofline that bench.py reports.  Index arrays are int32 (4 B), reals FP64.

`THIS_BUILD` adds what this implementation moves beyond that: the force
kernel writes eight corner forces per element (no float atomics) and the
nodal kernel reads them back, in place of the algorithmic 24 B of nodal
force; node indices and face links are computed from the element position
on structured meshes, so nodelist and the links are not read.
"""

R8, I4 = 8, 4

# phase -> (reads, writes): {array: bytes per element}
ALGORITHMIC = {
    "force": (
        {"nodelist": 8 * I4, "x,y,z": 3 * R8, "xd,yd,zd": 3 * R8,
         "p,q": 2 * R8, "v,volo": 2 * R8, "ss,elemMass": 2 * R8},
        {"fx,fy,fz (nodal)": 3 * R8},
    ),
    "nodal": (
        {"fx,fy,fz": 3 * R8, "nodalMass": R8, "x,y,z": 3 * R8, "xd,yd,zd": 3 * R8},
        {"x,y,z": 3 * R8, "xd,yd,zd": 3 * R8},
    ),
    "kinematics": (
        {"nodelist": 8 * I4, "x,y,z": 3 * R8, "xd,yd,zd": 3 * R8, "volo": R8, "v": R8},
        {"vnew,delv,arealg,vdov": 4 * R8, "delv_xi,eta,zeta": 3 * R8,
         "delx_xi,eta,zeta": 3 * R8},
    ),
    "eos": (
        {"elemBC": I4, "lxim..lzetap": 6 * I4, "delv_xi,eta,zeta": 3 * R8,
         "delx_xi,eta,zeta": 3 * R8, "vdov,elemMass,volo,vnew,delv": 5 * R8,
         "e,p,q": 3 * R8, "v": R8, "arealg": R8},
        {"e,p,q": 3 * R8, "v": R8, "ss": R8},
    ),
}


def phase_bytes(model=ALGORITHMIC) -> dict:
    """Bytes per element of each phase (reads + writes)."""
    return {ph: sum(r.values()) + sum(w.values()) for ph, (r, w) in model.items()}


def step_bytes(model=ALGORITHMIC) -> float:
    return float(sum(phase_bytes(model).values()))


def _this_build():
    m = {ph: (dict(r), dict(w)) for ph, (r, w) in ALGORITHMIC.items()}
    for ph in ("force", "kinematics"):
        del m[ph][0]["nodelist"]             # node indices from the element position
    del m["eos"][0]["elemBC"]                # boundary masks and links likewise
    del m["eos"][0]["lxim..lzetap"]
    m["force"][1].clear()
    m["force"][1]["fx,fy,fz_elem (8 corners)"] = 24 * R8
    del m["nodal"][0]["fx,fy,fz"]
    m["nodal"][0]["fx,fy,fz_elem (8 corners)"] = 24 * R8
    return m


THIS_BUILD = _this_build()
