"""ctypes front end of the CPU FP64 restatement (grains_oracle.cpp).

TEST INFRASTRUCTURE: used by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py as the checker; never by the product path.

The configuration is read from the Grains3D XML input with the standard
library's ElementTree, independently of the product's own C++ XML reader, so
the tests also cross-check that reader.  Materials get bits in order of first
definition, particles first and obstacles next
(ContactBuilderFactory::defineMaterial, Component/src/ContactBuilderFactory.cpp:
176-192), and a contact model is keyed by the OR of its two material bits.
"""
from __future__ import annotations

import ctypes
import subprocess
import xml.etree.ElementTree as ET
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle_grains.so"
SRC = HERE / "grains_oracle.cpp"

OR_ERR_CONTACT = 1
OR_ERR_MOTION = 2
OR_ERR_OUT_OF_GRID = 4


def build() -> Path:
    """Compiles the restatement (scalar C++, no FMA contraction)."""
    if not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared",
                        "-o", str(LIB), str(SRC)], check=True)
    return LIB


class _Config(ctypes.Structure):
    _fields_ = [
        ("origin", ctypes.c_double * 3),
        ("maxc", ctypes.c_double * 3),
        ("periodic", ctypes.c_int * 3),
        ("cell_size_factor", ctypes.c_double),
        ("gravity", ctypes.c_double * 3),
        ("dt", ctypes.c_double),
        ("n_types", ctypes.c_int),
        ("type_radius", ctypes.POINTER(ctypes.c_double)),
        ("type_crust", ctypes.POINTER(ctypes.c_double)),
        ("type_density", ctypes.POINTER(ctypes.c_double)),
        ("type_matbit", ctypes.POINTER(ctypes.c_int)),
        ("n_walls", ctypes.c_int),
        ("wall_centre", ctypes.POINTER(ctypes.c_double)),
        ("wall_extent", ctypes.POINTER(ctypes.c_double)),
        ("wall_crust", ctypes.POINTER(ctypes.c_double)),
        ("wall_matbit", ctypes.POINTER(ctypes.c_int)),
        ("n_models", ctypes.c_int),
        ("model_mask", ctypes.POINTER(ctypes.c_int)),
        ("model_params", ctypes.POINTER(ctypes.c_double)),
        ("type_shape", ctypes.POINTER(ctypes.c_int)),
        ("type_extent", ctypes.POINTER(ctypes.c_double)),
        ("type_poly", ctypes.POINTER(ctypes.c_int)),
        ("poly_verts", ctypes.POINTER(ctypes.c_double)),
        ("poly_faces", ctypes.POINTER(ctypes.c_int)),
    ]


_lib = None


def _load():
    global _lib
    if _lib is None:
        lib = ctypes.CDLL(str(build()))
        V = ctypes.c_void_p
        D = ctypes.POINTER(ctypes.c_double)
        I = ctypes.POINTER(ctypes.c_int)
        lib.or_create.argtypes = [ctypes.POINTER(_Config)]
        lib.or_create.restype = V
        lib.or_destroy.argtypes = [V]
        lib.or_set_particles.argtypes = [V, ctypes.c_int, I, D, D, D, D, D]
        lib.or_set_particles.restype = ctypes.c_int
        lib.or_init.argtypes = [V]
        lib.or_init.restype = ctypes.c_int
        lib.or_step.argtypes = [V, ctypes.c_int]
        lib.or_step.restype = ctypes.c_int
        lib.or_get_state.argtypes = [V, D, D, D, D, D, D, D]
        lib.or_get_cells.argtypes = [V, I]
        lib.or_get_curv.argtypes = [V, I]
        lib.or_get_basis.argtypes = [V, D]
        lib.or_get_grid.argtypes = [V, I, D, D]
        lib.or_num_contacts.argtypes = [V]
        lib.or_num_contacts.restype = ctypes.c_int
        lib.or_get_contacts.argtypes = [V, I, I, D, D, D]
        lib.or_num_history.argtypes = [V]
        lib.or_num_history.restype = ctypes.c_int
        lib.or_get_history.argtypes = [V, I, I, D, D, D]
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def read_xml(path):
    """Parses the subset of the Grains3D input the DEM step uses."""
    root = ET.parse(path).getroot()
    cons = root.find("Construction")
    lc = cons.find("LinkedCell")
    o = cons.find("Origin")
    per = cons.find("Periodicity")
    cfg = dict(
        maxc=[float(lc.get(k)) for k in ("MX", "MY", "MZ")],
        origin=[float(o.get(k)) for k in ("OX", "OY", "OZ")] if o is not None else [0.0] * 3,
        periodic=[int(per.get(k)) == 1 for k in ("PX", "PY", "PZ")] if per is not None else [0] * 3,
        cell_size_factor=float(lc.get("CellSizeFactor", "1.")),
    )
    bits = {}

    def matbit(name):
        if name not in bits:
            bits[name] = 1 << len(bits)
        return bits[name]

    types = []
    for p in cons.find("Particles").findall("Particle"):
        cv = p.find("Convex")
        t = dict(crust=float(cv.get("CrustThickness")), density=float(p.get("Density")),
                 matbit=matbit(p.find("Material").text.strip()), shape=0, radius=0.0,
                 extent=[0.0, 0.0, 0.0], verts=[], faces=[])
        if cv.find("Sphere") is not None:
            t["radius"] = float(cv.find("Sphere").get("Radius"))
        elif cv.find("Box") is not None:
            bx = cv.find("Box")
            t["shape"] = 1
            t["extent"] = [0.5 * float(bx.get(k)) for k in ("LX", "LY", "LZ")]
        elif cv.find("Polyhedron") is not None:
            t["shape"] = 2
            t["verts"], t["faces"] = read_poly(cv.find("Polyhedron").get("Name"))
        elif cv.find("Cylinder") is not None:
            cy = cv.find("Cylinder")
            t["shape"] = 3
            r = float(cy.get("Radius"))
            t["extent"] = [r, float(cy.get("Height")) / 2.0, r]
        else:
            raise ValueError("unsupported particle shape")
        types.append(t)
    walls = []
    obs = cons.find("Obstacles")
    if obs is not None:
        for on in obs.iter("Obstacle"):
            cv = on.find("Convex")
            bx = cv.find("Box")
            c = on.find("Centre")
            walls.append(dict(centre=[float(c.get(k)) for k in ("X", "Y", "Z")],
                              extent=[0.5 * float(bx.get(k)) for k in ("LX", "LY", "LZ")],
                              crust=float(cv.get("CrustThickness")),
                              matbit=matbit(on.find("Material").text.strip())))
    models = []
    for cf in cons.find("ContactForceModels"):
        m = cf.find("Material")
        mask = matbit(m.get("materialA")) | matbit(m.get("materialB"))
        law = cf.find("HookeMemory")
        memory = law is not None
        if not memory:
            law = cf.find("Hooke")
        if law is None:
            raise ValueError("only Hooke and HookeMemory contact laws are restated")

        def val(tag, dflt=None):
            e = law.find(tag)
            return float(e.text) if e is not None else dflt

        models.append(dict(mask=mask, params=[val("kn"), val("en"), val("etat", -1.0), val("muc"),
                                              val("kt", 0.0), val("mur", 0.0), val("etarpf", 0.0),
                                              val("epst", 0.0), val("kr", 0.0),
                                              1.0 if memory else 0.0]))
    g = root.find("Forces").find("Gravity")
    cfg.update(types=types, walls=walls, models=models,
               gravity=[float(g.get(k)) for k in ("GX", "GY", "GZ")],
               dt=float(root.find("Simulation").find("TimeStep").get("dt")))
    return cfg


def read_poly(path):
    """Polyhedron file (Polyhedron::create, Geometry/src/Polyhedron.cpp:127-160):
    '<token> <nb_vertices>', one vertex per line, '<nb_faces>', then one line
    of vertex indices per face."""
    lines = Path(path).read_text().splitlines()
    head = lines[0].split()
    nv = int(head[1])
    verts = [[float(x) for x in lines[1 + k].split()] for k in range(nv)]
    nf = int(lines[1 + nv].split()[0])
    faces = [[int(x) for x in lines[2 + nv + k].split()] for k in range(nf)]
    return verts, faces


class Oracle:
    """CPU FP64 restatement of one Grains3D system."""

    def __init__(self, xml_path):
        lib = _load()
        c = read_xml(xml_path)
        self.cfg = c
        self._keep = []

        def arr(vals, dt):
            a = np.ascontiguousarray(vals, dtype=dt).ravel()
            self._keep.append(a)
            return a

        cf = _Config()
        for d in range(3):
            cf.origin[d] = c["origin"][d]
            cf.maxc[d] = c["maxc"][d]
            cf.periodic[d] = int(c["periodic"][d])
            cf.gravity[d] = c["gravity"][d]
        cf.cell_size_factor = c["cell_size_factor"]
        cf.dt = c["dt"]
        T = c["types"]
        cf.n_types = len(T)
        cf.type_radius = _dp(arr([t["radius"] for t in T], np.float64))
        cf.type_crust = _dp(arr([t["crust"] for t in T], np.float64))
        cf.type_density = _dp(arr([t["density"] for t in T], np.float64))
        cf.type_matbit = _ip(arr([t["matbit"] for t in T], np.int32))
        W = c["walls"]
        cf.n_walls = len(W)
        cf.wall_centre = _dp(arr([w["centre"] for w in W] or [[0, 0, 0]], np.float64))
        cf.wall_extent = _dp(arr([w["extent"] for w in W] or [[0, 0, 0]], np.float64))
        cf.wall_crust = _dp(arr([w["crust"] for w in W] or [0], np.float64))
        cf.wall_matbit = _ip(arr([w["matbit"] for w in W] or [0], np.int32))
        cf.type_shape = _ip(arr([t["shape"] for t in T], np.int32))
        cf.type_extent = _dp(arr([t["extent"] for t in T], np.float64))
        tp, pv, pf = [], [], []
        for t in T:
            tp += [len(pv), len(t["verts"]), len(pf), 0]
            pv += t["verts"]
            for f in t["faces"]:
                pf += [len(f)] + list(f)
            tp[-1] = len(pf) - tp[-2]
        cf.type_poly = _ip(arr(tp, np.int32))
        cf.poly_verts = _dp(arr(pv or [[0.0, 0.0, 0.0]], np.float64))
        cf.poly_faces = _ip(arr(pf or [0], np.int32))
        M = c["models"]
        cf.n_models = len(M)
        cf.model_mask = _ip(arr([m["mask"] for m in M], np.int32))
        cf.model_params = _dp(arr([m["params"] for m in M], np.float64))
        self._cf = cf
        self._h = lib.or_create(ctypes.byref(cf))
        self.n = 0

    def close(self):
        if self._h:
            _load().or_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_particles(self, type, x, v, w, q, basis=None):
        n = len(type)
        self._t = np.ascontiguousarray(type, np.int32)
        arrs = [np.ascontiguousarray(a, np.float64) for a in (x, v, w, q)]
        self._b = None if basis is None else np.ascontiguousarray(basis, np.float64).reshape(n, 9)
        rc = _load().or_set_particles(self._h, n, _ip(self._t), *[_dp(a) for a in arrs],
                                      None if self._b is None else _dp(self._b))
        self.n = n
        return rc

    def init(self):
        return _load().or_init(self._h)

    def step(self, nsteps=1):
        return _load().or_step(self._h, nsteps)

    def state(self):
        n = self.n
        out = {k: np.empty((n, 3)) for k in ("x", "v", "w", "wbf", "F", "T")}
        out["q"] = np.empty((n, 4))
        _load().or_get_state(self._h, _dp(out["x"]), _dp(out["v"]), _dp(out["w"]),
                             _dp(out["wbf"]), _dp(out["q"]), _dp(out["F"]), _dp(out["T"]))
        return out

    def basis(self):
        b = np.empty((self.n, 9))
        _load().or_get_basis(self._h, _dp(b))
        return b

    def support_vertices(self):
        """Each particle's polyhedron support vertex (Polyhedron::m_curr_vertex)."""
        out = np.empty(self.n, np.int32)
        _load().or_get_curv(self._h, _ip(out))
        return out

    def cells(self):
        ijk = np.empty((self.n, 3), np.int32)
        _load().or_get_cells(self._h, _ip(ijk))
        return ijk

    def grid(self):
        nb = np.empty(3, np.int32)
        edge = np.empty(3)
        org = np.empty(3)
        _load().or_get_grid(self._h, _ip(nb), _dp(edge), _dp(org))
        return nb, edge, org

    def contacts(self):
        """(id0, id1, delta, point, f) of the last force evaluation; walls as
        id1 = -(k+2)."""
        lib = _load()
        m = lib.or_num_contacts(self._h)
        id0 = np.empty(m, np.int32)
        id1 = np.empty(m, np.int32)
        dl = np.empty(m)
        pt = np.empty((m, 3))
        f = np.empty((m, 3))
        lib.or_get_contacts(self._h, _ip(id0), _ip(id1), _dp(dl), _dp(pt), _dp(f))
        return id0, id1, dl, pt, f

    def history(self):
        lib = _load()
        m = lib.or_num_history(self._h)
        own = np.empty(m, np.int32)
        par = np.empty(m, np.int32)
        kd = np.empty((m, 3))
        pn = np.empty((m, 3))
        sp = np.empty((m, 3))
        lib.or_get_history(self._h, _ip(own), _ip(par), _dp(kd), _dp(pn), _dp(sp))
        return own, par, kd, pn, sp
