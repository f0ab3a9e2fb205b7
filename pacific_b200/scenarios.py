"""Seeded synthetic inputs for the Grains3D DEM step, written as Grains3D XML
(the reference's input format) plus the initial particle state.

The workloads follow the configurations the DEM step is measured on:

* ``settling_box``   - monodisperse spheres settling in a closed box with six
  planar walls (1,000 spheres, r = 1 mm, box 0.03 x 0.03 x 0.06 m, jittered
  cubic lattice of spacing 2.4 mm, HookeMemory kn = 1e4, en = 0.7, etat = 0,
  muc = 0.5, kt = 2/7 kn, dt = 1e-5 s).
* ``periodic_gas``   - polydisperse spheres (r uniform in [0.8, 1.2] mm,
  quantised to 256 radius classes) in a triply periodic cube at solid
  fraction ~0.45, Maxwellian velocities (sigma = 0.1 m/s), no gravity,
  HookeMemory kn = 1e5, en = 0.9, muc = 0.3, kt = 2/7 kn, dt = 5e-6 s.  Random
  sequential insertion jams near 0.38, so the positions are an FCC lattice of
  nearest-neighbour spacing 2.392 mm (n_fcc^3 * 4 sites) with radii redrawn
  until every lattice-neighbour pair has a gap; n_fcc = 63 gives the
  1,000,000-particle case (188 sites dropped at random).
* ``batched_boxes``  - independent closed-box settling instances with their
  own particle counts, radii and contact parameters.
* ``adjoint_box``    - 4,096 spheres in a 0.02 x 0.02 x 0.08 m box on an FCC
  lattice of 2.1 mm spacing with uniform +-0.2 m/s velocities.

All are deterministic functions of their seed.  The crust thickness, which
Grains3D requires, is 0.1 x radius.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np


def _f(v) -> str:
    """Shortest round-trip decimal form of a float."""
    return repr(float(v))


@dataclass
class Scenario:
    name: str
    origin: tuple
    maxc: tuple
    periodic: tuple
    gravity: tuple
    dt: float
    # particle classes: dicts with radius, crust, density, material
    types: list
    # walls: dicts with centre (3), size (LX, LY, LZ), crust, material
    walls: list
    # contact models: dicts with matA, matB, kn, en, etat (None = default), muc, kt
    models: list
    type: np.ndarray = field(repr=False)
    x: np.ndarray = field(repr=False)
    v: np.ndarray = field(repr=False)
    w: np.ndarray = field(repr=False)
    q: np.ndarray = field(repr=False)
    cell_size_factor: float = 1.0

    @property
    def n(self) -> int:
        return len(self.type)

    def counts(self) -> np.ndarray:
        return np.bincount(self.type, minlength=len(self.types))

    def xml(self) -> str:
        """Grains3D XML input (Grains3D/Construction/...; Grains.cpp:535-1030)."""
        ox, oy, oz = self.origin
        mx, my, mz = self.maxc
        px, py, pz = (int(p) for p in self.periodic)
        cnt = self.counts()
        L = ['<Grains3D Type="Standard">', "  <Construction>",
             f'    <LinkedCell MX="{_f(mx)}" MY="{_f(my)}" MZ="{_f(mz)}" '
             f'CellSizeFactor="{_f(self.cell_size_factor)}"/>',
             f'    <Origin OX="{_f(ox)}" OY="{_f(oy)}" OZ="{_f(oz)}"/>',
             f'    <Periodicity PX="{px}" PY="{py}" PZ="{pz}"/>',
             "    <Particles>"]
        for k, t in enumerate(self.types):
            shape = t.get("shape", "sphere")
            if shape == "box":
                s = t["size"]
                geo = f'          <Box LX="{_f(s[0])}" LY="{_f(s[1])}" LZ="{_f(s[2])}"/>'
            elif shape == "polyhedron":
                geo = f'          <Polyhedron Name="{t["file"]}"/>'
            elif shape == "cylinder":
                geo = (f'          <Cylinder Radius="{_f(t["cyl_radius"])}" '
                       f'Height="{_f(t["height"])}"/>')
            else:
                geo = f'          <Sphere Radius="{_f(t["radius"])}"/>'
            L += [f'      <Particle Number="{int(cnt[k])}" Density="{_f(t["density"])}">',
                  f'        <Convex CrustThickness="{_f(t["crust"])}">',
                  geo,
                  "        </Convex>",
                  '        <AngularPosition Type="Identity"></AngularPosition>',
                  f'        <Material>{t["material"]}</Material>',
                  "      </Particle>"]
        L.append("    </Particles>")
        if self.walls:
            L += ["    <Obstacles>", '      <Composite name="Box">']
            for k, w in enumerate(self.walls):
                c, s = w["centre"], w["size"]
                L += [f'        <Obstacle name="Wall{k}" Type="Standard">',
                      f'          <Convex CrustThickness="{_f(w["crust"])}">',
                      f'            <Box LX="{_f(s[0])}" LY="{_f(s[1])}" LZ="{_f(s[2])}"/>',
                      "          </Convex>",
                      f'          <Centre X="{_f(c[0])}" Y="{_f(c[1])}" Z="{_f(c[2])}"/>',
                      '          <AngularPosition Type="Identity"></AngularPosition>',
                      f'          <Material>{w["material"]}</Material>',
                      "        </Obstacle>"]
            L += ["      </Composite>", "    </Obstacles>"]
        L.append("    <ContactForceModels>")
        for m in self.models:
            law = m.get("law", "HookeMemory")
            L += ["      <ContactForceModel>",
                  f'        <Material materialA="{m["matA"]}" materialB="{m["matB"]}"/>',
                  f"        <{law}>",
                  f'          <kn>{_f(m["kn"])}</kn>',
                  f'          <en>{_f(m["en"])}</en>']
            if m.get("etat") is not None:
                L.append(f'          <etat>{_f(m["etat"])}</etat>')
            L.append(f'          <muc>{_f(m["muc"])}</muc>')
            if law == "Hooke":
                # HookeContactForceModel::defineParameters requires <kr>
                L += [f'          <kr>{_f(m.get("kr", 0.0))}</kr>', "        </Hooke>",
                      "      </ContactForceModel>"]
                continue
            L.append(f'          <kt>{_f(m["kt"])}</kt>')
            if m.get("mur"):
                L.append(f'          <mur>{_f(m["mur"])}</mur>')
            if m.get("epst") is not None:
                L.append(f'          <epst>{_f(m["epst"])}</epst>')
            L += ["        </HookeMemory>", "      </ContactForceModel>"]
        gx, gy, gz = self.gravity
        L += ["    </ContactForceModels>", "  </Construction>", "  <Forces>",
              f'    <Gravity GX="{_f(gx)}" GY="{_f(gy)}" GZ="{_f(gz)}"/>', "  </Forces>",
              "  <Simulation>",
              f'    <TimeInterval Start="0." End="{_f(self.dt * 1000)}"/>',
              f'    <TimeStep dt="{_f(self.dt)}"/>', "  </Simulation>", "</Grains3D>", ""]
        return "\n".join(L)

    def write_xml(self, path) -> Path:
        p = Path(path)
        p.write_text(self.xml())
        return p


def _box_walls(L, thickness, crust, material):
    """Six axis-aligned walls just outside [0, L] on each face."""
    Lx, Ly, Lz = L
    t = thickness
    walls = []
    for d in range(3):
        for side in (0, 1):
            c = [Lx / 2, Ly / 2, Lz / 2]
            s = [Lx + 2 * t, Ly + 2 * t, Lz + 2 * t]
            c[d] = -t / 2 if side == 0 else L[d] + t / 2
            s[d] = t
            walls.append(dict(centre=tuple(c), size=tuple(s), crust=crust, material=material))
    return walls


def settling_box(n=1000, seed=1235, box=(0.03, 0.03, 0.06), radius=1.0e-3, spacing=2.4e-3,
                 jitter=1.0e-4, vmax=0.05, kn=1.0e4, en=0.7, etat=0.0, muc=0.5,
                 dt=1.0e-5, density=2500.0, law="HookeMemory", kr=0.0) -> Scenario:
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(np.floor(b / spacing)) for b in box)
    if n > nx * ny * nz:
        raise ValueError("lattice too small")
    k, j, i = np.unravel_index(np.arange(n), (nz, ny, nx))
    x = np.stack([(i + 0.5) * spacing, (j + 0.5) * spacing, (k + 0.5) * spacing], axis=1)
    x = x + rng.uniform(-jitter, jitter, size=x.shape)
    v = rng.uniform(-vmax, vmax, size=(n, 3))
    w = np.zeros((n, 3))
    q = np.zeros((n, 4)); q[:, 3] = 1.0
    crust = 0.1 * radius
    types = [dict(radius=radius, crust=crust, density=density, material="matP")]
    walls = _box_walls(box, 2.0e-3, crust, "matW")
    kt = 2.0 / 7.0 * kn
    models = [dict(matA="matP", matB="matP", kn=kn, en=en, etat=etat, muc=muc, kt=kt, law=law,
                   kr=kr),
              dict(matA="matP", matB="matW", kn=kn, en=en, etat=etat, muc=muc, kt=kt, law=law,
                   kr=kr)]
    return Scenario("settling_box", (0.0, 0.0, 0.0), tuple(box), (0, 0, 0), (0.0, 0.0, -9.81), dt,
                    types, walls, models, np.zeros(n, np.int32), x, v, w, q)


def fcc_sites(n_fcc, a):
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]])
    g = np.stack(np.meshgrid(np.arange(n_fcc), np.arange(n_fcc), np.arange(n_fcc),
                             indexing="ij"), axis=-1).reshape(-1, 3)
    return ((g[:, None, :] + base[None, :, :]).reshape(-1, 3) + 0.25) * a


def periodic_gas(n_fcc=63, n_target=None, seed=1236, spacing=2.392e-3, rmin=0.8e-3,
                 rmax=1.2e-3, nclasses=256, sigma=0.1, kn=1.0e5, en=0.9, muc=0.3,
                 dt=5.0e-6, density=2500.0) -> Scenario:
    """FCC stand-in for the 1M-sphere granular gas (see module docstring)."""
    rng = np.random.default_rng(seed)
    a = spacing * np.sqrt(2.0)
    side = n_fcc * a
    x = fcc_sites(n_fcc, a)
    nsite = len(x)
    if n_target is None:
        n_target = 1_000_000 if n_fcc == 63 else nsite
    keep = np.sort(rng.permutation(nsite)[:n_target])
    x = x[keep]
    n = len(x)
    # radius classes; redraw until every lattice-neighbour pair keeps a gap
    width = (rmax - rmin) / nclasses
    radii = rmin + (np.arange(nclasses) + 0.5) * width
    cls = rng.integers(0, nclasses, size=n)
    # lattice neighbours through a hash of integer half-lattice coordinates
    half = np.rint((x / a - 0.25) * 2).astype(np.int64)
    m = 2 * n_fcc
    code = (half[:, 0] % m) * m * m + (half[:, 1] % m) * m + (half[:, 2] % m)
    index = -np.ones(m ** 3, np.int64)
    index[code] = np.arange(n)
    nbr_off = np.array([[1, 1, 0], [1, -1, 0], [-1, 1, 0], [-1, -1, 0],
                        [1, 0, 1], [1, 0, -1], [-1, 0, 1], [-1, 0, -1],
                        [0, 1, 1], [0, 1, -1], [0, -1, 1], [0, -1, -1]])
    nbrs = np.empty((n, 12), np.int64)
    for k, o in enumerate(nbr_off):
        h2 = (half + o) % m
        nbrs[:, k] = index[h2[:, 0] * m * m + h2[:, 1] * m + h2[:, 2]]
    limit = spacing * (1.0 - 1.0e-6)
    for _ in range(200):
        r = radii[cls]
        rn = np.where(nbrs >= 0, r[np.maximum(nbrs, 0)], 0.0)
        bad = np.any((rn + r[:, None] >= limit) & (nbrs >= 0), axis=1)
        # redraw only the lower index of each offending pair to converge
        idx = np.nonzero(bad)[0]
        if len(idx) == 0:
            break
        cls[idx] = rng.integers(0, nclasses, size=len(idx))
    else:
        raise RuntimeError("radius redraw did not converge")
    used = np.unique(cls)
    remap = -np.ones(nclasses, np.int64)
    remap[used] = np.arange(len(used))
    type_ = remap[cls].astype(np.int32)
    types = [dict(radius=float(radii[c]), crust=float(0.1 * radii[c]), density=density,
                  material="matP") for c in used]
    v = rng.normal(0.0, sigma, size=(n, 3))
    v -= v.mean(axis=0)
    w = np.zeros((n, 3))
    q = np.zeros((n, 4)); q[:, 3] = 1.0
    models = [dict(matA="matP", matB="matP", kn=kn, en=en, etat=None, muc=muc,
                   kt=2.0 / 7.0 * kn)]
    return Scenario("periodic_gas", (0.0, 0.0, 0.0), (side, side, side), (1, 1, 1),
                    (0.0, 0.0, 0.0), dt, types, [], models, type_, x, v, w, q)


def settling_instance(n, seed, rmin=0.8e-3, rmax=1.2e-3, nclasses=16, phi=0.3, kn=1.0e4,
                      en=0.7, muc=0.5, dt=1.0e-5, vmax=0.05, density=2500.0) -> Scenario:
    """One closed-box instance of the batched sweep: n polydisperse spheres
    (radius uniform in [rmin, rmax], quantised to nclasses classes) on a
    jittered cubic lattice in a cube whose side gives an initial solid
    fraction phi, settling under gravity between six walls."""
    rng = np.random.default_rng(seed)
    width = (rmax - rmin) / nclasses
    radii = rmin + (np.arange(nclasses) + 0.5) * width
    cls = rng.integers(0, nclasses, size=n)
    r = radii[cls]
    side = float((np.sum(4.0 / 3.0 * np.pi * r ** 3) / phi) ** (1.0 / 3.0))
    # FCC sites filling the cube from the bottom (a cubic lattice cannot hold
    # phi = 0.3 with r up to 1.2 mm)
    # (when n is just above 4 m^3 the lattice needs a slightly larger box:
    # the side is then the smallest that keeps every lattice gap open and the
    # achieved solid fraction is a little below phi)
    m = int(np.ceil((n / 4.0) ** (1.0 / 3.0)))
    off = 1.05 * rmax                                     # wall clearance
    a = max((side - 2 * off) / (m - 0.5), 2 * rmax * 1.02 * np.sqrt(2.0))
    side = (m - 0.5) * a + 2 * off
    nn = a / np.sqrt(2.0)
    sites = fcc_sites(m, a) - 0.25 * a + off
    order = np.lexsort((sites[:, 0], sites[:, 1], sites[:, 2]))
    x = sites[order[:n]]
    jit = min(0.3 * (nn - 2 * rmax), 0.4 * (off - rmax))
    x = x + rng.uniform(-jit, jit, size=x.shape)
    v = rng.uniform(-vmax, vmax, size=(n, 3))
    used = np.unique(cls)
    remap = -np.ones(nclasses, np.int64)
    remap[used] = np.arange(len(used))
    types = [dict(radius=float(radii[c]), crust=float(0.1 * radii[c]), density=density,
                  material="matP") for c in used]
    kt = 2.0 / 7.0 * kn
    models = [dict(matA="matP", matB="matP", kn=kn, en=en, etat=None, muc=muc, kt=kt),
              dict(matA="matP", matB="matW", kn=kn, en=en, etat=None, muc=muc, kt=kt)]
    walls = _box_walls((side, side, side), 2.0e-3, float(0.1 * rmin), "matW")
    q = np.zeros((n, 4)); q[:, 3] = 1.0
    return Scenario("settling_instance", (0.0, 0.0, 0.0), (side, side, side), (0, 0, 0),
                    (0.0, 0.0, -9.81), dt, types, walls, models, remap[cls].astype(np.int32), x,
                    v, np.zeros((n, 3)), q)


def batched_boxes(n_inst=512, seed=1237, nmin=500, nmax=20000, dt=1.0e-5):
    """Independent closed-box settling instances with their own particle
    count (uniform in [nmin, nmax]), radii and contact parameters (kn
    log-uniform in [1e3, 1e5], en uniform in [0.3, 0.95], muc uniform in
    [0.1, 0.8]); instance k uses seed + k."""
    out = []
    for k in range(n_inst):
        rng = np.random.default_rng(seed + k)
        n = int(rng.integers(nmin, nmax + 1))
        kn = float(10.0 ** rng.uniform(3.0, 5.0))
        en = float(rng.uniform(0.3, 0.95))
        muc = float(rng.uniform(0.1, 0.8))
        out.append(settling_instance(n, seed + 100000 + k, kn=kn, en=en, muc=muc, dt=dt))
    return out


def concat_state(instances):
    """Stacked (inst, type, x, v, w, q) of a batch, grouped by instance."""
    inst = np.concatenate([np.full(s.n, k, np.int32) for k, s in enumerate(instances)])
    cat = lambda a: np.concatenate([getattr(s, a) for s in instances])
    return inst, cat("type").astype(np.int32), cat("x"), cat("v"), cat("w"), cat("q")


def write_tetrahedron(path, edge=3.0e-3) -> Path:
    """Regular tetrahedron with its centroid at the origin, in the polyhedron
    file layout Grains3D reads (Polyhedron::create): '3 <nv>', vertices,
    '<nf>', one line of vertex indices per face."""
    a = edge / (2.0 * np.sqrt(2.0))
    verts = [(a, a, a), (a, -a, -a), (-a, a, -a), (-a, -a, a)]
    faces = [(0, 1, 2), (0, 3, 1), (0, 2, 3), (1, 3, 2)]
    lines = ["3 4"] + [" ".join(_f(c) for c in v) for v in verts] + ["4"] + \
            [" ".join(str(i) for i in f) for f in faces]
    p = Path(path)
    p.write_text("\n".join(lines) + "\n")
    return p


def random_quaternions(rng, n):
    """Uniform random unit quaternions (Shoemake), as (qx, qy, qz, qw)."""
    u1, u2, u3 = rng.random(n), rng.random(n), rng.random(n)
    q = np.stack([np.sqrt(1 - u1) * np.sin(2 * np.pi * u2), np.sqrt(1 - u1) * np.cos(2 * np.pi * u2),
                  np.sqrt(u1) * np.sin(2 * np.pi * u3), np.sqrt(u1) * np.cos(2 * np.pi * u3)], axis=1)
    return q


def rotation_matrices(q):
    """Row-major rotation matrices of unit quaternions (qx, qy, qz, qw), with
    the expression order of Matrix::setRotation (Geometry/src/Matrix.cpp:114-127)."""
    x, y, z, w = q[:, 0], q[:, 1], q[:, 2], q[:, 3]
    d = x * x + y * y + z * z + w * w
    s = 2.0 / d
    xs, ys, zs = x * s, y * s, z * s
    wx, wy, wz = w * xs, w * ys, w * zs
    xx, xy, xz = x * xs, x * ys, x * zs
    yy, yz, zz = y * ys, y * zs, z * zs
    return np.stack([1.0 - (yy + zz), xy - wz, xz + wy, xy + wz, 1.0 - (xx + zz), yz - wx,
                     xz - wy, yz + wx, 1.0 - (xx + yy)], axis=1)


def convex_pour(n=200_000, seed=1238, poly_path=None, box=(0.1, 0.1, 0.3), cube_edge=2.0e-3,
                tet_edge=3.0e-3, density=2000.0, kn=5.0e4, en=0.5, muc=0.4, dt=2.0e-6,
                vmax=0.0, cylinders=False) -> Scenario:
    """Half cubes, half regular tetrahedra with uniformly random orientations
    on a jittered lattice of spacing 1.02 x the tetrahedron's circumscribed
    diameter, poured under gravity into an open-top box of footprint
    box[0] x box[1].  The lattice does not fit in a box[2]-high container, so
    the side walls and the linked-cell domain extend up to the lattice top.
    With cylinders=True a third class, cylinders of radius 0.8 mm and height
    2 mm, takes a third of the sites."""
    rng = np.random.default_rng(seed)
    r_tet = tet_edge * np.sqrt(6.0) / 4.0
    spacing = 2.0 * r_tet * 1.02
    nx, ny = int(box[0] // spacing), int(box[1] // spacing)
    nz = int(np.ceil(n / (nx * ny)))
    height = max(box[2], (nz + 0.5) * spacing)
    k, j, i = np.unravel_index(np.arange(n), (nz, ny, nx))
    x = np.stack([(i + 0.5) * spacing, (j + 0.5) * spacing, (k + 0.5) * spacing], axis=1)
    x[:, 0] += 0.5 * (box[0] - nx * spacing)
    x[:, 1] += 0.5 * (box[1] - ny * spacing)
    jit = 0.2 * (spacing - 2.0 * r_tet)
    x = x + rng.uniform(-jit, jit, size=x.shape)
    v = rng.uniform(-vmax, vmax, size=(n, 3)) if vmax > 0 else np.zeros((n, 3))
    q = random_quaternions(rng, n)
    type_ = (rng.random(n) < 0.5).astype(np.int32)        # 0 cube, 1 tetrahedron
    if cylinders:
        type_ = rng.integers(0, 3, n).astype(np.int32)    # 2 cylinder
    r_cube = cube_edge * np.sqrt(3.0) / 2.0
    types = [dict(shape="box", size=(cube_edge,) * 3, radius=float(r_cube),
                  crust=float(0.1 * r_cube), density=density, material="matP"),
             dict(shape="polyhedron", file=str(poly_path), radius=float(r_tet),
                  crust=float(0.1 * r_tet), density=density, material="matP")]
    if cylinders:
        rc, hc = 0.8e-3, 2.0e-3
        r_cyl = float(np.hypot(rc, 0.5 * hc))
        types.append(dict(shape="cylinder", cyl_radius=rc, height=hc, radius=r_cyl,
                          crust=float(0.1 * r_cyl), density=density, material="matP"))
    dom = (box[0], box[1], height)
    walls = _box_walls(dom, 2.0e-3, float(0.1 * r_cube), "matW")
    kt = 2.0 / 7.0 * kn
    models = [dict(matA="matP", matB="matP", kn=kn, en=en, etat=None, muc=muc, kt=kt),
              dict(matA="matP", matB="matW", kn=kn, en=en, etat=None, muc=muc, kt=kt)]
    return Scenario("convex_pour", (0.0, 0.0, 0.0), dom, (0, 0, 0), (0.0, 0.0, -9.81), dt, types,
                    walls, models, type_, x, v, np.zeros((n, 3)), q)


def adjoint_box(n=4096, seed=1239, box=(0.02, 0.02, 0.08), radius=1.0e-3, spacing=2.1e-3,
                jitter=2.5e-5, vmax=0.2, kn=2.0e4, en=0.6, muc=0.35, dt=1.0e-5,
                density=2500.0, gravity=(0.0, 0.0, -9.81)) -> Scenario:
    """The calibration case: spheres of radius 1 mm on an FCC lattice of
    nearest-neighbour spacing 2.1 mm (a cubic lattice of 2.4 mm holds only
    2,112 in the 0.02 x 0.02 x 0.08 m box), centres at least r from the walls,
    the first n sites in (z, y, x) order, jitter up to +-0.025 mm per axis
    (sites closer than r + jitter to a wall are dropped),
    velocities uniform in +-0.2 m/s, HookeMemory with kt = 2/7 kn."""
    rng = np.random.default_rng(seed)
    a = spacing * np.sqrt(2.0)
    base = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) * a
    ncell = [int(np.ceil(b / a)) + 1 for b in box]
    g = np.stack(np.meshgrid(*[np.arange(k) for k in ncell], indexing="ij"), axis=-1).reshape(-1, 3)
    sites = (g[:, None, :] * a + base[None, :, :]).reshape(-1, 3) + (radius + jitter)
    inside = np.all((sites >= radius + jitter) & (sites <= np.array(box) - radius - jitter), axis=1)
    sites = sites[inside]
    order = np.lexsort((sites[:, 0], sites[:, 1], sites[:, 2]))
    sites = sites[order]
    if n > len(sites):
        raise ValueError("lattice too small")
    x = sites[:n] + rng.uniform(-jitter, jitter, size=(n, 3))
    v = rng.uniform(-vmax, vmax, size=(n, 3))
    w = np.zeros((n, 3))
    q = np.zeros((n, 4)); q[:, 3] = 1.0
    crust = 0.1 * radius
    types = [dict(radius=radius, crust=crust, density=density, material="matP")]
    walls = _box_walls(box, 2.0e-3, crust, "matW")
    kt = 2.0 / 7.0 * kn
    models = [dict(matA="matP", matB="matP", kn=kn, en=en, etat=None, muc=muc, kt=kt),
              dict(matA="matP", matB="matW", kn=kn, en=en, etat=None, muc=muc, kt=kt)]
    return Scenario("adjoint_box", (0.0, 0.0, 0.0), tuple(box), (0, 0, 0), tuple(gravity), dt,
                    types, walls, models, np.zeros(n, np.int32), x, v, w, q)


def solid_fraction(sc: Scenario) -> float:
    r = np.array([t["radius"] for t in sc.types])[sc.type]
    vol = np.prod(np.array(sc.maxc) - np.array(sc.origin))
    return float(np.sum(4.0 / 3.0 * np.pi * r ** 3) / vol)
