"""Scene description and seeded synthetic scenes for the DEM path.

A Scene carries the arguments of the reference's runSimulateCUDA
(src/ParticleStabilizerCUDA/PhysicsEngineCUDA.cpp:86-97): the particle state
in the reference's ParticlePrimitive layout (x, y, z, vx, vy, vz, radius,
mass per row), the box, gravity, wall restitutions in the order zMin, zMax,
xMin, xMax, yMin, yMax, spring and sphere restitution coefficients, dt and an
optional triangle container (9 doubles per triangle).

The generators build the five workloads the path is measured on, from
numpy.random.default_rng(seed).  No public dataset is involved; the shapes,
sizes and value distributions are the workloads' own.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

ZMIN, ZMAX, XMIN, XMAX, YMIN, YMAX = range(6)


@dataclass
class Scene:
    state: np.ndarray                      # (n, 8) float64
    box_min: tuple = (0.0, 0.0, 0.0)
    box_max: tuple = (1.0, 1.0, 1.0)
    gravity: tuple = (0.0, 0.0, -9.8)
    e_wall: tuple = (0.8,) * 6             # zMin, zMax, xMin, xMax, yMin, yMax
    k_spring: float = 1e4
    e_sphere: float = 0.5
    dt: float = 1e-5
    tri: np.ndarray | None = None          # (p, 9) float64
    interval: float = 0.0                  # grid cell; 0 = reference rule 2.1 * r_max
    edge_quirk: int = 1
    widen_domain: int = 0
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n(self) -> int:
        return int(self.state.shape[0])

    def r_max(self) -> float:
        return float(self.state[:, 6].max()) if self.n else 0.0

    def domain(self):
        """Grid domain: the box, or the mesh AABB (optionally widened by the
        initial particle AABB)."""
        if self.tri is None:
            return tuple(self.box_min), tuple(self.box_max)
        v = self.tri.reshape(-1, 3)
        lo, hi = v.min(axis=0), v.max(axis=0)
        if self.widen_domain and self.n:
            r = self.r_max()
            lo = np.minimum(lo, self.state[:, :3].min(axis=0) - r)
            hi = np.maximum(hi, self.state[:, :3].max(axis=0) + r)
        return tuple(float(x) for x in lo), tuple(float(x) for x in hi)

    def copy(self, **kw) -> "Scene":
        d = dict(self.__dict__)
        d["state"] = self.state.copy()
        d["meta"] = dict(self.meta)
        d.update(kw)
        return Scene(**d)


def mass_of(radius: np.ndarray, density: float) -> np.ndarray:
    """density * 4/3 * pi * r^3 (ParticleIO.cpp:131)."""
    return density * 4.0 / 3.0 * math.pi * np.power(radius, 3.0)


def _state(pos: np.ndarray, vel: np.ndarray, r: np.ndarray, density: float) -> np.ndarray:
    n = pos.shape[0]
    st = np.empty((n, 8), dtype=np.float64)
    st[:, 0:3] = pos
    st[:, 3:6] = vel
    st[:, 6] = r
    st[:, 7] = mass_of(r, density)
    return st


# ---- small, CPU-runnable workload (4,096 spheres) ----------------------------
def lattice_c1(seed: int = 1, side: int = 16) -> Scene:
    """side^3 spheres of radius 0.01 on a jittered cubic lattice (jitter uniform
    +-0.002) in the upper half of the box [0,1]^3; zero velocity, density 1000,
    spring 1e4, sphere restitution 0.5, walls 0.8, gravity (0,0,-9.8), dt 1e-5."""
    rng = np.random.default_rng(seed)
    i = np.arange(side)
    gx, gy, gz = np.meshgrid(i, i, i, indexing="ij")
    pos = np.stack([(gx.ravel() + 0.5) / side, (gy.ravel() + 0.5) / side,
                    0.5 + (gz.ravel() + 0.5) * 0.5 / side], axis=1)
    pos += rng.uniform(-0.002, 0.002, size=pos.shape)
    n = pos.shape[0]
    st = _state(pos, np.zeros((n, 3)), np.full(n, 0.01), 1000.0)
    return Scene(st, (0, 0, 0), (1, 1, 1), (0, 0, -9.8), (0.8,) * 6, 1e4, 0.5, 1e-5, name="lattice_c1")


def pile(n: int = 1024, seed: int = 3, k_spring: float = 1.0, e_sphere: float = 0.5) -> Scene:
    """Contact-rich fixture: polydisperse spheres (r in [0.004, 0.006]) packed on
    a jittered lattice of pitch 0.0118 < 2 r_max in a narrow box, random
    velocities N(0, 0.1^2).  Many pairs overlap from the first step."""
    rng = np.random.default_rng(seed)
    pitch = 0.0118
    nx = ny = max(2, int(round((n / 4) ** (1 / 3) * 1.0)))
    nz = int(math.ceil(n / (nx * ny)))
    idx = np.arange(nx * ny * nz)[:n]
    pos = np.stack([(idx // (ny * nz)) % nx, (idx // nz) % ny, idx % nz], axis=1).astype(np.float64)
    pos = (pos + 0.5) * pitch + rng.uniform(-2e-4, 2e-4, size=(n, 3))
    r = rng.uniform(0.004, 0.006, size=n)
    vel = rng.normal(0.0, 0.1, size=(n, 3))
    st = _state(pos, vel, r, 1000.0)
    hi = (nx * pitch, ny * pitch, nz * pitch * 1.5)
    return Scene(st, (0, 0, 0), hi, (0, 0, -9.8), (0.7, 0.6, 0.8, 0.75, 0.85, 0.65), k_spring, e_sphere, 1e-5,
                 name="pile")


def settle_pile(side: int = 16, seed: int = 9) -> Scene:
    """Long-run fixture: side^3 spheres of radius 0.01 at rest on a lattice of
    pitch 0.0225 (jitter +-0.001) in a box of base (side * 0.0225)^2 and
    height 1, spring 40 (k dt / m = 0.095, stable under the reference
    scheme), sphere restitution 0.5, walls 0.5, dt 1e-5.  The lattice
    collapses into a pile that is close to rest after about 40,000 steps."""
    rng = np.random.default_rng(seed)
    pitch, r = 0.0225, 0.01
    ijk = np.stack(np.meshgrid(np.arange(side), np.arange(side), np.arange(side), indexing="ij"), -1)
    ijk = ijk.reshape(-1, 3).astype(np.float64)
    pos = (ijk + 0.5) * pitch + rng.uniform(-0.001, 0.001, size=ijk.shape)
    st = _state(pos, np.zeros_like(pos), np.full(pos.shape[0], r), 1000.0)
    edge = side * pitch
    return Scene(st, (0, 0, 0), (edge, edge, 1.0), (0, 0, -9.8), (0.5,) * 6, 40.0, 0.5, 1e-5, name="settle_pile")


def slab_packing_fraction(state: np.ndarray, box_min, box_max, z_lo: float, z_hi: float) -> float:
    """Fraction of the box's volume between the planes z_lo and z_hi that the
    spheres fill (exact sphere-slab intersection volumes; the spheres are
    inside the box and overlaps are small)."""
    z, r = state[:, 2], state[:, 6]
    t1 = np.clip(z_lo - z, -r, r)
    t2 = np.clip(z_hi - z, -r, r)
    vol = np.pi * ((r * r * t2 - t2 ** 3 / 3.0) - (r * r * t1 - t1 ** 3 / 3.0))
    area = (box_max[0] - box_min[0]) * (box_max[1] - box_min[1])
    return float(vol.sum() / (area * (z_hi - z_lo)))


def height_histogram(state: np.ndarray, z_max: float, bins: int = 24) -> np.ndarray:
    """Fraction of sphere centres in each of `bins` equal height bins over [0, z_max]."""
    h, _ = np.histogram(state[:, 2], bins=bins, range=(0.0, z_max))
    return h / max(1, state.shape[0])


# ---- the 1M-sphere workload ---------------------------------------------------
def c2_scene(n: int = 1 << 20, seed: int = 2, k_spring: float = 5e4) -> Scene:
    """1,048,576 spheres, log-normal radii (median 0.002, sigma 0.25, clipped to
    [0.001, 0.004]), non-overlapping placement by rejection on a grid of
    2*r_max slots in the box [0,1]x[0,1]x[0,4], velocities N(0, 0.05^2) per
    component; spring 5e4, sphere restitution 0.4, walls 0.7, dt 5e-6,
    grid cell 2*r_max.  Density 1000.

    Under the reference's scheme (kick k*overlap/m, not scaled by dt) spring
    5e4 gives k*dt/m up to 60 for the smallest spheres, and the first
    contacts diverge; k_spring=0.25 (k*dt/m <= 0.3) is the same scene with a
    spring the scheme integrates stably."""
    rng = np.random.default_rng(seed)
    r = np.clip(rng.lognormal(math.log(0.002), 0.25, size=n), 0.001, 0.004)
    slot = 2.0 * 0.004
    dims = (int(1.0 / slot), int(1.0 / slot), int(4.0 / slot))
    n_slots = dims[0] * dims[1] * dims[2]
    if n > n_slots:
        raise ValueError("too many spheres for the slot grid")
    chosen = rng.choice(n_slots, size=n, replace=False)
    ix = chosen // (dims[1] * dims[2])
    iy = (chosen // dims[2]) % dims[1]
    iz = chosen % dims[2]
    centre = (np.stack([ix, iy, iz], axis=1).astype(np.float64) + 0.5) * slot
    room = (slot / 2 - r)[:, None]
    pos = centre + rng.uniform(-1.0, 1.0, size=(n, 3)) * room
    vel = rng.normal(0.0, 0.05, size=(n, 3))
    st = _state(pos, vel, r, 1000.0)
    name = "c2_1M" if k_spring == 5e4 else f"c2_1M_k{k_spring:g}"
    return Scene(st, (0, 0, 0), (1, 1, 4), (0, 0, -9.8), (0.7,) * 6, k_spring, 0.4, 5e-6, interval=2.0 * 0.004,
                 name=name)


# ---- mesh container workload -------------------------------------------------
def funnel_triangles(n_seg: int = 200, n_cone: int = 40, n_cyl: int = 6, n_ring: int = 4) -> np.ndarray:
    """Closed funnel as a surface of revolution with outward normals: cone from
    radius 0.5 at z=1 to 0.08 at z=0.3, cylinder of radius 0.08 down to z=0,
    flat disk bottom (concentric rings, no single hub vertex).  About
    2*n_seg*(n_cone+n_cyl+n_ring) triangles; the defaults give 20,000."""
    th = np.linspace(0.0, 2.0 * math.pi, n_seg, endpoint=False)
    c, s = np.cos(th), np.sin(th)
    rings = []  # (radius, z) from the top rim down the wall, then the bottom rings inward
    for k in range(n_cone + 1):
        t = k / n_cone
        rings.append((0.5 + (0.08 - 0.5) * t, 1.0 + (0.3 - 1.0) * t))
    for k in range(1, n_cyl + 1):
        rings.append((0.08, 0.3 - 0.3 * k / n_cyl))
    for k in range(1, n_ring + 1):
        rings.append((0.08 * (1 - k / (n_ring + 0.5)), 0.0))
    tris = []
    for a in range(len(rings) - 1):
        (r0, z0), (r1, z1) = rings[a], rings[a + 1]
        for j in range(n_seg):
            j1 = (j + 1) % n_seg
            p00 = (r0 * c[j], r0 * s[j], z0)
            p01 = (r0 * c[j1], r0 * s[j1], z0)
            p10 = (r1 * c[j], r1 * s[j], z1)
            p11 = (r1 * c[j1], r1 * s[j1], z1)
            # outward normal: (p10 - p00) x (p01 - p00) points away from the axis/down
            tris.append((p00, p10, p01))
            tris.append((p01, p10, p11))
    # innermost ring closed with a small fan (the last ring radius is 0.08/(4.5))
    rl, zl = rings[-1]
    for j in range(n_seg):
        j1 = (j + 1) % n_seg
        tris.append(((rl * c[j], rl * s[j], zl), (0.0, 0.0, zl), (rl * c[j1], rl * s[j1], zl)))
    t = np.asarray(tris, dtype=np.float64).reshape(-1, 9)
    # single-precision vertices, as an OBJ read through assimp would give
    return t.astype(np.float32).astype(np.float64)


def box_container(lo=(-0.1, -0.1, 0.0), hi=(0.1, 0.1, 0.25), n: int = 4) -> np.ndarray:
    """Closed axis-aligned box as a triangle mesh: n x n quads per face, two
    triangles each, normals pointing out; single-precision vertices."""
    lo = np.asarray(lo, dtype=np.float64)
    hi = np.asarray(hi, dtype=np.float64)
    tris = []
    for axis in range(3):
        u, v = [a for a in range(3) if a != axis]
        for side, sign in ((lo[axis], -1.0), (hi[axis], 1.0)):
            for i in range(n):
                for j in range(n):
                    def pt(a, b):
                        p = np.zeros(3)
                        p[axis] = side
                        p[u] = lo[u] + (hi[u] - lo[u]) * a / n
                        p[v] = lo[v] + (hi[v] - lo[v]) * b / n
                        return p
                    p00, p10, p01, p11 = pt(i, j), pt(i + 1, j), pt(i, j + 1), pt(i + 1, j + 1)
                    t1, t2 = [p00, p10, p11], [p00, p11, p01]
                    if np.sign(np.cross(t1[1] - t1[0], t1[2] - t1[0])[axis]) != sign:
                        t1, t2 = [p00, p11, p10], [p00, p01, p11]
                    tris.append(np.concatenate(t1))
                    tris.append(np.concatenate(t2))
    return np.asarray(tris).astype(np.float32).astype(np.float64)


def box_mesh_scene(n: int = 120, seed: int = 41) -> Scene:
    """Spheres in a closed triangulated box; the outer layers overlap the
    side walls and the floor from the first step.  Spring 2, dt 1e-4."""
    rng = np.random.default_rng(seed)
    g = np.stack(np.meshgrid(np.arange(5), np.arange(5), np.arange(5), indexing="ij"), -1).reshape(-1, 3)[:n]
    pos = np.array([-0.092, -0.092, 0.006]) + g * 0.046 + rng.uniform(-0.002, 0.002, size=(n, 3))
    vel = rng.normal(0, 0.5, size=(n, 3))
    st = _state(pos, vel, np.full(n, 0.012), 1000.0)
    return Scene(st, (-0.1, -0.1, 0.0), (0.1, 0.1, 0.25), (0, 0, -9.8), (0.7,) * 6, 2.0, 0.5, 1e-4,
                 tri=box_container(), name="box_mesh")


def fan_floor_box(half: float = 0.05, height: float = 0.1, n_fan: int = 300) -> np.ndarray:
    """Closed box [-half, half]^2 x [0, height] whose floor is a fan of
    n_fan triangles around the floor's centre (every floor triangle has a
    vertex at the origin); the other faces are two triangles each.  Normals
    point out."""
    box = box_container((-half, -half, 0.0), (half, half, height), n=1)
    walls = box[~np.all(box[:, 2::3] == 0.0, axis=1)]
    # perimeter points of the floor square, counter-clockwise from (-h, -h)
    corners = np.array([[-half, -half], [half, -half], [half, half], [-half, half]])
    per_side = n_fan // 4
    pts = []
    for k in range(4):
        a, b = corners[k], corners[(k + 1) % 4]
        for j in range(per_side):
            pts.append(a + (b - a) * j / per_side)
    pts = np.asarray(pts)
    fan = []
    for k in range(len(pts)):
        p, q = pts[k], pts[(k + 1) % len(pts)]
        # (origin, q, p): clockwise seen from above, so the normal points down (out)
        fan.append([0.0, 0.0, 0.0, q[0], q[1], 0.0, p[0], p[1], 0.0])
    tri = np.concatenate([np.asarray(fan), walls])
    return tri.astype(np.float32).astype(np.float64)


def fan_floor_scene(n_fan: int = 300, seed: int = 43) -> Scene:
    """Spheres of radius 0.01 in a box whose floor is a fine triangle fan
    (fan_floor_box): one sphere sits on the fan's centre 1e-5 deep, so it
    touches all n_fan floor triangles at once; two more press on the fan
    away from the centre and touch a few tens; a loose layer above falls.
    Spring 2, dt 1e-4.  Density 1000."""
    rng = np.random.default_rng(seed)
    r = 0.01
    low = np.array([[0.0, 0.0, r - 1e-5], [0.025, 0.0, r - 2e-4], [-0.02, 0.015, r - 1e-4]])
    g = np.stack(np.meshgrid(np.arange(4), np.arange(4), np.arange(2), indexing="ij"), -1).reshape(-1, 3)
    high = np.array([-0.036, -0.036, 0.045]) + g * 0.024 + rng.uniform(-0.001, 0.001, size=(len(g), 3))
    pos = np.concatenate([low, high])
    vel = np.concatenate([np.zeros((3, 3)), rng.normal(0, 0.05, size=(len(g), 3))])
    st = _state(pos, vel, np.full(len(pos), r), 1000.0)
    return Scene(st, (-0.05, -0.05, 0.0), (0.05, 0.05, 0.1), (0, 0, -9.8), (0.7,) * 6, 2.0, 0.5, 1e-4,
                 tri=fan_floor_box(n_fan=n_fan), name="fan_floor")


def funnel_wall_scene(n: int = 2000, seed: int = 7, coarse: bool = True, z_max: float = 1.05,
                      widen: bool = True) -> Scene:
    """Spheres (r 0.003) on rings just inside the funnel's cone wall at
    heights 0.45..z_max, pressing outward (with the default z_max some start
    above the rim): every step has triangle contacts.  A coarse funnel keeps
    the all-pairs oracle fast.  With z_max below 1 every centre lies inside
    the mesh AABB, the grid domain of the reference's CUDA path."""
    rng = np.random.default_rng(seed)
    tri = funnel_triangles(64, 12, 3, 2) if coarse else funnel_triangles()
    z = rng.uniform(0.45, z_max, size=n)
    t = np.clip((1.0 - z) / 0.7, 0.0, 1.0)
    wall_r = 0.5 + (0.08 - 0.5) * t
    rad = wall_r - rng.uniform(0.0, 0.004, size=n)
    th = rng.uniform(0, 2 * math.pi, size=n)
    pos = np.stack([rad * np.cos(th), rad * np.sin(th), z], 1)
    vel = np.stack([0.3 * np.cos(th), 0.3 * np.sin(th), rng.normal(0, 0.1, n)], 1)
    st = _state(pos, vel, np.full(n, 0.003), 1000.0)
    e = (0.6,) * 6
    return Scene(st, (-0.5, -0.5, 0.0), (0.5, 0.5, 1.0), (0, 0, -9.8), e, 2e-2, 0.5, 5e-6, tri=tri,
                 widen_domain=1 if widen else 0, name="funnel_wall")


def write_obj(path: str, tri: np.ndarray) -> None:
    """Triangle soup as OBJ (one vertex line per corner, %.9g = exact float)."""
    with open(path, "w") as f:
        for t in tri.reshape(-1, 9):
            for k in range(3):
                f.write("v %.9g %.9g %.9g\n" % (t[3 * k], t[3 * k + 1], t[3 * k + 2]))
        for i in range(tri.shape[0]):
            f.write("f %d %d %d\n" % (3 * i + 1, 3 * i + 2, 3 * i + 3))


def c3_scene(n: int = 262144, seed: int = 4, widen: bool = True) -> Scene:
    """262,144 spheres of radius 0.003 on a jittered lattice above z=1, poured
    into the funnel; polygon restitution 0.6 (passed as the zMin wall value),
    spring 2e4, dt 5e-6.  Density 1000."""
    rng = np.random.default_rng(seed)
    tri = funnel_triangles()
    pitch = 0.0075
    rad = 0.45
    g = np.arange(-rad, rad + 1e-12, pitch)
    gx, gy = np.meshgrid(g, g, indexing="ij")
    keep = gx ** 2 + gy ** 2 <= rad ** 2
    xy = np.stack([gx[keep], gy[keep]], axis=1)
    layers = int(math.ceil(n / xy.shape[0]))
    pos = np.concatenate([np.column_stack([xy, np.full(xy.shape[0], 1.01 + k * pitch)]) for k in range(layers)])[:n]
    pos += rng.uniform(-5e-4, 5e-4, size=pos.shape)
    st = _state(pos, np.zeros((n, 3)), np.full(n, 0.003), 1000.0)
    e = (0.6, 0.6, 0.6, 0.6, 0.6, 0.6)
    return Scene(st, (-0.5, -0.5, 0.0), (0.5, 0.5, 1.0), (0, 0, -9.8), e, 2e4, 0.5, 5e-6, tri=tri,
                 widen_domain=1 if widen else 0, name="c3_funnel")


# ---- differentiation workload -----------------------------------------------
def c4_scene(n: int = 65536, seed: int = 5, edge: float = 0.5, k_spring: float = 1e4) -> Scene:
    """65,536 spheres of radius 0.004 in the box [0,0.5]^3 placed without
    overlap on a grid of 0.009 slots, velocities N(0, 0.01^2), spring 1e4,
    sphere restitution 0.5, walls 0.8, dt 1e-5.  Density 1000.  `edge`
    enlarges the box for larger n (1M spheres need edge >= 0.918).

    The reference's contact kick k*overlap/m is not scaled by dt, so the
    explicit update is stable only for k*dt/m below about 1; with spring 1e4
    that ratio is 373 and the first sphere-sphere contacts (after about
    1,300 steps, when the lowest layers meet) diverge.  k_spring=5 (ratio
    0.19) keeps the scene finite with contacts."""
    rng = np.random.default_rng(seed)
    slot = 0.009
    d = int(edge / slot)
    if n > d ** 3:
        raise ValueError(f"{n} spheres do not fit {d}^3 slots")
    chosen = rng.choice(d ** 3, size=n, replace=False)
    ijk = np.stack([chosen // (d * d), (chosen // d) % d, chosen % d], axis=1).astype(np.float64)
    pos = (ijk + 0.5) * slot + rng.uniform(-2e-4, 2e-4, size=(n, 3))
    vel = rng.normal(0.0, 0.01, size=(n, 3))
    st = _state(pos, vel, np.full(n, 0.004), 1000.0)
    name = "c4_65k" if (n, edge) == (65536, 0.5) else f"c4_{n}_edge{edge:g}"
    if k_spring != 1e4:
        name += f"_k{k_spring:g}"
    return Scene(st, (0, 0, 0), (edge, edge, edge), (0, 0, -9.8), (0.8,) * 6, k_spring, 0.5, 1e-5, name=name)


# ---- batching workload ---------------------------------------------------------
def c5_scenes(n_scenes: int = 256, seed: int = 6, n_lo: int = 1024, n_hi: int = 65536,
              k_range: tuple[float, float] = (5e3, 5e4)) -> list[Scene]:
    """Independent scenes: particle count log-uniform in [n_lo, n_hi], radii
    uniform in [0.002, 0.006], cubic box of edge uniform in [0.2, 1.0],
    spring log-uniform in k_range (default [5e3, 5e4]), restitutions uniform
    in [0.3, 0.9], dt 5e-6.  Spheres are placed without overlap on 2*r_max
    slots (the count is capped by the slots the box holds).

    With the default springs k*dt/m reaches 27..7,460 and the reference's
    scheme diverges at the first contacts; k_range=(0.25, 2.5) keeps
    k*dt/m <= 0.37 and every scene finite.  The other draws do not depend on
    k_range, so both sets share particle counts, radii, boxes and states."""
    rng = np.random.default_rng(seed)
    out = []
    for s in range(n_scenes):
        n = int(round(math.exp(rng.uniform(math.log(n_lo), math.log(n_hi)))))
        edge = float(rng.uniform(0.2, 1.0))
        r = rng.uniform(0.002, 0.006, size=n)
        slot = 2.0 * 0.006
        d = int(edge / slot)
        n = min(n, d ** 3)
        r = r[:n]
        chosen = rng.choice(d ** 3, size=n, replace=False)
        ijk = np.stack([chosen // (d * d), (chosen // d) % d, chosen % d], axis=1).astype(np.float64)
        pos = (ijk + 0.5) * slot + rng.uniform(-1, 1, size=(n, 3)) * (slot / 2 - r)[:, None]
        vel = rng.normal(0.0, 0.05, size=(n, 3))
        u = rng.uniform(0.0, 1.0)
        k = float(math.exp(math.log(k_range[0]) + u * (math.log(k_range[1]) - math.log(k_range[0]))))
        e_s = float(rng.uniform(0.3, 0.9))
        e_w = tuple(float(x) for x in rng.uniform(0.3, 0.9, size=6))
        out.append(Scene(_state(pos, vel, r, 1000.0), (0, 0, 0), (edge, edge, edge), (0, 0, -9.8), e_w, k, e_s, 5e-6,
                         name=f"c5_{s}"))
    return out
