"""Seeded synthetic inputs for the IB coupling benchmarks and tests.

No public dataset is involved: the workloads are red-cell and platelet
surfaces sampled on Fibonacci spheres, placed in periodic boxes or in a
walled channel, with iid Gaussian point forces and face velocities.

Units follow the reference (include/units.h:16-18, 221-243): internal length
unit 10 um (``UM = 0.1``), time unit 1 ms, mass unit 1 ug, so 1 pN = 1e-4 and
1 um/s = 1e-4 internal units.  Point arrays use the reference layout
``x[d*n + p]`` with the points of one cell contiguous
(include/bases/container.h:40-58).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

UM = 0.1            # internal length units per micrometre
PN = 1e-4           # internal force units per piconewton
UM_PER_S = 1e-4     # internal velocity units per um/s
H_UM = 0.25         # grid spacing of every configuration (um)

# Evans-Fung biconcave disc, R = 3.91 um
RBC_RADIUS_UM = 3.91
RBC_COEFFS = (0.2072, 2.0026, -1.1228)
# Oblate spheroid platelet: 1.8 um semi-axis, 0.5 um half-thickness
PLT_AXES_UM = (1.8, 1.8, 0.5)


def fibonacci_sphere(n: int) -> np.ndarray:
    """n points on the unit sphere (Fibonacci / golden-angle spiral), (n, 3)."""
    i = np.arange(n, dtype=np.float64) + 0.5
    z = 1.0 - 2.0 * i / n
    rho = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    phi = i * math.pi * (3.0 - math.sqrt(5.0))
    return np.stack([rho * np.cos(phi), rho * np.sin(phi), z], axis=1)


def rbc_surface(n: int) -> np.ndarray:
    """Evans-Fung biconcave RBC (disc normal along local z), in um, (n, 3).

    z = +/- 0.5 R sqrt(1 - rho^2) (c0 + c1 rho^2 + c2 rho^4), rho = radial/R.
    """
    s = fibonacci_sphere(n)
    rho2 = np.minimum(1.0, s[:, 0] ** 2 + s[:, 1] ** 2)
    c0, c1, c2 = RBC_COEFFS
    R = RBC_RADIUS_UM
    h = 0.5 * R * np.sqrt(1.0 - rho2) * (c0 + c1 * rho2 + c2 * rho2 * rho2)
    return np.stack([R * s[:, 0], R * s[:, 1], np.sign(s[:, 2]) * h], axis=1)


def platelet_surface(n: int) -> np.ndarray:
    """Oblate spheroid platelet (symmetry axis local z), in um, (n, 3)."""
    s = fibonacci_sphere(n)
    return s * np.asarray(PLT_AXES_UM)[None, :]


def rotation(axis: np.ndarray, angle: float) -> np.ndarray:
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + math.sin(angle) * K + (1 - math.cos(angle)) * (K @ K)


def random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def flat_rotation(rng: np.random.Generator, max_tilt_deg: float = 5.0) -> np.ndarray:
    """Rotation taking local z to (nearly) the channel's wall normal y: a full
    random turn about y and a tilt of at most max_tilt_deg."""
    to_y = rotation([1.0, 0.0, 0.0], -math.pi / 2)          # local z -> y
    tilt_axis = rng.normal(size=3)
    tilt_axis[1] = 0.0
    tilt = rotation(tilt_axis if np.linalg.norm(tilt_axis) > 0 else [1, 0, 0],
                    math.radians(rng.uniform(0, max_tilt_deg)))
    spin = rotation([0.0, 1.0, 0.0], rng.uniform(0, 2 * math.pi))
    return spin @ tilt @ to_y


@dataclass
class Workload:
    name: str
    lengths: list              # internal units
    boundaries: list           # 0 periodic, 1 solid
    refinement: int
    cells: list = field(default_factory=list)   # per cell: (kind, n_points)
    x: np.ndarray = None       # (dims*n,) float64, reference layout
    f: np.ndarray = None       # (dims*n,) float64
    seed: int = 0
    velocity: str = "gaussian"  # or "poiseuille"

    @property
    def dims(self) -> int:
        return len(self.lengths)

    @property
    def n(self) -> int:
        return self.x.size // self.dims


def _assemble(parts):
    """parts: list of (n_i, 3) arrays in internal units -> reference layout."""
    pts = np.concatenate(parts, axis=0)
    return np.ascontiguousarray(pts.T).reshape(-1)


def _forces(rng, n, dims=3):
    return rng.normal(size=dims * n) * PN


def single_rbc(seed: int = 0, n_points: int = 2210) -> Workload:
    """Triply periodic 16 um cube, MAC 64^3, one RBC at a random centre and
    rotation; forces iid N(0,1) pN."""
    rng = np.random.default_rng(seed)
    L = 16.0
    ref = rbc_surface(n_points)
    R = random_rotation(rng)
    c = rng.uniform(0, L, size=3)
    pts = (ref @ R.T + c) * UM
    w = Workload("single-rbc-64^3", [L * UM] * 3, [0, 0, 0], 64, [("rbc", n_points)], seed=seed)
    w.x = _assemble([pts])
    w.f = _forces(rng, w.n)
    return w


def _slot_packing(rng, box_um, n_rbc, rbc_pts, n_plt, plt_pts, wall_gap_um=0.5):
    """Random non-overlapping placement in a walled channel (walls normal to
    y).  The channel is cut into slots of 8.0 x 3.2 x 8.0 um; each slot holds
    one RBC (7.82 um across, <= 3.1 um tall at <= 5 deg tilt) or a 2x2x2
    stack of platelets (3.6 um across, <= 1.32 um tall).  Slots are chosen at
    random; each cell gets a random turn about y, a small tilt and a random
    shift inside its slot, so no two cells can overlap and every cell stays
    >= wall_gap_um from the walls."""
    Lx, Ly, Lz = box_um
    sx, sy, sz = 8.0, 3.2, 8.0
    nx, nz = int(Lx // sx), int(Lz // sz)
    ny = int((Ly - 2 * wall_gap_um) // sy)
    slots = [(i, j, k) for i in range(nx) for j in range(ny) for k in range(nz)]
    n_plt_slots = (n_plt + 7) // 8
    if n_rbc + n_plt_slots > len(slots):
        raise ValueError("channel too small for the requested cells")
    order = rng.permutation(len(slots))
    y0 = wall_gap_um + 0.5 * ((Ly - 2 * wall_gap_um) - ny * sy)
    rbc_ref = rbc_surface(rbc_pts)
    plt_ref = platelet_surface(plt_pts)
    parts, cells = [], []

    def place(ref, centre, half_extent_xz, half_extent_y, slot_half):
        R = flat_rotation(rng)
        body = ref @ R.T
        slack = np.maximum(0.0, np.array(slot_half) - np.array([half_extent_xz, half_extent_y, half_extent_xz]))
        c = np.asarray(centre) + rng.uniform(-1, 1, size=3) * slack * 0.9
        return body + c

    for s in range(n_rbc):
        i, j, k = slots[order[s]]
        centre = ((i + 0.5) * sx, y0 + (j + 0.5) * sy, (k + 0.5) * sz)
        parts.append(place(rbc_ref, centre, RBC_RADIUS_UM, 1.55, (sx / 2, sy / 2, sz / 2)))
        cells.append(("rbc", rbc_pts))
    placed = 0
    for s in range(n_plt_slots):
        i, j, k = slots[order[n_rbc + s]]
        for a in range(2):
            for b in range(2):
                for c in range(2):
                    if placed == n_plt:
                        break
                    centre = ((i + 0.25 + 0.5 * a) * sx, y0 + (j + 0.25 + 0.5 * c) * sy,
                              (k + 0.25 + 0.5 * b) * sz)
                    parts.append(place(plt_ref, centre, 1.8, 0.66, (sx / 4, sy / 4, sz / 4)))
                    cells.append(("platelet", plt_pts))
                    placed += 1
    return parts, cells


def channel(seed: int = 0, box_um=(32.0, 16.0, 32.0), refinement: int = 64,
            n_rbc: int = 40, n_plt: int = 60, rbc_pts: int = 2210, plt_pts: int = 605,
            name: str = "channel-128x64x128") -> Workload:
    """Periodic-x/z channel with no-slip walls at y = 0 and y = Ly."""
    rng = np.random.default_rng(seed)
    parts, cells = _slot_packing(rng, box_um, n_rbc, rbc_pts, n_plt, plt_pts)
    w = Workload(name, [b * UM for b in box_um], [0, 1, 0], refinement, cells, seed=seed,
                 velocity="poiseuille")
    w.x = _assemble([p * UM for p in parts])
    w.f = _forces(rng, w.n)
    return w


def large_channel(seed: int = 0) -> Workload:
    """128 x 64 x 128 um channel, MAC 512x256x512, 3300 RBCs of 2210 points
    and 6000 platelets of 605 points (10,923,000 points)."""
    w = channel(seed, box_um=(128.0, 64.0, 128.0), refinement=256, n_rbc=3300, n_plt=6000,
                name="large-channel-512x256x512")
    w.velocity = "gaussian"
    return w


def medium_channel(seed: int = 0) -> Workload:
    """64 x 32 x 64 um channel, MAC 256x128x256, 412 RBCs + 750 platelets
    (1/8 of the large channel; its fields still exceed L2)."""
    w = channel(seed, box_um=(64.0, 32.0, 64.0), refinement=128, n_rbc=412, n_plt=750,
                name="medium-channel-256x128x256")
    w.velocity = "gaussian"
    return w


GRID_SIDES = (32, 48, 64, 96, 128)
CELL_CHOICES = (("rbc", 864), ("rbc", 2210), ("rbc", 8832), ("platelet", 386), ("platelet", 1552))


def ensemble_instance(rng: np.random.Generator, name: str = "instance") -> Workload:
    """One batched instance: periodic cube of side n*h, n drawn from
    {32,48,64,96,128}, 1-50 cells drawn from RBC 864/2210/8832 and platelet
    386/1552, uniformly placed and rotated (overlaps allowed)."""
    side = int(rng.choice(GRID_SIDES))
    L = side * H_UM
    ncell = int(rng.integers(1, 51))
    parts, cells = [], []
    for _ in range(ncell):
        kind, npts = CELL_CHOICES[int(rng.integers(0, len(CELL_CHOICES)))]
        ref = rbc_surface(npts) if kind == "rbc" else platelet_surface(npts)
        pts = ref @ random_rotation(rng).T + rng.uniform(0, L, size=3)
        parts.append(pts * UM)
        cells.append((kind, npts))
    w = Workload(f"{name}-{side}^3", [L * UM] * 3, [0, 0, 0], side, cells)
    w.x = _assemble(parts)
    w.f = _forces(rng, w.n)
    return w


def small_instance(rng: np.random.Generator, side: int, ncell: int, walls: bool = False,
                   name: str = "small") -> Workload:
    """A test-sized instance: side^3 cells of h = 0.25 um (a walled channel
    along y when walls is set), ncell platelets or small RBCs (386 / 864
    points) placed at random (inside the walls, overlaps allowed)."""
    L = side * H_UM
    parts, cells = [], []
    for _ in range(ncell):
        kind, npts = [("plt", 386), ("rbc", 864)][int(rng.integers(0, 2))]
        ref = rbc_surface(npts) if kind == "rbc" else platelet_surface(npts)
        centre = rng.uniform(0, L, size=3)
        if walls:
            centre[1] = rng.uniform(0.45 * L, 0.55 * L)
            ref = ref * min(1.0, 0.3 * L / RBC_RADIUS_UM)
        parts.append((ref @ random_rotation(rng).T + centre) * UM)
        cells.append((kind, npts))
    w = Workload(f"{name}-{side}^3", [L * UM] * 3, [0, 1 if walls else 0, 0], side, cells)
    w.x = _assemble(parts)
    w.f = _forces(rng, w.n)
    return w


def ensemble(seed: int = 0, count: int = 256):
    rng = np.random.default_rng(seed)
    return [ensemble_instance(rng, f"member{i}") for i in range(count)]


def grid_velocity(w: Workload, sizes, points, rng: np.random.Generator | None = None):
    """Face velocities per component as flat numpy arrays (x-fastest)."""
    rng = rng or np.random.default_rng(w.seed + 1)
    ue = []
    for c, s in enumerate(sizes):
        u = rng.normal(size=s) * UM_PER_S
        if w.velocity == "poiseuille" and c == 0:
            # u_x(y) = 4 Umax y (H - y) / H^2 with Umax = 100 um/s, noise N(0,1)
            p = points[c]
            H = w.lengths[1]
            ny = p[1]
            y = (np.arange(ny) + 0.5) / ny * H
            prof = 4 * 100.0 * UM_PER_S * y * (H - y) / (H * H)
            u = u.reshape(p[2], p[1], p[0]) + prof[None, :, None]
            u = u.reshape(-1)
        ue.append(np.ascontiguousarray(u))
    return ue


CONFIGS = {
    "single-rbc": single_rbc,
    "channel": channel,
    "medium-channel": medium_channel,
    "large-channel": large_channel,
}
