"""Seeded synthetic scenes written directly as mechanic-gpu ABI rows.

The reference builds rows from a ``CompiledCreation`` (compile.rs:256-609,
device.rs:429-523).  These generators write the same rows without the
construction graph, following the reference's own rules:

* part mass and inertia: compile.rs:839-879 (cuboid and cylinder sector);
* compound aggregation at the centre of mass with identity root rotation:
  compile.rs:768-821, :330-337;
* 16 cuboid colliders per cylinder: compile.rs:881-929;
* analytic cylinder ground roles: device.rs:3008-3045.

Randomness is a counter-based SplitMix64 (one stream per field, seeded with
``seed ^ scene_index``), so the GPU library and the CPU oracle see identical
rows.  All row arithmetic is float32, as in the reference.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from . import abi

CUBOID_DENSITY = np.float32(1000.0)   # the reference hard-codes 500 (mechanic-core lib.rs:35); the
                                      # benchmark scenes ask for 1000 kg/m^3
CYLINDER_COLLIDER_COUNT = 16          # compile.rs:15

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def splitmix64(seed: int, index: np.ndarray) -> np.ndarray:
    """SplitMix64 output for counter ``index`` of stream ``seed`` (vectorised)."""
    with np.errstate(over="ignore"):
        z = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + (index.astype(np.uint64) + np.uint64(1)) * _GOLDEN
        z = (z ^ (z >> np.uint64(30))) * _M1
        z = (z ^ (z >> np.uint64(27))) * _M2
        return z ^ (z >> np.uint64(31))


class Rng:
    """Independent named streams over one seed."""

    def __init__(self, seed: int):
        self.seed = seed

    def _stream(self, name: str) -> int:
        h = 1469598103934665603
        for ch in name.encode():
            h = ((h ^ ch) * 1099511628211) & 0xFFFFFFFFFFFFFFFF
        return (self.seed * 0x2545F4914F6CDD1D ^ h) & 0xFFFFFFFFFFFFFFFF

    def uniform(self, name: str, n: int, lo: float = 0.0, hi: float = 1.0) -> np.ndarray:
        u = (splitmix64(self._stream(name), np.arange(n)) >> np.uint64(11)).astype(np.float64)
        u *= 2.0 ** -53
        return lo + (hi - lo) * u

    def normal(self, name: str, n: int) -> np.ndarray:
        u1 = self.uniform(name + ".u1", n)
        u2 = self.uniform(name + ".u2", n)
        return np.sqrt(-2.0 * np.log1p(-u1)) * np.cos(2.0 * np.pi * u2)

    def unit_quaternions(self, name: str, n: int) -> np.ndarray:
        """Uniform rotations (Shoemake 1992), xyzw."""
        u1, u2, u3 = (self.uniform(f"{name}.{k}", n) for k in range(3))
        a, b = np.sqrt(1.0 - u1), np.sqrt(u1)
        q = np.stack([a * np.sin(2 * np.pi * u2), a * np.cos(2 * np.pi * u2),
                      b * np.sin(2 * np.pi * u3), b * np.cos(2 * np.pi * u3)], axis=1)
        return q


# ------------------------------------------------------------------ quats
def quat_yaw(angle: np.ndarray) -> np.ndarray:
    """``Quat::from_rotation_y`` (xyzw)."""
    h = np.asarray(angle, np.float64) * 0.5
    z = np.zeros_like(h)
    return np.stack([z, np.sin(h), z, np.cos(h)], axis=-1)


def quat_mul(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    ax, ay, az, aw = np.moveaxis(a, -1, 0)
    bx, by, bz, bw = np.moveaxis(b, -1, 0)
    return np.stack([aw * bx + ax * bw + ay * bz - az * by,
                     aw * by - ax * bz + ay * bw + az * bx,
                     aw * bz + ax * by - ay * bx + az * bw,
                     aw * bw - ax * bx - ay * by - az * bz], axis=-1)


def quat_rotate(q: np.ndarray, v: np.ndarray) -> np.ndarray:
    u = q[..., :3]
    t = 2.0 * np.cross(u, v)
    return v + q[..., 3:4] * t + np.cross(u, t)


def quat_matrix(q: np.ndarray) -> np.ndarray:
    """Rotation matrices (..., 3, 3) with columns R*e_i."""
    eye = np.eye(3)
    cols = [quat_rotate(q, np.broadcast_to(eye[i], q.shape[:-1] + (3,))) for i in range(3)]
    return np.stack(cols, axis=-1)


# ------------------------------------------------------------- part rules
def cuboid_mass_properties(size: np.ndarray, density=CUBOID_DENSITY):
    """compile.rs:841-852: mass, local centre (0) and principal inertia."""
    size = np.asarray(size, np.float32)
    sx, sy, sz = size[..., 0], size[..., 1], size[..., 2]
    mass = (density * sx * sy * sz).astype(np.float32)
    twelve = np.float32(12.0)
    inertia = np.stack([mass * (sy * sy + sz * sz) / twelve,
                        mass * (sx * sx + sz * sz) / twelve,
                        mass * (sx * sx + sy * sy) / twelve], axis=-1).astype(np.float32)
    return mass, np.zeros(size.shape, np.float32), inertia


def cylinder_mass_properties(outer_diameter, inner_diameter, length, sweep_degrees=360.0,
                             density=CUBOID_DENSITY):
    """compile.rs:853-876: hollow cylinder sector about local Y, centroid on +X."""
    f = np.float32
    outer = f(np.asarray(outer_diameter, np.float32) * f(0.5))
    inner = f(np.asarray(inner_diameter, np.float32) * f(0.5))
    length = np.asarray(length, np.float32)
    sweep = np.float32(np.deg2rad(np.float32(sweep_degrees)))
    sweep = np.broadcast_to(sweep, outer.shape).astype(np.float32)
    radial_squared = outer * outer + inner * inner
    mass = (density * sweep * (outer * outer - inner * inner) * length * f(0.5)).astype(np.float32)
    sin_half = np.sin(sweep * f(0.5)).astype(np.float32)
    center_x = (f(4.0) * sin_half * (outer ** 3 - inner ** 3)
                / (f(3.0) * sweep * (outer * outer - inner * inner))).astype(np.float32)
    sin_sweep = np.sin(sweep).astype(np.float32)
    radial_parallel = radial_squared * (sweep + sin_sweep) / (f(4.0) * sweep)
    radial_perpendicular = radial_squared * (sweep - sin_sweep) / (f(4.0) * sweep)
    axial_variance = length * length / f(12.0)
    inertia = np.stack([
        mass * (axial_variance + radial_perpendicular),
        mass * (radial_parallel + radial_perpendicular - center_x * center_x),
        mass * (radial_parallel + axial_variance - center_x * center_x),
    ], axis=-1).astype(np.float32)
    local_center = np.stack([center_x, np.zeros_like(center_x), np.zeros_like(center_x)], axis=-1)
    return mass, local_center.astype(np.float32), inertia


def world_inertia(rotation: np.ndarray, principal: np.ndarray) -> np.ndarray:
    """R diag(I) R^T of one single-part compound (compile.rs:784-794, offset 0)."""
    r = quat_matrix(np.asarray(rotation, np.float64)).astype(np.float32)
    d = np.asarray(principal, np.float32)
    return np.einsum("...ij,...j,...kj->...ik", r, d, r).astype(np.float32)


def cylinder_segments(outer_diameter, inner_diameter, length, sweep_degrees=360.0):
    """compile.rs:896-926: per segment (local centre offset in part frame, yaw angle,
    half extents).  Returns arrays of shape (..., 16, 3), (..., 16), (..., 3)."""
    f = np.float32
    outer = np.asarray(outer_diameter, np.float32) * f(0.5)
    inner = np.asarray(inner_diameter, np.float32) * f(0.5)
    half_radial = (outer - inner) * f(0.5)
    center_radius = (outer + inner) * f(0.5)
    sweep = f(np.deg2rad(np.float32(sweep_degrees)))
    segment_angle = f(sweep / f(16.0))
    half_tangent = (outer * f(np.tan(segment_angle * f(0.5)))).astype(np.float32)
    start = f(-segment_angle * f(0.5)) if float(sweep_degrees) == 360.0 else f(-sweep * f(0.5))
    seg = np.arange(16, dtype=np.float32)
    angle = (start + segment_angle * (seg + f(0.5))).astype(np.float32)
    radial = np.stack([np.cos(angle), np.zeros_like(angle), np.sin(angle)], axis=-1).astype(np.float32)
    offset = radial * center_radius[..., None, None]
    half = np.stack([half_radial, np.asarray(length, np.float32) * f(0.5), half_tangent], axis=-1)
    return offset.astype(np.float32), angle, half.astype(np.float32), center_radius


# ------------------------------------------------------------------ scene
@dataclasses.dataclass
class Scene:
    """Flattened creation: exactly the arrays ``mk_create`` receives."""

    transforms: np.ndarray
    velocities: np.ndarray
    masses: np.ndarray
    spatial_inertias: np.ndarray
    colliders: np.ndarray
    bearings: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, abi.BEARING))
    suppressed_pairs: np.ndarray = dataclasses.field(default_factory=lambda: np.zeros(0, abi.PAIR))
    mechanism_bodies: np.ndarray | None = None
    root_flags: np.ndarray | None = None
    preorder: np.ndarray | None = None
    body_components: np.ndarray | None = None
    drives: np.ndarray | None = None
    coordinate_count: int = 0
    max_depth: int = 0
    closure_count: int = 0
    has_dynamic_root: int = 0
    name: str = "scene"
    scene_offsets: np.ndarray | None = None   # batched scenes: body offset per scene (+ total)

    @property
    def body_count(self) -> int:
        return int(self.transforms.shape[0])

    @property
    def collider_count(self) -> int:
        return int(self.colliders.shape[0])

    @property
    def bearing_count(self) -> int:
        return int(self.bearings.shape[0])

    def creation(self) -> abi.MkCreation:
        """ctypes view; the arrays must outlive the returned structure."""
        c = abi.MkCreation()
        c.body_count = self.body_count
        c.collider_count = self.collider_count
        c.bearing_count = self.bearing_count
        c.suppression_count = int(self.suppressed_pairs.shape[0])
        c.coordinate_count = int(self.coordinate_count)
        c.max_depth = int(self.max_depth)
        c.transforms = abi.ptr(self.transforms)
        c.velocities = abi.ptr(self.velocities)
        c.masses = abi.ptr(self.masses)
        c.spatial_inertias = abi.ptr(self.spatial_inertias)
        c.colliders = abi.ptr(self.colliders)
        c.bearings = abi.ptr(self.bearings) if self.bearing_count else None
        c.suppressed_pairs = abi.ptr(self.suppressed_pairs) if len(self.suppressed_pairs) else None
        c.mechanism_bodies = abi.ptr(self.mechanism_bodies)
        c.root_flags = abi.ptr(self.root_flags)
        c.preorder = abi.ptr(self.preorder)
        c.body_components = abi.ptr(self.body_components)
        c.drives = abi.ptr(self.drives)
        c.closure_count = int(self.closure_count)
        c.has_dynamic_root = int(self.has_dynamic_root)
        return c


def _body_rows(translation, inverse_inertia, inertia, mass, dynamic=True):
    """Mass rows of device.rs:449-477 for single-part compounds."""
    n = translation.shape[0]
    transforms = np.zeros(n, abi.TRANSFORM)
    transforms["position"][:, :3] = translation
    transforms["rotation"][:, 3] = 1.0                      # root_rotation = IDENTITY (compile.rs:333)
    masses = np.zeros(n, abi.MASS)
    inv_m = np.where(dynamic, np.float32(1.0) / mass, np.float32(0.0)).astype(np.float32)
    masses["inverse_mass"][:, 0] = inv_m
    masses["inverse_inertia_x"][:, :3] = inverse_inertia[:, :, 0]
    masses["inverse_inertia_y"][:, :3] = inverse_inertia[:, :, 1]
    masses["inverse_inertia_z"][:, :3] = inverse_inertia[:, :, 2]
    spatial = np.zeros(n, abi.SPATIAL_INERTIA)
    spatial["mass"][:, 0] = mass
    spatial["inertia_x"][:, :3] = inertia[:, :, 0]
    spatial["inertia_y"][:, :3] = inertia[:, :, 1]
    spatial["inertia_z"][:, :3] = inertia[:, :, 2]
    return transforms, masses, spatial


def _invert(m: np.ndarray) -> np.ndarray:
    return np.linalg.inv(m.astype(np.float64)).astype(np.float32)


def _assemble(translation, part_rotation, is_cylinder, outer_d, inner_d, length, cube_size,
              name, velocities=None, density=CUBOID_DENSITY):
    """Rows for single-part bodies: cuboids (cube_size) or full cylinders."""
    n = translation.shape[0]
    translation = np.asarray(translation, np.float32)
    part_rotation = np.asarray(part_rotation, np.float64)
    cube_idx = np.nonzero(~is_cylinder)[0]
    cyl_idx = np.nonzero(is_cylinder)[0]
    mass = np.zeros(n, np.float32)
    principal = np.zeros((n, 3), np.float32)
    local_c = np.zeros((n, 3), np.float32)
    size = np.broadcast_to(np.asarray(cube_size, np.float32), (len(cube_idx), 3))
    m, lc, pi = cuboid_mass_properties(size, density)
    mass[cube_idx], local_c[cube_idx], principal[cube_idx] = m, lc, pi
    if len(cyl_idx):
        m, lc, pi = cylinder_mass_properties(outer_d[cyl_idx], inner_d[cyl_idx], length[cyl_idx],
                                             360.0, density)
        mass[cyl_idx], local_c[cyl_idx], principal[cyl_idx] = m, lc, pi
    rot_f = part_rotation.astype(np.float32)
    com = (translation + quat_rotate(part_rotation, local_c.astype(np.float64))).astype(np.float32)
    inertia = world_inertia(part_rotation, principal)
    inverse = _invert(inertia)
    transforms, masses, spatial = _body_rows(com, inverse, inertia, mass)

    counts = np.where(is_cylinder, CYLINDER_COLLIDER_COUNT, 1).astype(np.int64)
    starts = np.concatenate([[0], np.cumsum(counts)[:-1]])
    total = int(counts.sum())
    colliders = np.zeros(total, abi.COLLIDER)
    body_of = np.repeat(np.arange(n, dtype=np.uint32), counts)
    colliders["metadata"][:, 0] = body_of
    colliders["metadata"][:, 1] = body_of          # source part slot (one part per body)
    colliders["metadata"][:, 2] = 0                # source generation
    # cuboids
    cs = starts[cube_idx]
    colliders["local_center"][cs, :3] = (translation[cube_idx] - com[cube_idx])
    colliders["local_rotation"][cs] = rot_f[cube_idx]
    colliders["half_extents"][cs, :3] = size * np.float32(0.5)
    # cylinders (compile.rs:896-926; ground data device.rs:3008-3045)
    if len(cyl_idx):
        offset, angle, half, center_radius = cylinder_segments(outer_d[cyl_idx], inner_d[cyl_idx],
                                                               length[cyl_idx])
        rq = part_rotation[cyl_idx]
        seg_rot = quat_mul(rq[:, None, :], quat_yaw(-angle.astype(np.float64))[None, :, :])
        seg_center = (translation[cyl_idx, None, :] - com[cyl_idx, None, :]
                      + quat_rotate(np.broadcast_to(rq[:, None, :], offset.shape[:-1] + (4,)),
                                    offset.astype(np.float64))).astype(np.float32)
        rows = starts[cyl_idx][:, None] + np.arange(16)[None, :]
        colliders["local_center"][rows, :3] = seg_center
        colliders["local_rotation"][rows] = seg_rot.astype(np.float32)
        colliders["half_extents"][rows, :3] = half[:, None, :]
        mean_center = seg_center.astype(np.float64).mean(axis=1, keepdims=True)
        cr = np.linalg.norm(seg_center[:, :1].astype(np.float64) - mean_center, axis=-1).astype(np.float32)
        outer_r = (cr[:, 0] + half[:, 0]).astype(np.float32)
        colliders["local_center"][rows, 3] = cr
        colliders["half_extents"][rows, 3] = outer_r[:, None]
        colliders["metadata"][rows, 3] = np.arange(1, 17, dtype=np.uint32)[None, :]
    vel = np.zeros(n, abi.VELOCITY) if velocities is None else velocities
    return Scene(transforms=transforms, velocities=vel, masses=masses, spatial_inertias=spatial,
                 colliders=colliders, root_flags=np.ones(n, np.uint32),
                 body_components=np.arange(n, dtype=np.uint32), name=name)


# -------------------------------------------------------------- configs
def falling_cubes(n: int = 1000, seed: int = 0, box: float = 10.0) -> Scene:
    """Plain method, small: n 0.25 m cubes, centres uniform in a box x z in
    [-box/2, box/2), y in [0.25, box + 0.25), uniform orientations, N(0, 1)
    linear and angular velocity per axis."""
    rng = Rng(seed)
    x = rng.uniform("x", n, -box / 2, box / 2)
    y = rng.uniform("y", n, 0.25, box + 0.25)
    z = rng.uniform("z", n, -box / 2, box / 2)
    translation = np.stack([x, y, z], 1).astype(np.float32)
    rotation = rng.unit_quaternions("q", n)
    vel = np.zeros(n, abi.VELOCITY)
    vel["linear"][:, 0] = rng.normal("vx", n)
    vel["linear"][:, 1] = rng.normal("vy", n)
    vel["linear"][:, 2] = rng.normal("vz", n)
    vel["angular"][:, 0] = rng.normal("wx", n)
    vel["angular"][:, 1] = rng.normal("wy", n)
    vel["angular"][:, 2] = rng.normal("wz", n)
    zeros = np.zeros(n)
    return _assemble(translation, rotation, np.zeros(n, bool), zeros, zeros, zeros,
                     (0.25, 0.25, 0.25), f"falling_cubes_{n}", vel)


def stack_grid(nx: int = 50, ny: int = 40, nz: int = 50, seed: int = 0, spacing: float = 0.26,
               cylinder_fraction: float = 0.2, jitter: float = 0.005) -> Scene:
    """Plain method at scale: bodies on an nx*ny*nz grid (spacing 0.26 m) above the
    ground, jitter U(-0.005, 0.005) m, yaw U(0, 2 pi); 80% 0.25 m cubes, 20% hollow
    cylinders (outer diameter U(0.25, 1), inner U(0, outer - 0.05), length
    U(0.25, 2), 360 degrees) with 16 OBB segments each, density 1000 kg/m^3."""
    rng = Rng(seed)
    n = nx * ny * nz
    idx = np.arange(n)
    ix, iy, iz = idx % nx, (idx // nx) % ny, idx // (nx * ny)
    x = (ix - (nx - 1) * 0.5) * spacing + rng.uniform("jx", n, -jitter, jitter)
    y = spacing * 0.5 + iy * spacing + rng.uniform("jy", n, -jitter, jitter)
    z = (iz - (nz - 1) * 0.5) * spacing + rng.uniform("jz", n, -jitter, jitter)
    translation = np.stack([x, y, z], 1).astype(np.float32)
    rotation = quat_yaw(rng.uniform("yaw", n, 0.0, 2.0 * math.pi))
    is_cyl = rng.uniform("kind", n) < cylinder_fraction
    outer = rng.uniform("outer", n, 0.25, 1.0).astype(np.float32)
    inner = (rng.uniform("inner", n) * (outer - 0.05)).astype(np.float32)
    length = rng.uniform("length", n, 0.25, 2.0).astype(np.float32)
    return _assemble(translation, rotation, is_cyl, outer, inner, length, (0.25, 0.25, 0.25),
                     f"stack_grid_{nx}x{ny}x{nz}")


def config_plain_small(seed: int = 0) -> Scene:
    """1,000 falling cubes (the reference's CPU-runnable case)."""
    return falling_cubes(1000, seed)


def config_plain_scale(seed: int = 0) -> Scene:
    """100,000 bodies on a 50x40x50 grid, 20% cylinders."""
    return stack_grid(50, 40, 50, seed)


def config_full(seed: int = 0, grid: int = 100, chains: int = 50_000) -> Scene:
    """The full form at scale: the 100,000-body mix on a grid x grid x grid lattice
    (1,000,000 bodies at grid 100) and `chains` five-body bearing chains (10%
    loop-closed), laid out 100 m beside the lattice so the two do not overlap."""
    lattice = stack_grid(grid, grid, grid, seed)
    field = translated(bearing_chains(chains, 5, seed=seed + 1, closure_fraction=0.1), (100.0, 0.0, 0.0))
    scene, _ = concatenate([lattice, field])
    return scene


def with_suppression(scene: Scene, body_pairs: np.ndarray) -> Scene:
    """Adds sorted, de-duplicated suppressed body pairs (compile.rs:373, ordered_pair)."""
    p = np.sort(np.asarray(body_pairs, np.uint32).reshape(-1, 2), axis=1)
    p = np.unique(p, axis=0)
    rows = np.zeros(len(p), abi.PAIR)
    rows["collider_a"], rows["collider_b"] = p[:, 0], p[:, 1]
    return dataclasses.replace(scene, suppressed_pairs=rows)


def compound_mass_properties(parts, density=CUBOID_DENSITY):
    """compile.rs:768-821 for a weld group: parts are (kind, translation, rotation xyzw,
    size) with kind "cuboid" (size = edge lengths) or "cylinder" (size = outer diameter,
    inner diameter, length; 360 degrees).  Returns (mass, centre of mass, inertia 3x3)
    about the centre of mass in world axes."""
    props = []
    for kind, translation, rotation, size in parts:
        rotation = np.asarray(rotation, np.float64)
        if kind == "cuboid":
            m, lc, pi = cuboid_mass_properties(np.asarray(size, np.float32)[None, :], density)
        else:
            m, lc, pi = cylinder_mass_properties(*(np.float32(s) for s in size), 360.0, density)
            m, lc, pi = np.atleast_1d(m), np.atleast_2d(lc), np.atleast_2d(pi)
        center = np.asarray(translation, np.float64) + quat_rotate(rotation, lc[0].astype(np.float64))
        props.append((float(m[0]), center, rotation, pi[0].astype(np.float64)))
    total = sum(p[0] for p in props)
    com = sum(p[0] * p[1] for p in props) / total
    inertia = np.zeros((3, 3))
    for m, center, rotation, principal in props:
        r = quat_matrix(rotation)
        own = r @ np.diag(principal) @ r.T
        off = center - com
        inertia += own + m * (np.eye(3) * off.dot(off) - np.outer(off, off))
    return np.float32(total), com.astype(np.float32), inertia.astype(np.float32)


REFERENCE_DENSITY = np.float32(500.0)   # CUBOID_DENSITY_KG_M3 (mechanic-core lib.rs:35)


def dense_grid(count: int = 100_000) -> Scene:
    """mechanic-bench's dense scene (crates/mechanic-bench/src/main.rs:442-454): `count`
    one-metre cubes on a 50 x 40 x z grid of 1 m pitch, centres at (x, y + 0.5, z), resting
    and touching, reference density 500 kg/m^3, zero velocity."""
    idx = np.arange(count)
    x = (idx % 50).astype(np.float32)
    y = ((idx // 50) % 40).astype(np.float32) + np.float32(0.5)
    z = (idx // 2000).astype(np.float32)
    translation = np.stack([x, y, z], 1).astype(np.float32)
    rotation = np.zeros((count, 4))
    rotation[:, 3] = 1.0
    zeros = np.zeros(count)
    return _assemble(translation, rotation, np.zeros(count, bool), zeros, zeros, zeros, (1.0, 1.0, 1.0),
                     f"dense_{count}", density=REFERENCE_DENSITY)


def _unit_vectors(rng: Rng, name: str, n: int) -> np.ndarray:
    """Uniform directions on the sphere."""
    z = rng.uniform(name + ".z", n, -1.0, 1.0)
    phi = rng.uniform(name + ".phi", n, 0.0, 2.0 * math.pi)
    r = np.sqrt(np.maximum(0.0, 1.0 - z * z))
    return np.stack([r * np.cos(phi), r * np.sin(phi), z], axis=1)


def _mechanism_rows(scene: Scene, parents: np.ndarray, tree_bearing: np.ndarray, components: np.ndarray,
                    depth: np.ndarray, preorder_pos: np.ndarray, postorder_pos: np.ndarray) -> None:
    """GpuMechanismBody rows (device.rs:1699-1760) for identity root rotations."""
    n = scene.body_count
    rows = np.zeros(n, abi.MECHANISM_BODY)
    root = parents < 0
    idx = np.arange(n, dtype=np.uint32)
    rows["metadata"][:, 0] = np.where(root, idx, parents.astype(np.int64)).astype(np.uint32)
    rows["metadata"][:, 1] = np.where(root, abi.INVALID_INDEX, tree_bearing.astype(np.int64)).astype(np.uint32)
    rows["metadata"][:, 2] = 0                       # bearing.compound_a is the parent
    rows["metadata"][:, 3] = root.astype(np.uint32)
    rows["traversal"][:, 0] = components
    rows["traversal"][:, 1] = depth
    rows["traversal"][:, 2] = preorder_pos
    rows["traversal"][:, 3] = postorder_pos
    p = scene.transforms["position"][:, :3]
    rel = np.where(root[:, None], 0.0, p - p[np.maximum(parents, 0)])
    rows["bind_relative_position"][:, :3] = rel.astype(np.float32)
    rows["bind_relative_rotation"][:, 3] = 1.0
    scene.mechanism_bodies = rows
    scene.root_flags = root.astype(np.uint32)
    order = np.argsort(preorder_pos, kind="stable")
    scene.preorder = order.astype(np.uint32)
    scene.body_components = components.astype(np.uint32)


def bearing_chains(chains: int = 4000, links: int = 5, seed: int = 0, closure_fraction: float = 0.1,
                   driven_fraction: float = 0.5, size: float = 0.25, height: float = 1.0,
                   columns: int = 40, pitch_x: float = 1.5, pitch_z: float = 0.5) -> Scene:
    """Articulated config: `chains` serial chains of `links` 0.25 m cubes (density 1000)
    joined face to face by revolute bearings with random unit axes, travel limits
    U(+-30, +-180) degrees, half of them driven at U(-3, 3) rad/s (max speed 3 rad/s,
    unlimited torque, the DriveLimits defaults of mechanic-core drive.rs:534, 650-651),
    and a loop-closure bearing between the first and last body of `closure_fraction`
    of the chains.  Chains lie along x at `height` on a grid; roots are dynamic."""
    rng = Rng(seed)
    n = chains * links
    c = np.arange(chains)
    cx, cz = c % columns, c // columns
    x0 = (cx - (columns - 1) * 0.5) * pitch_x
    z0 = (cz - (chains // columns - 1) * 0.5) * pitch_z
    k = np.arange(links)
    x = (x0[:, None] + (k[None, :] - (links - 1) * 0.5) * size).reshape(-1)
    translation = np.stack([x, np.full(n, height), np.repeat(z0, links)], 1).astype(np.float32)
    rotation = np.zeros((n, 4))
    rotation[:, 3] = 1.0
    zeros = np.zeros(n)
    scene = _assemble(translation, rotation, np.zeros(n, bool), zeros, zeros, zeros, (size, size, size),
                      f"chains_{chains}x{links}")
    has_closure = rng.uniform("closure", chains) < closure_fraction
    tree_axes = _unit_vectors(rng, "axis", chains * (links - 1)).reshape(chains, links - 1, 3)
    closure_axes = _unit_vectors(rng, "closure_axis", chains)
    # bearing rows: per chain its links-1 tree bearings, then its closure (if any)
    per_chain = (links - 1) + has_closure.astype(np.int64)
    first_row = np.concatenate([[0], np.cumsum(per_chain)[:-1]])
    J = int(per_chain.sum())
    bearings = np.zeros(J, abi.BEARING)
    coord_of_row = np.full(J, abi.INVALID_INDEX, np.uint32)
    parents = np.full(n, -1, np.int64)
    tree_bearing = np.full(n, -1, np.int64)
    depth = np.tile(k, chains).astype(np.uint32)
    pos = translation.astype(np.float64)
    for j in range(links - 1):
        rows = first_row + j
        a = c * links + j
        b = a + 1
        anchor = pos[a] + np.array([size * 0.5, 0.0, 0.0])
        bearings["local_anchor_a"][rows, :3] = anchor - pos[a]
        bearings["local_anchor_b"][rows, :3] = anchor - pos[b]
        bearings["local_axis_a"][rows, :3] = tree_axes[:, j]
        bearings["local_axis_b"][rows, :3] = tree_axes[:, j]
        bearings["metadata"][rows, 0] = a
        bearings["metadata"][rows, 1] = b
        coords = c * (links - 1) + j
        bearings["metadata"][rows, 2] = coords
        coord_of_row[rows] = coords
        parents[b] = a
        tree_bearing[b] = rows
    closed = np.nonzero(has_closure)[0]
    rows = first_row[closed] + (links - 1)
    a = closed * links
    b = a + links - 1
    anchor = 0.5 * (pos[a] + pos[b])
    bearings["local_anchor_a"][rows, :3] = anchor - pos[a]
    bearings["local_anchor_b"][rows, :3] = anchor - pos[b]
    bearings["local_axis_a"][rows, :3] = closure_axes[closed]
    bearings["local_axis_b"][rows, :3] = closure_axes[closed]
    bearings["metadata"][rows, 0] = a
    bearings["metadata"][rows, 1] = b
    bearings["metadata"][rows, 2] = abi.INVALID_INDEX
    bearings["metadata"][rows, 3] = 1
    scene.bearings = bearings
    Q = chains * (links - 1)
    limit = np.deg2rad(rng.uniform("limit", Q, 30.0, 180.0)).astype(np.float32)
    drives = np.zeros(Q, abi.MECHANISM_DRIVE)
    driven = rng.uniform("driven", Q) < driven_fraction
    drives["mode"] = np.where(driven, abi.DRIVE_MODE_SPEED, abi.DRIVE_MODE_PASSIVE)
    drives["max_acceleration"] = np.where(driven, np.inf, 0.0)
    drives["max_speed"] = np.where(driven, 3.0, 0.0)
    drives["target_speed"] = np.where(driven, rng.uniform("target", Q, -3.0, 3.0), 0.0)
    drives["min_angle"] = -limit
    drives["max_angle"] = limit
    scene.drives = drives
    scene.coordinate_count = Q
    scene.max_depth = links - 1
    scene.closure_count = int(len(closed))
    scene.has_dynamic_root = 1
    comp = np.repeat(c, links).astype(np.uint32)
    _mechanism_rows(scene, parents, tree_bearing, comp, depth, np.arange(n, dtype=np.uint32),
                    np.arange(n, dtype=np.uint32))
    pairs = np.stack([bearings["metadata"][:, 0], bearings["metadata"][:, 1]], 1)
    return with_suppression(scene, pairs)


def four_bar(invalid: bool = False) -> Scene:
    """mechanic-bench's four_bar / invalid_loop (crates/mechanic-bench/src/main.rs:372-440):
    four 1 m cubes at (0,0,0), (1,0,0), (1,1,0), (0,1,0) joined by bearings about X, Y, -X, -Y
    at the shared face centres; the last edge closes the loop.  `invalid` moves the closure's
    anchor on body b by (0.2, 0.13, 0.07) m (main.rs:431-438)."""
    translation = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    rotation = np.zeros((4, 4))
    rotation[:, 3] = 1.0
    zeros = np.zeros(4)
    scene = _assemble(translation, rotation, np.zeros(4, bool), zeros, zeros, zeros, (1.0, 1.0, 1.0),
                      "invalid_loop" if invalid else "four_bar", density=REFERENCE_DENSITY)
    edges = [(0, 1, (0.5, 0, 0), (1, 0, 0)), (1, 2, (1, 0.5, 0), (0, 1, 0)),
             (2, 3, (0.5, 1, 0), (-1, 0, 0)), (3, 0, (0, 0.5, 0), (0, -1, 0))]
    bearings = np.zeros(4, abi.BEARING)
    for r, (a, b, anchor, axis) in enumerate(edges):
        anchor = np.array(anchor, np.float32)
        bearings["local_anchor_a"][r, :3] = anchor - translation[a]
        bearings["local_anchor_b"][r, :3] = anchor - translation[b]
        bearings["local_axis_a"][r, :3] = axis
        bearings["local_axis_b"][r, :3] = axis
        bearings["metadata"][r] = (a, b, r if r < 3 else abi.INVALID_INDEX, 0 if r < 3 else 1)
    if invalid:
        bearings["local_anchor_b"][3, :3] += np.array([0.2, 0.13, 0.07], np.float32)
    scene.bearings = bearings
    scene.drives = abi.passive_drive_rows(3)
    scene.coordinate_count = 3
    scene.max_depth = 3
    scene.closure_count = 1
    scene.has_dynamic_root = 1
    _mechanism_rows(scene, np.array([-1, 0, 1, 2]), np.array([-1, 0, 1, 2]), np.zeros(4, np.uint32),
                    np.arange(4, dtype=np.uint32), np.arange(4, dtype=np.uint32),
                    np.array([3, 2, 1, 0], np.uint32))
    return with_suppression(scene, [(0, 1), (1, 2), (2, 3), (3, 0)])


# ---------------------------------------------------- mechanism compilation
class _DisjointSet:
    """Union by rank with path compression; on equal ranks the first argument's root
    stays the root (compile.rs:936-976), so representatives match the reference's."""

    def __init__(self, n: int):
        self.parent = list(range(n))
        self.rank = [0] * n

    def find(self, item: int) -> int:
        root = item
        while self.parent[root] != root:
            root = self.parent[root]
        while self.parent[item] != item:
            self.parent[item], item = root, self.parent[item]
        return root

    def union(self, a: int, b: int) -> None:
        ra, rb = self.find(a), self.find(b)
        if ra == rb:
            return
        if self.rank[ra] < self.rank[rb]:
            ra, rb = rb, ra
        self.parent[rb] = ra
        if self.rank[ra] == self.rank[rb]:
            self.rank[ra] += 1


def compile_mechanism(scene: Scene, body_a, body_b, anchors, axes, driven=None, drives=None) -> Scene:
    """Bearing topology of a creation, as mechanic-core's compile does it, for bearings
    given in graph order as (body a, body b, shared world anchor, world axis); bodies are
    single compounds with identity root rotation (compile.rs:333), so a bearing's local
    anchors are the anchor minus each body's centre and both local axes are the axis.

    Restates compile.rs:394-475 (spanning forest: driven bearings first, then the rest, in
    graph order, never joining two fixed trees; tree bearings get coordinates in graph
    order, the others are loop closures), :477-486 (mechanism components: bearing-connected
    bodies keyed by their union-find representative), :504-609 (BFS from each component's
    static bodies, else its first body, over tree bearings sorted by (neighbour, bearing,
    direction); postorder by depth descending, then body) and device.rs:1699-1760 (the
    GpuMechanismBody rows).  `drives` (one GpuMechanismDrive per coordinate) defaults to
    passive rows.  Returns the scene with bearings, drives, mechanism rows and the
    bearing-connected body pairs suppressed (compile.rs:373)."""
    n = scene.body_count
    a = np.asarray(body_a, np.int64)
    b = np.asarray(body_b, np.int64)
    J = len(a)
    anchors = np.asarray(anchors, np.float64).reshape(J, 3)
    axes = np.asarray(axes, np.float32).reshape(J, 3)
    driven = np.zeros(J, bool) if driven is None else np.asarray(driven, bool)
    static = scene.masses["inverse_mass"][:, 0] == 0.0
    # spanning forest (compile.rs:401-425)
    forest = _DisjointSet(n)
    fixed = static.tolist()
    tree = np.zeros(J, bool)
    al, bl = a.tolist(), b.tolist()
    for driven_pass in (True, False):
        for j in np.nonzero(driven == driven_pass)[0].tolist():
            ra, rb = forest.find(al[j]), forest.find(bl[j])
            if ra == rb or (fixed[ra] and fixed[rb]):
                continue
            has_fixed = fixed[ra] or fixed[rb]
            forest.union(ra, rb)
            fixed[forest.find(ra)] = has_fixed
            tree[j] = True
    if np.any(driven & ~tree):
        raise ValueError("a driven bearing closes a loop (TopologyError::DrivenClosureBearing)")
    coord = np.full(J, abi.INVALID_INDEX, np.uint32)
    coord[tree] = np.arange(int(tree.sum()), dtype=np.uint32)
    pos = scene.transforms["position"][:, :3].astype(np.float64)
    rows = np.zeros(J, abi.BEARING)
    rows["local_anchor_a"][:, :3] = (anchors - pos[a]).astype(np.float32)
    rows["local_anchor_b"][:, :3] = (anchors - pos[b]).astype(np.float32)
    rows["local_axis_a"][:, :3] = axes
    rows["local_axis_b"][:, :3] = axes
    rows["metadata"][:, 0] = a
    rows["metadata"][:, 1] = b
    rows["metadata"][:, 2] = coord
    rows["metadata"][:, 3] = (~tree).astype(np.uint32)
    # mechanism components (compile.rs:348, :477-484): representative order, bodies ascending
    comps = _DisjointSet(n)
    for j in range(J):
        comps.union(al[j], bl[j])
    rep = np.array([comps.find(i) for i in range(n)], np.int64)
    reps, first = np.unique(rep, return_index=True)          # ascending representative
    component_of = np.searchsorted(reps, rep).astype(np.uint32)
    members = [np.nonzero(rep == r)[0] for r in reps] if len(reps) < 64 else None
    # adjacency over tree bearings, sorted by (neighbour, bearing row, direction)
    ta, tb, tj = a[tree], b[tree], np.nonzero(tree)[0]
    nb = np.concatenate([tb, ta])
    src = np.concatenate([ta, tb])
    jj = np.concatenate([tj, tj])
    dirn = np.concatenate([np.zeros(len(tj), np.int64), np.ones(len(tj), np.int64)])
    order = np.lexsort((dirn, jj, nb, src))
    src, nb, jj, dirn = src[order], nb[order], jj[order], dirn[order]
    starts = np.searchsorted(src, np.arange(n + 1))
    parent = np.full(n, -1, np.int64)
    tree_bearing = np.full(n, -1, np.int64)
    direction = np.zeros(n, np.uint32)
    depth = np.zeros(n, np.int64)
    pre = np.zeros(n, np.int64)
    visited = np.zeros(n, bool)
    count = 0
    from collections import deque
    nb_l, jj_l, dir_l, st_l = nb.tolist(), jj.tolist(), dirn.tolist(), starts.tolist()
    for ci, r in enumerate(reps.tolist()):
        body_list = members[ci] if members is not None else np.nonzero(rep == r)[0]
        roots = [int(x) for x in body_list if static[x]] or [int(body_list[0])]
        for root in roots:
            if visited[root]:
                continue
            visited[root] = True
            queue = deque([root])
            while queue:
                p = queue.popleft()
                pre[p] = count
                count += 1
                for e in range(st_l[p], st_l[p + 1]):
                    c = nb_l[e]
                    if visited[c]:
                        continue
                    visited[c] = True
                    parent[c] = p
                    tree_bearing[c] = jj_l[e]
                    direction[c] = dir_l[e]
                    depth[c] = depth[p] + 1
                    queue.append(c)
    post_order = np.lexsort((np.arange(n), -depth))
    post = np.zeros(n, np.int64)
    post[post_order] = np.arange(n)
    scene = dataclasses.replace(scene, bearings=rows)
    q = int(tree.sum())
    scene.drives = abi.passive_drive_rows(q) if drives is None else drives
    scene.coordinate_count = q
    scene.max_depth = int(depth.max()) if n else 0
    scene.closure_count = int((~tree).sum())
    root = parent < 0
    scene.has_dynamic_root = int(np.any(root & ~static))
    _mechanism_rows(scene, parent, tree_bearing, component_of, depth.astype(np.uint32), pre.astype(np.uint32),
                    post.astype(np.uint32))
    scene.mechanism_bodies["metadata"][:, 2] = np.where(root, 0, direction).astype(np.uint32)
    return with_suppression(scene, np.stack([a, b], 1))


def loops_grid(width: int = 100, height: int = 100, depth: int = 10) -> Scene:
    """mechanic-bench's loops_100k (crates/mechanic-bench/src/main.rs:456-524): a width x
    height x depth lattice of one-metre cubes at 1 m pitch, centres at (x, y, z) metres,
    reference density 500 kg/m^3; in every z layer each cube is joined to its +x
    neighbour by a bearing about X at the shared face centre and to its +y neighbour by
    one about Y, and the (0, 0) cubes of consecutive layers by bearings about Z.  At
    100 x 100 x 10: 100,000 bodies, 198,009 bearings, 99,999 tree coordinates and 98,010
    loop closures."""
    part = lambda x, y, z: (z * height + y) * width + x   # noqa: E731
    n = width * height * depth
    idx = np.arange(n)
    x, y, z = idx % width, (idx // width) % height, idx // (width * height)
    translation = np.stack([x, y, z], 1).astype(np.float32)
    rotation = np.zeros((n, 4))
    rotation[:, 3] = 1.0
    zeros = np.zeros(n)
    scene = _assemble(translation, rotation, np.zeros(n, bool), zeros, zeros, zeros, (1.0, 1.0, 1.0),
                      f"loops_{n}", density=REFERENCE_DENSITY)
    A, Bb, anchor, axis = [], [], [], []
    gx, gy = np.meshgrid(np.arange(width - 1), np.arange(height), indexing="xy")
    hx, hy = np.meshgrid(np.arange(width), np.arange(height - 1), indexing="xy")
    for zz in range(depth):
        xa = part(gx, gy, zz).ravel()
        A.append(xa)
        Bb.append(xa + 1)
        anchor.append(np.stack([gx.ravel() + 0.5, gy.ravel(), np.full(gx.size, zz)], 1))
        axis.append(np.tile([1.0, 0.0, 0.0], (gx.size, 1)))
        ya = part(hx, hy, zz).ravel()
        A.append(ya)
        Bb.append(ya + width)
        anchor.append(np.stack([hx.ravel(), hy.ravel() + 0.5, np.full(hx.size, zz)], 1))
        axis.append(np.tile([0.0, 1.0, 0.0], (hx.size, 1)))
    zs = np.arange(depth - 1)
    A.append(part(0, 0, zs))
    Bb.append(part(0, 0, zs + 1))
    anchor.append(np.stack([np.zeros(depth - 1), np.zeros(depth - 1), zs + 0.5], 1))
    axis.append(np.tile([0.0, 0.0, 1.0], (depth - 1, 1)))
    return compile_mechanism(scene, np.concatenate(A), np.concatenate(Bb), np.concatenate(anchor),
                             np.concatenate(axis))


# ------------------------------------------------------------ batched scenes
def translated(scene: Scene, offset) -> Scene:
    """The scene moved by `offset` (x, y, z)."""
    tr = scene.transforms.copy()
    tr["position"][:, :3] += np.asarray(offset, np.float32)
    return dataclasses.replace(scene, transforms=tr)


def concatenate(scene_list) -> tuple[Scene, np.ndarray]:
    """Scenes as one creation, rows concatenated scene by scene with body, bearing,
    coordinate and mechanism-component indices offset (the layout mk_create_batch
    builds).  Returns (combined scene, scene index of each collider)."""
    any_mech = any(s.max_depth > 0 for s in scene_list)
    parts = {k: [] for k in ("transforms", "velocities", "masses", "inertias", "colliders", "bearings",
                             "suppressed", "mech", "roots", "preorder", "components", "drives", "scene")}
    bo = jo = qo = comp_o = 0
    max_depth = closures = dyn = 0
    for si, s in enumerate(scene_list):
        n = s.body_count
        parts["transforms"].append(s.transforms)
        parts["velocities"].append(s.velocities if s.velocities is not None else np.zeros(n, abi.VELOCITY))
        parts["masses"].append(s.masses)
        parts["inertias"].append(s.spatial_inertias if s.spatial_inertias is not None
                                 else np.zeros(n, abi.SPATIAL_INERTIA))
        col = s.colliders.copy()
        col["metadata"][:, 0] += bo
        parts["colliders"].append(col)
        parts["scene"].append(np.full(s.collider_count, si, np.uint32))
        br = s.bearings.copy()
        if len(br):
            br["metadata"][:, 0] += bo
            br["metadata"][:, 1] += bo
            valid = br["metadata"][:, 2] != abi.INVALID_INDEX
            br["metadata"][valid, 2] += qo
        parts["bearings"].append(br)
        sp = s.suppressed_pairs.copy()
        if len(sp):
            sp["collider_a"] += bo
            sp["collider_b"] += bo
        parts["suppressed"].append(sp)
        comp = (s.body_components.astype(np.int64) if s.body_components is not None else np.arange(n))
        parts["components"].append((comp + comp_o).astype(np.uint32))
        parts["roots"].append(s.root_flags.astype(np.uint32) if s.root_flags is not None else np.ones(n, np.uint32))
        if any_mech:
            if s.max_depth > 0:
                mb = s.mechanism_bodies.copy()
                mb["metadata"][:, 0] += bo
                valid = mb["metadata"][:, 1] != abi.INVALID_INDEX
                mb["metadata"][valid, 1] += jo
                mb["traversal"][:, 0] += comp_o
                mb["traversal"][:, 2] += bo
                mb["traversal"][:, 3] += bo
                parts["preorder"].append((s.preorder.astype(np.int64) + bo).astype(np.uint32))
            else:
                mb = np.zeros(n, abi.MECHANISM_BODY)
                idx = np.arange(n, dtype=np.uint32) + np.uint32(bo)
                mb["metadata"][:, 0] = idx
                mb["metadata"][:, 1] = abi.INVALID_INDEX
                mb["metadata"][:, 3] = 1
                mb["traversal"][:, 0] = (comp + comp_o).astype(np.uint32)
                mb["traversal"][:, 2] = idx
                mb["traversal"][:, 3] = idx
                mb["bind_relative_rotation"][:, 3] = 1.0
                parts["preorder"].append(idx)
            parts["mech"].append(mb)
        q = int(s.coordinate_count)
        parts["drives"].append(s.drives if s.drives is not None else abi.passive_drive_rows(q))
        max_depth = max(max_depth, int(s.max_depth))
        closures += int(s.closure_count)
        dyn |= int(s.has_dynamic_root)
        bo += n
        jo += s.bearing_count
        qo += q
        comp_o += int(comp.max()) + 1 if n else 0
    cat = lambda k, dt: np.concatenate(parts[k]) if parts[k] else np.zeros(0, dt)  # noqa: E731
    combined = Scene(
        transforms=cat("transforms", abi.TRANSFORM), velocities=cat("velocities", abi.VELOCITY),
        masses=cat("masses", abi.MASS), spatial_inertias=cat("inertias", abi.SPATIAL_INERTIA),
        colliders=cat("colliders", abi.COLLIDER), bearings=cat("bearings", abi.BEARING),
        suppressed_pairs=cat("suppressed", abi.PAIR),
        mechanism_bodies=cat("mech", abi.MECHANISM_BODY) if any_mech else None,
        root_flags=cat("roots", np.uint32), preorder=cat("preorder", np.uint32) if any_mech else None,
        body_components=cat("components", np.uint32), drives=cat("drives", abi.MECHANISM_DRIVE) if qo else None,
        coordinate_count=qo, max_depth=max_depth, closure_count=closures, has_dynamic_root=dyn,
        name="+".join(s.name for s in scene_list[:3]) + ("..." if len(scene_list) > 3 else ""))
    return combined, np.concatenate(parts["scene"]) if parts["scene"] else np.zeros(0, np.uint32)


def take_bodies(scene: Scene, n: int) -> Scene:
    """The first n bodies of a scene without bearings (colliders are contiguous per body)."""
    assert scene.bearing_count == 0 and scene.max_depth == 0
    keep = scene.colliders["metadata"][:, 0] < n
    return dataclasses.replace(scene, transforms=scene.transforms[:n], velocities=scene.velocities[:n],
                               masses=scene.masses[:n], spatial_inertias=scene.spatial_inertias[:n],
                               colliders=scene.colliders[keep],
                               root_flags=None if scene.root_flags is None else scene.root_flags[:n],
                               body_components=None if scene.body_components is None else scene.body_components[:n])


def mixed_scene(n: int, seed: int, bearing_fraction: float = 0.02) -> Scene:
    """One scene of the batched config: n bodies, the 100,000-body config's cube/cylinder
    mix on a 0.26 m grid, with about `bearing_fraction` of the bodies in five-link
    bearing chains (10% of them loop-closed) beside the grid."""
    chain_links = 5
    chains = int(round(bearing_fraction * n / chain_links))
    n_grid = max(1, n - chains * chain_links)
    ny = max(1, int(round(n_grid ** (1.0 / 3.0) * 0.75)))
    nx = max(1, int(math.ceil(math.sqrt(n_grid / ny))))
    nz = max(1, int(math.ceil(n_grid / (nx * ny))))
    grid = take_bodies(stack_grid(nx, ny, nz, seed=seed), n_grid)
    if chains == 0:
        return dataclasses.replace(grid, name=f"mixed_{n}_{seed}")
    ch = bearing_chains(chains=chains, links=chain_links, seed=seed + 7919, closure_fraction=0.1, height=0.3,
                        columns=max(1, min(chains, 8)))
    ch = translated(ch, (nx * 0.13 + 2.0, 0.0, 0.0))
    combined, _ = concatenate([grid, ch])
    return dataclasses.replace(combined, name=f"mixed_{n}_{seed}")


def batched_uneven(count: int = 256, seed: int = 0, lo: int = 64, hi: int = 8192,
                   bearing_fraction: float = 0.02) -> list[Scene]:
    """Batched config: `count` independent scenes with body counts log-uniform in
    [lo, hi], each a mixed scene seeded by its index (seed + index)."""
    rng = Rng(seed)
    u = rng.uniform("batch_sizes", count)
    sizes = np.floor(np.exp(np.log(lo) + u * (np.log(hi) - np.log(lo)))).astype(np.int64)
    return [mixed_scene(int(sizes[i]), seed + i, bearing_fraction) for i in range(count)]
