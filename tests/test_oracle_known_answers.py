"""The CPU oracle pinned against the reference's own known answers.

collision.rs:185-233 (CPU narrowphase tests) are restated for both the CPU
SAT of collision.rs and the GPU kernel order of collision.wgsl:393-486;
compile.rs:1010-1142 pin the mass rules of the scene generator; and the
fixtures in tests/golden/known_answers.json (generated by
tests/golden/make_known_answers.py from the values in the reference's test
sources) are checked here.
"""
import json
import math
import os

import numpy as np
import pytest

import oracle
from mechanic_b200 import abi, scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "known_answers.json")
IDENTITY = np.array([0, 0, 0, 1], np.float32)
HALF = np.full(3, 0.5, np.float32)


def box(center, quat=IDENTITY, half=HALF):
    """16-float world box for oracle.obb_sat: rows {c, hx}, {ax, hy}, {ay, hz}, {az, 0}."""
    m = scenes.quat_matrix(np.asarray(quat, np.float64)).astype(np.float32)
    b = np.zeros((4, 4), np.float32)
    b[0, :3] = center
    b[0, 3], b[1, 3], b[2, 3] = half
    b[1, :3], b[2, :3], b[3, :3] = m[:, 0], m[:, 1], m[:, 2]
    return b.reshape(-1)


def yaw(angle):
    return scenes.quat_yaw(np.float64(angle)).astype(np.float32)


# ---------------------------------------------------- collision.rs:199-232
def test_cpu_sat_rejects_separated_boxes():
    assert oracle.cpu_obb_sat([0, 0, 0], IDENTITY, HALF, [1.01, 0, 0], IDENTITY, HALF) is None


def test_cpu_sat_finds_minimum_face_axis():
    n, pen = oracle.cpu_obb_sat([0, 0, 0], IDENTITY, HALF, [0.75, 0, 0], IDENTITY, HALF)
    assert np.allclose(n, [1, 0, 0], atol=1e-6)
    assert abs(pen - 0.25) < 1e-6


def test_cpu_face_contact_retains_four_stable_points():
    n, pen, pts = oracle.cpu_contact_manifold([0, 0, 0], IDENTITY, HALF, [1, 0, 0], IDENTITY, HALF)
    assert len(pts) == 4
    assert np.all(np.abs(pts[:, 0] - 0.5) < 1e-6)


def test_cpu_rotated_edge_overlap_is_detected():
    assert oracle.cpu_obb_sat([0, 0, 0], IDENTITY, HALF, [0.8, 0, 0], yaw(math.pi / 4), HALF) is not None


# The same answers from the GPU-order SAT (collision.wgsl:393-486), which
# emits a contact unless the penetration is below -1e-5.
def test_gpu_sat_separated_boxes_do_not_emit():
    np_out, feat = oracle.obb_sat(box([0, 0, 0]), box([1.01, 0, 0]))
    assert np_out[3] < -1e-5 and feat & (1 << 16)      # early exit on the separating axis
    assert feat & 0xFF == 0                             # axis A0


def test_gpu_sat_minimum_face_axis():
    np_out, feat = oracle.obb_sat(box([0, 0, 0]), box([0.75, 0, 0]))
    assert np.allclose(np_out[:3], [1, 0, 0], atol=1e-6) and abs(np_out[3] - 0.25) < 1e-6
    assert feat & 0xFF == 0 and not feat & (1 << 16)


def test_gpu_contact_point_of_face_contact_lies_on_the_face():
    a, b = box([0, 0, 0]), box([1, 0, 0])
    np_out, _ = oracle.obb_sat(a, b)
    n = np_out[:3].copy()
    p = np.zeros(3, np.float32)
    oracle.lib().or_contact_point_f32(a.ctypes.data, b.ctypes.data, n.ctypes.data, p.ctypes.data)
    assert abs(p[0] - 0.5) < 1e-6 and abs(p[1]) < 1e-6 and abs(p[2]) < 1e-6


def test_gpu_sat_rotated_edge_overlap():
    np_out, feat = oracle.obb_sat(box([0, 0, 0]), box([0.8, 0, 0], yaw(math.pi / 4)))
    assert np_out[3] >= -1e-5 and not feat & (1 << 16)


def test_gpu_sat_axis_order_and_near_face_count():
    """Touching faces: A0 and B0 both within 1e-4 (near_face_axes counts face axes only)."""
    np_out, feat = oracle.obb_sat(box([0, 0, 0]), box([1.0, 0.2, 0.1]))
    assert feat & 0xFF == 0                    # first minimum (A0) wins ties against B0
    assert (feat >> 8) & 0xFF == 2


# ------------------------------------------------------------- Morton
def test_morton30_matches_lbvh_wgsl():
    # lbvh.wgsl:93-98: floor(c + 512) clamped to [0, 1023], x in bit 0
    assert oracle.morton30(-512.0, -512.0, -512.0) == 0
    assert oracle.morton30(-511.0, -512.0, -512.0) == 1
    assert oracle.morton30(-512.0, -511.0, -512.0) == 2
    assert oracle.morton30(-512.0, -512.0, -511.0) == 4
    assert oracle.morton30(600.0, 600.0, 600.0) == (1 << 30) - 1


def test_morton63_orders_along_each_axis():
    # frame of a scene whose centres span [-5, 5]^3: 2^21 - 1 cells over 10 m
    lo, scale = (-5.0, -5.0, -5.0), float(np.float32(2097151.0) / np.float32(10.0))
    assert oracle.morton63(-5.0, -5.0, -5.0, lo, scale) == 0
    assert oracle.morton63(5.0, 5.0, 5.0, lo, scale) == (1 << 63) - 1
    assert oracle.morton63(9.0, 9.0, 9.0, lo, scale) == (1 << 63) - 1     # clamped
    cell = 10.0 / 2097151.0
    a = oracle.morton63(0.0, 0.0, 0.0, lo, scale)
    assert oracle.morton63(2 * cell, 0.0, 0.0, lo, scale) > a
    assert oracle.morton63(0.0, 2 * cell, 0.0, lo, scale) > a
    assert oracle.morton63(0.0, 0.0, 2 * cell, lo, scale) > a


def test_morton39_is_13_bits_per_axis():
    # 2^13 - 1 cells over 10 m; the top corner fills all 39 bits
    lo, scale = (-5.0, -5.0, -5.0), float(np.float32(8191.0) / np.float32(10.0))
    assert oracle.morton39(-5.0, -5.0, -5.0, lo, scale) == 0
    assert oracle.morton39(5.0, 5.0, 5.0, lo, scale) == (1 << 39) - 1
    assert oracle.morton39(-4.0, 9.0, -5.0, lo, scale) >> 1 & 1 == 1       # y clamped high: bit 1 set
    cell = 10.0 / 8191.0
    assert oracle.morton39(-5.0 + 1.5 * cell, -5.0, -5.0, lo, scale) == 1   # one cell along x: bit 0
    assert oracle.morton39(-5.0, -5.0 + 1.5 * cell, -5.0, lo, scale) == 2
    assert oracle.morton39(-5.0, -5.0, -5.0 + 1.5 * cell, lo, scale) == 4
    # the same point's 39-bit key is its 48-bit key's cell at a coarser grid: both keep axis order
    assert oracle.morton39(1.0, 2.0, 3.0, lo, scale) < oracle.morton39(1.0, 2.0, 3.5, lo, scale)


def test_morton30a_is_10_bits_per_axis():
    lo, scale = (-5.0, -5.0, -5.0), float(np.float32(1023.0) / np.float32(10.0))
    assert oracle.morton30a(-5.0, -5.0, -5.0, lo, scale) == 0
    assert oracle.morton30a(5.0, 5.0, 5.0, lo, scale) == (1 << 30) - 1
    cell = 10.0 / 1023.0
    assert oracle.morton30a(-5.0 + 1.5 * cell, -5.0, -5.0, lo, scale) == 1
    assert oracle.morton30a(-5.0, -5.0, -5.0 + 1.5 * cell, lo, scale) == 4


def test_morton48_is_16_bits_per_axis():
    # 2^16 - 1 cells over 10 m; the top corner fills all 48 bits
    lo, scale = (-5.0, -5.0, -5.0), float(np.float32(65535.0) / np.float32(10.0))
    assert oracle.morton48(-5.0, -5.0, -5.0, lo, scale) == 0
    assert oracle.morton48(5.0, 5.0, 5.0, lo, scale) == (1 << 48) - 1
    assert oracle.morton48(-4.0, 9.0, -5.0, lo, scale) >> 1 & 1 == 1       # y clamped high: bit 1 set
    cell = 10.0 / 65535.0
    x1 = oracle.morton48(-5.0 + 1.5 * cell, -5.0, -5.0, lo, scale)
    assert x1 == 1                                                         # one cell along x: bit 0
    assert oracle.morton48(-5.0, -5.0 + 1.5 * cell, -5.0, lo, scale) == 2
    assert oracle.morton48(-5.0, -5.0, -5.0 + 1.5 * cell, lo, scale) == 4


# ---------------------------------------------- compile.rs mass rules
def test_hollow_cylinder_mass_and_inertia():
    """compile.rs:1010-1038 at the reference density of 500 kg/m^3."""
    m, center, inertia = scenes.cylinder_mass_properties(np.float32(1.0), np.float32(0.5), np.float32(2.0),
                                                         360.0, density=np.float32(500.0))
    outer, inner = 0.5, 0.25
    expected_mass = 500 * math.pi * (outer ** 2 - inner ** 2) * 2.0
    axial = expected_mass * (outer ** 2 + inner ** 2) * 0.5
    transverse = expected_mass * (3 * (outer ** 2 + inner ** 2) + 4) / 12
    assert abs(float(m) - expected_mass) < 1e-3
    assert np.allclose(center, 0, atol=1e-6)
    assert abs(float(inertia[0]) - transverse) < 1e-3
    assert abs(float(inertia[1]) - axial) < 1e-3
    assert abs(float(inertia[2]) - transverse) < 1e-3
    offset, _, half, _ = scenes.cylinder_segments(np.float32(1.0), np.float32(0.5), np.float32(2.0))
    assert offset.shape[0] == scenes.CYLINDER_COLLIDER_COUNT
    assert np.all(np.abs(half[..., 1] - 1.0) < 1e-6)
    assert np.all(np.linalg.norm(offset, axis=-1) >= inner - 1e-6)


def test_cylinder_sector_offset_mass_properties():
    """compile.rs:1041-1095 (90 degree sector)."""
    m, center, inertia = scenes.cylinder_mass_properties(np.float32(1.0), np.float32(0.5), np.float32(2.0),
                                                         90.0, density=np.float32(500.0))
    outer, inner, length, sweep = 0.5, 0.25, 2.0, math.pi / 2
    expected_mass = 500 * sweep * (outer ** 2 - inner ** 2) * length * 0.5
    cx = 4 * math.sin(sweep / 2) * (outer ** 3 - inner ** 3) / (3 * sweep * (outer ** 2 - inner ** 2))
    rs = outer ** 2 + inner ** 2
    rpar = rs * (sweep + math.sin(sweep)) / (4 * sweep)
    rperp = rs * (sweep - math.sin(sweep)) / (4 * sweep)
    assert abs(float(m) - expected_mass) < 1e-3
    assert abs(float(center[0]) - cx) < 1e-6
    assert abs(float(inertia[0]) - expected_mass * (length ** 2 / 12 + rperp)) < 1e-3
    assert abs(float(inertia[1]) - expected_mass * (rpar + rperp - cx * cx)) < 1e-3


def test_welded_compound_parallel_axis_inertia():
    """compile.rs:1117-1142: two welded 1 m cubes at x = 0 and x = 1."""
    mass, com, inertia = scenes.compound_mass_properties(
        [("cuboid", (0.0, 0.0, 0.0), IDENTITY, (1.0, 1.0, 1.0)),
         ("cuboid", (1.0, 0.0, 0.0), IDENTITY, (1.0, 1.0, 1.0))], density=np.float32(500.0))
    assert abs(mass - 1000.0) < 1e-3
    assert np.allclose(com, [0.5, 0, 0], atol=1e-6)
    assert abs(inertia[0, 0] - 166.66667) < 1e-3
    assert abs(inertia[1, 1] - 416.6667) < 1e-3
    assert abs(inertia[2, 2] - 416.6667) < 1e-3


# ---------------------------------------------------- golden fixtures
def test_golden_fixtures_against_oracle():
    data = json.load(open(GOLDEN))
    assert data["source"].startswith("jens-hj/mechanic")
    for case in data["sat_cases"]:
        a = box(case["a"]["center"], yaw(case["a"].get("yaw", 0.0)), np.full(3, case["a"]["half"], np.float32))
        b = box(case["b"]["center"], yaw(case["b"].get("yaw", 0.0)), np.full(3, case["b"]["half"], np.float32))
        np_out, feat = oracle.obb_sat(a, b)
        emitted = not (np_out[3] < -1e-5)
        assert emitted == case["overlap"], case["cite"]
        if "normal" in case:
            assert np.allclose(np_out[:3], case["normal"], atol=1e-6), case["cite"]
        if "penetration" in case:
            assert abs(float(np_out[3]) - case["penetration"]) < 1e-6, case["cite"]
    for case in data["mass_cases"]:
        if case["kind"] == "cylinder":
            m, c, i = scenes.cylinder_mass_properties(np.float32(case["outer_diameter"]),
                                                      np.float32(case["inner_diameter"]),
                                                      np.float32(case["length"]), case["sweep_degrees"],
                                                      density=np.float32(case["density"]))
            assert abs(float(m) - case["mass"]) < 1e-3, case["cite"]
    assert abi.ROW_SIZES["GpuContact"][1] == data["row_sizes"]["GpuContact"]
    for name, size in data["row_sizes"].items():
        assert abi.ROW_SIZES[name][1] == size, name


# ------------------------------------------- end-to-end behaviour (oracle)
def test_falling_cube_lands_on_ground_and_stays_above_it():
    """One 0.25 m cube dropped from 1 m settles near y = 0.125 (cf. device.rs:4224 car-drop settle test)."""
    scene = scenes.falling_cubes(1, seed=0)
    scene.transforms["position"][0, :3] = [0.0, 1.0, 0.0]
    scene.colliders["local_rotation"][0] = IDENTITY
    scene.velocities[:] = 0
    w = oracle.OracleWorld(scene)
    for tick in range(1, 241):
        w.step(tick)
    tr, vel = w.state()
    y = float(tr["position"][0, 1])
    assert 0.09 < y < 0.14, y
    # the relaxed-Jacobi contact (omega = 0.125, 8 iterations) leaves at most about one
    # tick of gravity, g * dt = 0.1635 m/s, in the resting cube's vertical velocity
    assert abs(float(vel["linear"][0, 1])) < 0.2
    assert int(w.diagnostics()["error_flags"]) == 0


def test_oracle_fp32_and_fp64_agree_on_one_tick():
    scene = scenes.falling_cubes(200, seed=3)
    a = oracle.OracleWorld(scene, precision=32)
    b = oracle.OracleWorld(scene, precision=64)
    a.step(1)
    b.step(1)
    assert a.pair_count == b.pair_count and a.contact_count == b.contact_count
    pa = a.state()[0]["position"][:, :3].astype(np.float64)
    pb = b.state_f64()[0][:, :3]
    assert np.max(np.abs(pa - pb)) < 1e-5
