"""ABI layout and library surface (no GPU needed).

Row sizes restate abi.rs:298-315 and the alignment test abi.rs:326-357; the
C header is compiled with gcc to check that its structs match the numpy and
ctypes mirrors byte for byte; the built library must export every function
the header declares.
"""
import ctypes
import os
import re
import subprocess
import sys

import numpy as np
import pytest

from mechanic_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mechanic_b200.h")


@pytest.mark.parametrize("name", sorted(abi.ROW_SIZES))
def test_row_sizes_match_reference(name):
    dtype, size = abi.ROW_SIZES[name]
    assert dtype.itemsize == size


def test_rows_are_sixteen_byte_multiples():
    """abi.rs:326-348: every GPU row except GpuPair/GpuMechanismCoordinate is a 16-byte multiple."""
    for name, (dtype, size) in abi.ROW_SIZES.items():
        if name in ("GpuPair", "GpuMechanismCoordinate"):
            assert size == 8
        else:
            assert size % 16 == 0, name


def test_passive_drive_never_clamps():
    """abi.rs:350-357."""
    row = abi.passive_drive_rows(1)[0]
    assert row["mode"] == abi.DRIVE_MODE_PASSIVE
    assert abs(row["max_acceleration"]) < np.finfo(np.float32).eps
    assert np.isneginf(row["min_angle"]) and np.isposinf(row["max_angle"])


def test_header_struct_sizes_with_gcc(tmp_path):
    names = list(abi.ROW_SIZES) + ["MkCreation", "MkConfig", "MkCapacities", "MkError", "MkSubmission",
                                   "MkKernelTimings", "MkTickReadback", "MkDeviceState", "MkHostState",
                                   "MkTuning", "MkWaitProbe", "MkPublishedState"]
    src = tmp_path / "sizes.c"
    body = "\n".join(f'    printf("{n} %zu\\n", sizeof({n}));' for n in names)
    src.write_text(f'#include <stdio.h>\n#include "{HEADER}"\nint main(void) {{\n{body}\n    return 0;\n}}\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    sizes = dict(line.split() for line in out.strip().splitlines())
    for name, (dtype, size) in abi.ROW_SIZES.items():
        assert int(sizes[name]) == size, name
    for name in ("MkCreation", "MkConfig", "MkCapacities", "MkError", "MkSubmission", "MkKernelTimings",
                 "MkTickReadback", "MkDeviceState", "MkHostState", "MkTuning", "MkWaitProbe", "MkPublishedState"):
        assert int(sizes[name]) == ctypes.sizeof(getattr(abi, name)), name


def _declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^MK_API\s+[\w\s\*]+?\b(mk_\w+)\(", text, re.M)))


def test_library_exports_every_declared_function():
    from mechanic_b200 import build, physics
    build.build()
    declared = _declared_functions()
    assert len(declared) >= 20
    out = subprocess.run(["nm", "-D", "--defined-only", physics.LIB_PATH], check=True, capture_output=True,
                         text=True).stdout
    exported = set(re.findall(r"\bT (mk_\w+)$", out, re.M))
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    assert sorted(physics.EXPORTS) == declared


def test_library_loads_without_gpu_and_reports_version():
    from mechanic_b200 import physics
    lib = physics.library()
    assert physics.version().startswith("mechanic_b200")
    # configuration defaults mirror GpuPhysicsConfig::default (device.rs:33-41)
    c = abi.MkConfig()
    lib.mk_config_default(ctypes.byref(c))
    assert (c.collisions_enabled, c.mechanism_self_collisions, c.solver_iterations) == (1, 1, 8)
    assert c.use_graph == 1 and c.morton_mode == abi.MORTON_39
    # the host-side default row (used without loading the library) is the same bytes
    assert bytes(abi.config_default()) == bytes(c)


def test_config_row_needs_no_library():
    """GpuPhysicsConfig.to_c() (used by the CPU oracle's callers) does not load libmechanic_b200."""
    code = ("import sys; sys.path.insert(0, %r)\n"
            "from mechanic_b200.physics import GpuPhysicsConfig\n"
            "from mechanic_b200 import physics\n"
            "c = GpuPhysicsConfig(solver_iterations=4).to_c()\n"
            "assert c.solver_iterations == 4 and physics._lib is None\n"
            "maps = open('/proc/self/maps').read()\n"
            "assert 'libmechanic_b200' not in maps, 'library mapped'\n") % ROOT
    subprocess.run([sys.executable, "-c", code], check=True)


def test_create_rejects_over_capacity_before_touching_a_device():
    """device.rs:405-422: capacity errors carry {required, capacity} and come first."""
    from mechanic_b200 import scenes
    from mechanic_b200.physics import BodyCapacity, ColliderCapacity, GpuPhysics
    scene = scenes.falling_cubes(40, seed=1)
    with pytest.raises(BodyCapacity) as e:
        GpuPhysics(scene, capacities={"max_bodies": 10})
    assert (e.value.required, e.value.capacity) == (40, 10)
    with pytest.raises(ColliderCapacity) as e:
        GpuPhysics(scene, capacities={"max_colliders": 39})
    assert (e.value.required, e.value.capacity) == (40, 39)
