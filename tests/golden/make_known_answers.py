"""Writes tests/golden/known_answers.json: the reference's own known answers.

Each case carries the file:line of the reference test it restates.  When the
reference sources are present (this script is run where they are mounted),
every cited line is checked to contain the literal that the case encodes, so
the fixture cannot drift from the reference tests.  Usage:

    python tests/golden/make_known_answers.py [path/to/mechanic]
"""
import json
import math
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

SAT_CASES = [
    {"cite": "crates/mechanic-gpu/src/collision.rs:201", "literal": "Vec3::new(1.01, 0.0, 0.0)",
     "a": {"center": [0, 0, 0], "half": 0.5}, "b": {"center": [1.01, 0, 0], "half": 0.5}, "overlap": False},
    {"cite": "crates/mechanic-gpu/src/collision.rs:206", "literal": "Vec3::new(0.75, 0.0, 0.0)",
     "a": {"center": [0, 0, 0], "half": 0.5}, "b": {"center": [0.75, 0, 0], "half": 0.5}, "overlap": True,
     "normal": [1, 0, 0], "penetration": 0.25},
    {"cite": "crates/mechanic-gpu/src/collision.rs:214", "literal": "Vec3::new(1.0, 0.0, 0.0)",
     "a": {"center": [0, 0, 0], "half": 0.5}, "b": {"center": [1.0, 0, 0], "half": 0.5}, "overlap": True,
     "normal": [1, 0, 0], "penetration": 0.0},
    {"cite": "crates/mechanic-gpu/src/collision.rs:227", "literal": "Vec3::new(0.8, 0.0, 0.0)",
     "a": {"center": [0, 0, 0], "half": 0.5},
     "b": {"center": [0.8, 0, 0], "half": 0.5, "yaw": math.pi / 4}, "overlap": True},
]

MASS_CASES = [
    {"cite": "crates/mechanic-core/src/compile.rs:1013", "literal": "CylinderDimensions::new(1.0, 0.5, 2.0)",
     "kind": "cylinder", "outer_diameter": 1.0, "inner_diameter": 0.5, "length": 2.0, "sweep_degrees": 360.0,
     "density": 500.0, "mass": 500.0 * math.pi * (0.25 - 0.0625) * 2.0},
    {"cite": "crates/mechanic-core/src/compile.rs:1045", "literal": "with_sweep_angle_degrees(90)",
     "kind": "cylinder", "outer_diameter": 1.0, "inner_diameter": 0.5, "length": 2.0, "sweep_degrees": 90.0,
     "density": 500.0, "mass": 500.0 * (math.pi / 2) * (0.25 - 0.0625) * 2.0 * 0.5},
]

ROW_SIZES = {"GpuTickConfig": 64, "GpuDiagnostics": 32, "GpuTransform": 32, "GpuVelocity": 32, "GpuMass": 64,
             "GpuSpatialInertia": 64, "GpuCollider": 64, "GpuBearing": 80, "GpuPair": 8, "GpuContact": 64,
             "GpuPersistentManifold": 48, "GpuMechanismBody": 64, "GpuMechanismCoordinate": 8,
             "GpuMechanismDrive": 32, "GpuLinkState": 48, "GpuContractionNode": 16}
ROW_CITE = "crates/mechanic-gpu/src/abi.rs:298-315"


def verify(ref_root: str) -> None:
    for case in SAT_CASES + MASS_CASES:
        path, line = case["cite"].split(":")
        text = open(os.path.join(ref_root, path)).read().splitlines()
        assert case["literal"] in text[int(line) - 1], (case["cite"], text[int(line) - 1])
    abi_text = open(os.path.join(ref_root, "crates/mechanic-gpu/src/abi.rs")).read()
    for name, size in ROW_SIZES.items():
        assert f"size_of::<{name}>() == {size}" in abi_text, name


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MECHANIC_REFERENCE", "")
    if ref and os.path.isdir(ref):
        verify(ref)
        verified = True
    else:
        verified = False
    data = {"source": "jens-hj/mechanic test sources", "verified_against_sources": verified,
            "sat_cases": SAT_CASES, "mass_cases": MASS_CASES, "row_sizes": ROW_SIZES, "row_cite": ROW_CITE}
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
