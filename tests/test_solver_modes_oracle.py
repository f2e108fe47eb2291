"""The oracle's contact solve to a residual (no reference counterpart).

The fixed-pass solve of collision.wgsl:752-906 is repeated until the
normal-row residual falls below a relative tolerance; these tests check the
oracle's version on the 1,000-cube scene: it converges to 1e-5 within the
pass cap, it reports the cap when the tolerance is unreachable, and it
leaves the fixed-pass form untouched when the tolerance is 0.
"""
import numpy as np

import oracle
from mechanic_b200 import abi, scenes


def _config(tol=0.0, cap=0):
    c = abi.MkConfig()
    c.collisions_enabled = 1
    c.mechanism_self_collisions = 1
    c.solver_iterations = 8
    c.contact_tolerance = tol
    c.contact_max_iterations = cap
    return c


def test_residual_mode_converges_to_tolerance():
    w = oracle.OracleWorld(scenes.falling_cubes(300, seed=1), _config(1e-5, 512))
    seen = 0
    for t in range(1, 41):
        w.step(t)
        st = w.solve_stats()
        if w.active_count:
            seen += 1
            assert st["converged"] == 1
            assert st["relative_residual"] <= 1e-5
            assert 2 <= st["iterations"] < 512
    assert seen > 10


def test_residual_mode_reports_the_cap():
    w = oracle.OracleWorld(scenes.falling_cubes(300, seed=1), _config(1e-12, 7))
    for t in range(1, 41):
        w.step(t)
        if w.active_count:
            st = w.solve_stats()
            assert st["iterations"] == 7 and st["converged"] == 0


def test_tolerance_zero_keeps_the_fixed_passes():
    a = oracle.OracleWorld(scenes.falling_cubes(300, seed=2), _config(0.0, 512))
    b = oracle.OracleWorld(scenes.falling_cubes(300, seed=2), _config())
    for t in range(1, 31):
        a.step(t)
        b.step(t)
    ta, va = a.state()
    tb, vb = b.state()
    assert ta.tobytes() == tb.tobytes() and va.tobytes() == vb.tobytes()
    assert a.solve_stats()["iterations"] == 0


def test_learned_candidate_with_exact_impulses_wins():
    """Predictions equal to the converged impulses of the same state must be chosen."""
    scene = scenes.falling_cubes(300, seed=4)
    ref = oracle.OracleWorld(scene, _config(1e-5, 512))
    learned = oracle.OracleWorld(scene, _config(1e-5, 512))
    for t in range(1, 26):
        ref.step(t)
        learned.step(t)
    st = ref.state()
    man = ref.manifold()
    # converge tick 26 on the reference world and feed its impulses as predictions
    probe = oracle.OracleWorld(scene, _config(1e-7, 2000))
    probe.set_state(*st)
    probe.set_manifold(man, 25)
    probe.step(26)
    lam = probe.contacts()["arm_a_impulse"][probe.active(), 3]
    learned.set_warm_predictions(lam)
    learned.step(26)
    ref.step(26)
    assert learned.solve_stats()["chosen"] == 1
    assert learned.solve_stats()["iterations"] < ref.solve_stats()["iterations"]
