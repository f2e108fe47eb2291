"""FixedStepScheduler restated (scheduler.rs:82-106 tests)."""
from mechanic_b200.scheduler import FixedStepScheduler


def test_one_second_always_produces_exactly_sixty_ticks():
    s = FixedStepScheduler()
    ticks = s.advance(1_000_000_000)
    assert len(ticks) == 60
    assert list(ticks) == list(range(1, 61))


def test_render_sized_fragments_do_not_drop_or_duplicate_ticks():
    s = FixedStepScheduler()
    emitted = []
    for _ in range(144):
        emitted.extend(s.advance(6_944_444))
    emitted.extend(s.advance(64))
    assert emitted == list(range(1, 61))


def test_interpolation_alpha_is_the_phase_fraction():
    s = FixedStepScheduler()
    s.advance(8_333_333)             # half a 60 Hz tick
    assert list(s.advance(0)) == []
    assert abs(s.interpolation_alpha() - 0.49999998) < 1e-9
    assert list(s.advance(8_333_334)) == [1]
    assert s.interpolation_alpha() == 20 / 1e9   # 1,000,000,020 - 10^9 left in the phase
