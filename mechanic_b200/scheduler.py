"""Host-side fixed-step clock that drives dispatch_tick and the render hand-off.

Restates FixedStepScheduler (crates/mechanic-gpu/src/scheduler.rs:40-80):
elapsed nanoseconds times the tick rate accumulate in an integer phase with
denominator 10^9, every whole 10^9 is one due tick (no catch-up cap), and
the remainder is the interpolation fraction between the last complete tick
and the next one.  That fraction is the `alpha` GpuPhysics.interpolate_snapshot
takes.
"""
from __future__ import annotations

PHYSICS_TPS = 60                  # mechanic-gpu lib.rs
PHASE_DENOMINATOR = 1_000_000_000
U64_MAX = (1 << 64) - 1
U128_MAX = (1 << 128) - 1


class FixedStepScheduler:
    def __init__(self):
        self.phase = 0
        self.next_tick = 1

    def advance(self, elapsed_ns: int) -> range:
        """Adds elapsed time; returns every due tick index (scheduler.rs:56-67)."""
        self.phase = min(self.phase + min(int(elapsed_ns) * PHYSICS_TPS, U128_MAX), U128_MAX)
        due = self.phase // PHASE_DENOMINATOR
        self.phase %= PHASE_DENOMINATOR
        count = min(due, U64_MAX)
        first = self.next_tick
        self.next_tick = min(self.next_tick + count, U64_MAX)
        return range(first, first + count)

    def interpolation_alpha(self) -> float:
        """Fraction between the latest complete tick and the next (scheduler.rs:69-73)."""
        return min(self.phase, 0xFFFFFFFF) / 1_000_000_000.0
