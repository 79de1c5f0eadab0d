"""The autotuner's timing loop (no GPU): shapes take turns frame by frame, so a
scene whose frames cost more as it evolves does not favour the shapes timed first."""
from particles4all_b200.autotune import interleaved


class FakeLib:
    """Records the shape the tuner selects (p4a_tune_clear / p4a_tune_set)."""

    def __init__(self):
        self.variant = None
        self.sets = []

    def p4a_tune_clear(self, kernel):
        self.variant = None

    def p4a_tune_set(self, kernel, bound, variant):
        self.variant = variant
        self.sets.append((kernel, bound, variant))


def test_interleaved_is_not_biased_by_a_growing_frame_cost():
    L = FakeLib()
    frame = [0]
    base = {0: 1.00, 1: 0.97, 2: 1.10}  # shape 1 is the fastest

    def step():
        frame[0] += 1

    def profile(step_fn):
        step_fn()
        # every frame costs 5 % more than the one before; 8 launches per frame
        ms = base[L.variant] * (1.05 ** frame[0]) * 8
        return {"lambda": (ms, 8), "delta": (1.0, 8)}

    times = interleaved(step, profile, L, 4, "lambda", [0, 1, 2], rounds=6)
    assert min(range(3), key=times.__getitem__) == 1
    assert frame[0] == 18  # one frame per shape per round
    assert {v for _, _, v in L.sets} == {0, 1, 2} and all(b == 1 << 40 for _, b, _ in L.sets)
    # shapes timed one after another would have picked shape 0
    seq = [base[v] * sum(1.05 ** f for f in range(1 + 6 * v, 7 + 6 * v)) for v in range(3)]
    assert min(range(3), key=seq.__getitem__) == 0


def test_interleaved_ignores_frames_without_the_kernel():
    L = FakeLib()

    def profile(step_fn):
        return {} if L.variant == 1 else {"aniso": (2.0 * (L.variant + 1), 1)}

    times = interleaved(lambda: None, profile, L, 3, "aniso", [0, 1, 2], rounds=2)
    assert times[0] == 2.0 and times[2] == 6.0 and times[1] == float("inf")
    assert min(range(3), key=times.__getitem__) == 0
