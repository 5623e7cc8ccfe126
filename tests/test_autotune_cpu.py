"""The autotuner's search on the host, with a fake timer in place of CUDA events.

The knobs are set through the C ABI (host-only calls); the timer returns a cost per
setting, so the search can be checked without a GPU: a real win is kept, a win that
appears only in one noisy timing is rejected when the winner is re-timed against
the starting setting, and the search always leaves its answer applied."""
import pytest


@pytest.fixture(scope="module")
def autotune():
    from doubleeye_b200 import autotune, build
    build.build()
    return autotune


def fake_timer(autotune, cost, noise=None):
    """Time = cost(knobs); ``noise`` maps a setting to a one-off reading returned on
    its first timing only."""
    seen = set()

    def _time(run, reps, warmup):
        knobs = autotune.current()
        key = tuple(sorted(knobs.items()))
        if noise and key not in seen and key in noise:
            seen.add(key)
            return noise[key]
        seen.add(key)
        return cost(knobs)
    return _time


def restore(autotune):
    saved = autotune.current()
    return lambda: autotune.apply(saved)


def test_real_win_is_kept(autotune, monkeypatch):
    undo = restore(autotune)
    try:
        autotune.apply({"rows_ctas_per_sm": 32, "cols_kt": 0, "cols_pf": 0, "cols_cta": 0,
                        "solve_threads": 0, "batch_streams": 2, "cols_async": 1})
        cost = lambda k: 10.0 - (1.0 if k["cols_kt"] == 16 else 0.0) \
            - (0.5 if k["solve_threads"] == 512 else 0.0)
        monkeypatch.setattr(autotune, "_time", fake_timer(autotune, cost))
        best, ms = autotune.tune(lambda: None)
        assert best["cols_kt"] == 16 and best["solve_threads"] == 512
        assert ms == pytest.approx(8.5)
        assert autotune.current() == best
    finally:
        undo()


def test_one_off_fast_reading_is_rejected(autotune, monkeypatch):
    undo = restore(autotune)
    try:
        start = {"rows_ctas_per_sm": 32, "cols_kt": 0, "cols_pf": 0, "cols_cta": 0,
                 "solve_threads": 0, "batch_streams": 2, "cols_async": 1}
        autotune.apply(start)
        lucky = dict(start, cols_cta=128)
        noise = {tuple(sorted(lucky.items())): 9.0}        # 10% faster once, by chance
        monkeypatch.setattr(autotune, "_time", fake_timer(autotune, lambda k: 10.0, noise))
        best, ms = autotune.tune(lambda: None)
        assert best == start
        assert ms == pytest.approx(10.0)
        assert autotune.current() == start
    finally:
        undo()


def test_every_knob_value_is_settable(autotune):
    undo = restore(autotune)
    try:
        for k, values in autotune.KNOBS.items():
            for v in values:
                autotune.apply({k: v})
                assert autotune.current()[k] == v, (k, v)
    finally:
        undo()
