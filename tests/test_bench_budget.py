"""bench.py's wall-clock budget (CPU): the surrogate leg's fixed size does not
grow with --steps, the driver's 20-step run keeps it inside the default
budget at the measured 37 s per flow step, and a slow step skips it."""
import importlib.util
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def _bench():
    spec = importlib.util.spec_from_file_location("bench", os.path.join(HERE, "..", "bench.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def test_surrogate_leg_estimate_and_budget():
    b = _bench()
    n, samples, epochs = 1048576, 524288, 150
    step = 37.2
    est = b.surrogate_leg_seconds(step, samples, n, epochs)
    # the measured leg took 61 s; the estimate errs on the safe side
    assert 61.0 < est < 200.0
    # the driver's run: 357 s up to the leg with 1 + 3 steps, then 21 more steps
    elapsed = 357.0 + 21 * step
    assert b.fits_budget(elapsed, est, 1500.0)
    # a flow step twice as slow leaves no room for it
    assert not b.fits_budget(357.0 + 21 * 2 * step, b.surrogate_leg_seconds(2 * step, samples, n, epochs),
                             1500.0)


def test_profile_and_bench_flags_parse():
    import subprocess
    import sys
    out = subprocess.run([sys.executable, os.path.join(HERE, "..", "bench.py"), "--help"],
                         capture_output=True, text=True, check=True).stdout
    for flag in ("--budget-s", "--graph", "--profile", "--kernel", "--impl"):
        assert flag in out
