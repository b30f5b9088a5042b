"""Autotuner candidate lists (CPU)."""
from openhurricane_b200 import autotune


def test_candidates_by_mechanism_size():
    small = autotune.candidates(9)
    assert (2, 64) in small and (4, 64) in small and (3, 64) in small and (6, 64) in small
    large = autotune.candidates(53)
    assert large == [(2, 64)]
