"""Host logic of the batched-path autotuner (no GPU): grid candidates and workload signatures."""
import numpy as np

from protomol3_b200 import autotune as AT
from protomol3_b200 import waterbox as W


def smooth(n):
    for p in (2, 3, 5):
        while n % p == 0:
            n //= p
    return n == 1


def test_grid_candidates_never_coarser_than_the_spacing():
    for edge in (14.4, 18.62, 25.1, 31.0, 39.1, 99.34):
        c = AT.grid_candidates(edge, spacing=1.0, headroom=0.15)
        assert c[0] == W.pme_grid_for(edge)
        assert all(smooth(n) for n in c)
        assert all(edge / n <= 1.0 for n in c)
        assert c == sorted(set(c)) and c[-1] <= c[0] * 1.15
    assert AT.grid_candidates(30.0, headroom=0.0) == [30]
    assert AT.grid_candidates(31.0, headroom=0.15) == [32, 36]


def test_signature_distinguishes_workloads():
    a = [W.water_box(100, seed=1), W.water_box(150, seed=2)]
    b = [W.water_box(100, seed=1), W.water_box(151, seed=2)]
    s = AT.Autotuner.signature
    assert s(a, 9.0, 7.5, 4, "mixed") == s(list(a), 9.0, 7.5, 4, "mixed")
    assert s(a, 9.0, 7.5, 4, "mixed") != s(b, 9.0, 7.5, 4, "mixed")
    assert s(a, 9.0, 7.5, 4, "mixed") != s(a, 10.0, 7.5, 4, "mixed")
    assert s(a, 9.0, 7.5, 4, "mixed") != s(a, 9.0, 7.5, 4, "fp64")
