"""Binomial (Revolve) checkpoint schedule of the gradient (host logic, no
GPU): the macro-steps the library's schedule advances equal the optimum of
Griewank's recursion, computed here by brute force, and the classic limits
hold (enough slots: every macro-step advanced once in the first sweep; no
slot: the quadratic count)."""
import functools

import pytest


def _brute(M, S):
    @functools.lru_cache(maxsize=None)
    def T(l, c):
        if l == 1:
            return 0
        if c == 0:
            return l * (l - 1) // 2
        return min(d + T(l - d, c - 1) + T(d, c) for d in range(1, l))

    return T(M, S)


@pytest.mark.parametrize("M", [1, 2, 3, 7, 16, 40, 75])
@pytest.mark.parametrize("S", [0, 1, 2, 3, 5])
def test_schedule_cost_is_optimal(M, S, gpu_free_lib):
    import ttifd

    assert ttifd.schedule_cost(M, S) == _brute(M, S)


def test_schedule_limits(gpu_free_lib):
    import ttifd

    for M in (5, 30, 300):
        assert ttifd.schedule_cost(M, M - 1) == M - 1        # every start stored in one sweep
        assert ttifd.schedule_cost(M, 0) == M * (M - 1) // 2  # restart from step 0 each time
    # Revolve's binomial law: with 30 slots 3000 macro-steps need 3 sweeps' worth of advances
    # at most (beta(30, 3) = C(33, 3) = 5456 >= 3000 > beta(30, 2) = 496)
    c = ttifd.schedule_cost(3000, 30)
    assert 2 * 3000 < c < 3 * 3000
