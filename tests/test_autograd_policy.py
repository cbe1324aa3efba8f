"""The TRSM recompute policy of the autograd binding (CPU: host logic only)."""
from __future__ import annotations


def test_recompute_policy_threshold():
    from zynum_b200 import autograd as ag
    gib = 1 << 30
    assert not ag.recompute_policy(16 << 20, 40 * gib)          # 16 MiB against 40 GiB free: keep X
    assert ag.recompute_policy(12 * gib, 40 * gib)               # above a quarter of the free memory
    assert ag.recompute_policy(1 << 20, 2 << 20, fraction=0.25)  # tight memory
    assert not ag.recompute_policy(1 << 20, 8 << 20, fraction=0.25)
    old = ag.RECOMPUTE_FRACTION
    try:
        ag.RECOMPUTE_FRACTION = 0.0
        assert ag.recompute_policy(1, 1 << 40)                  # fraction 0: always recompute
    finally:
        ag.RECOMPUTE_FRACTION = old
