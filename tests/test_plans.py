"""Launch-plan table (bsofi_plan_get / _set / _clear): host logic, no GPU."""
import pytest

from bsofi_b200 import api


@pytest.fixture(autouse=True)
def _clear_plans():
    api.plan_clear()
    yield
    api.plan_clear()


def test_default_plan_follows_the_tuned_sizes():
    # 2n = 512 fills 128-wide tiles and 256 tiles per step: persistent 128x128.
    assert api.plan_get(256, 32) == (False, [0, 4, 32, 4])
    # Small N: one GEMM launch per BSOI step; BSTRI in groups of 2 rows.
    assert api.plan_get(144, 20) == (False, [1, 4, 32, 4])
    assert api.plan_get(64, 16) == (False, [1, 2, 32, 2])
    # 2n = 392: 64x64 tiles, persistent for mid-size N, per step for N >= 20k.
    assert api.plan_get(196, 40) == (False, [5, 4, 32, 4])
    assert api.plan_get(324, 80) == (False, [2, 4, 32, 0])
    # 2n a multiple of 160 (800 = 5 x 160, 480 = 3 x 160): persistent 128x160
    # TMA tiles once a step has 148 tiles; below that the 64x64 plans.
    assert api.plan_get(400, 64) == (False, [0, 4, 32, 0])
    assert api.plan_get(240, 40) == (False, [0, 4, 32, 4])
    assert api.plan_get(240, 8) == (False, [1, 2, 32, 2])


def test_set_get_clear_roundtrip():
    assert api.plan_set(100, 8, [3, 0, 48, 0]) == 0
    assert api.plan_get(100, 8) == (True, [3, 0, 48, 0])
    assert api.plan_get(100, 9)[0] is False
    api.plan_clear()
    assert api.plan_get(100, 8)[0] is False


def test_bstri_group_is_stored():
    assert api.plan_set(100, 8, [1, 2, 32, 4]) == 0
    assert api.plan_get(100, 8) == (True, [1, 2, 32, 4])


@pytest.mark.parametrize("plan", [[6, 2, 32, 0], [-1, 2, 32, 0], [0, 5, 32, 0], [0, 2, 0, 0],
                                  [0, 2, 32, 1], [0, 2, 32, 9], [0, 2, 32, -1]])
def test_invalid_plans_rejected(plan):
    assert api.plan_set(64, 4, plan) == -1
    assert api.plan_get(64, 4)[0] is False
