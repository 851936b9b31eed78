"""The plain form's branch-free division and square root (exact_arith.cuh)
against CUDA's IEEE operators, bit for bit, on 2^26 operand pairs per seed:
the whole valid range, the force loops' physical ranges and mantissa edge
cases (powers of two, all-ones mantissas, zero and negative dividends)."""
import pytest

from cosims_b200 import engine

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_branch_free_division_and_sqrt_are_ieee(seed):
    bad_div, bad_sqrt = engine.check_exact_arith(0, seed, 1 << 26)
    assert bad_div == 0 and bad_sqrt == 0, (bad_div, bad_sqrt)
