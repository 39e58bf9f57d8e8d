"""tipl::reg::linear over lists of image pairs (reg/linear.hpp:421-440, 517-525; the
mm_linear branch of reg/mm_reg.hpp:356-358) through regb_linear_multi.

Bars: two identical pairs give exactly the one-pair search (their summed cost / 4
equals the one-pair cost / 2 at every candidate, so every decision is the same: arg,
cost and evaluation count bit-exact); with two different pairs the reported cost is
(cost of pair 1 + cost of pair 2) / 4 at the returned parameters, by the oracle."""
import numpy as np
import pytest

import tipl_b200 as tb
from tipl_b200 import phantom as ph

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pairs():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(ph.seed_for(6, 7))
    t, m, _ = ph.affine_pair((40, 44, 36), rng=rng)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    f2 = np.where(f8 > 0, 255 - f8, 0).astype(np.uint8)
    m2 = np.where(m8 > 0, 255 - m8, 0).astype(np.uint8)
    return f8, m8, f2, m2


@pytest.mark.parametrize("cost_type", [tb.reg.MI, tb.reg.CORR])
def test_identical_pairs_equal_one_pair(pairs, cost_type):
    f8, m8, _, _ = pairs
    p = tb.reg.linear_param(cost_type=cost_type)
    c1, a1, e1 = tb.reg.linear(f8, (1, 1, 1), m8, (1, 1, 1), param=p)
    c2, a2, e2 = tb.reg.linear([f8, f8], (1, 1, 1), [m8, m8], (1, 1, 1), param=p)
    assert np.array_equal(a1, a2) and c1 == c2 and e1 == e2


def test_two_pairs_cost_is_the_pair_mean(pairs, orc):
    """Narrow bound (no mask start, no pyramid, L-BFGS from arg): the final cost is the
    optimum the search recorded at the returned parameters."""
    f8, m8, f2, m2 = pairs
    start = np.array([1.0, -1.0, 0.5, 0.02, -0.01, 0.03, 1.02, 0.98, 1.0, 0.01, 0, -0.01], np.float32)
    p = tb.reg.linear_param(bound=1)  # narrow
    cost, arg, evals = tb.reg.linear([f8, f2], (1, 1, 1), [m8, m2], (1, 1, 1), arg=start, param=p)
    assert evals > 1 and not np.array_equal(arg, start)
    T = orc.affine_to_matrix(arg, f8.shape, (1, 1, 1), m8.shape, (1, 1, 1))
    want = (0.0 + orc.mi_cost(f8, m8, T) + orc.mi_cost(f2, m2, T)) / np.float32(2 * 2.0)
    assert cost == pytest.approx(float(np.float32(want)), rel=1e-6)
    c_one, _, _ = tb.reg.linear(f8, (1, 1, 1), m8, (1, 1, 1), arg=start, param=p)
    assert cost != c_one


def test_rejects_bad_pairs(pairs):
    f8, m8, f2, _ = pairs
    with pytest.raises(tb.RegbError):
        tb.reg.linear([f8, f2[:-1]], (1, 1, 1), [m8, m8], (1, 1, 1))  # from volumes of different dims
    with pytest.raises(tb.RegbError):
        tb.reg.linear([f8] * 13, (1, 1, 1), [m8] * 13, (1, 1, 1))  # more than 12 pairs
