"""cdm_common over lists of modality pairs (reg/cdm.hpp:373-474, 534-558) through
regb_cdm_multi: every iteration composes and differentiates each modality, sums the
gradients in modality order and averages the costs (reg/cdm.hpp:419-435).

Bars: the field bit-exact with the reference's own CPU cdm (its SHA-256 in the
cdm_multi fixture, pinned to the oracle by test_oracle_golden) on uint8 and float
lists of 1-3 modalities with mixed gradient types; the same REGB_FALSE where a
partial cost sum is zero."""
import numpy as np
import pytest

import tipl_b200 as tb
from test_oracle_golden import cdm_multi_case, field_digest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def g(golden):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return golden("cdm_multi")


@pytest.mark.parametrize("ci", range(6))
def test_lists_match_reference(g, ci):
    It, Is, gt, res = cdm_multi_case(g, ci)
    d, ok = tb.reg.cdm(It, Is, tb.reg.cdm_param(resolution=res), gradient_types=gt)
    assert ok == bool(g[f"c{ci}_ok"])
    if ok:
        assert field_digest(d) == str(g[f"c{ci}_sha256"]), float(np.abs(d).max())


def test_device_lists_and_single_volume_call(g):
    """Device-resident lists give the host lists' field; a one-element list is the
    single-volume call; the longer list is cut to the shorter one's length."""
    import torch

    It, Is, gt, res = cdm_multi_case(g, 4)
    p = tb.reg.cdm_param(resolution=res)
    d_host, ok = tb.reg.cdm(It, Is, p)
    assert ok and field_digest(d_host) == str(g["c4_sha256"])
    d_one, ok1 = tb.reg.cdm(It[0], Is[0], p)
    assert ok1 and np.array_equal(d_one, d_host)
    extra = [It[0], np.zeros_like(It[0])]
    d_cut, ok2 = tb.reg.cdm(extra, Is, p)  # Is has one entry: the zero template is dropped
    assert ok2 and np.array_equal(d_cut, d_host)
    It2, Is2, gt2, res2 = cdm_multi_case(g, 1)
    dev_t = [torch.from_numpy(a).cuda() for a in It2]
    dev_s = [torch.from_numpy(a).cuda() for a in Is2]
    d_dev, ok3 = tb.reg.cdm(dev_t, dev_s, tb.reg.cdm_param(resolution=res2), gradient_types=gt2)
    torch.cuda.synchronize()
    assert ok3 and field_digest(d_dev.cpu().numpy()) == str(g["c1_sha256"])


def test_rejects_bad_lists(g):
    It, Is, _, _ = cdm_multi_case(g, 0)
    with pytest.raises(tb.RegbError):
        tb.reg.cdm(It, [Is[0], Is[1][:-1]])  # shapes differ
    with pytest.raises(tb.RegbError):
        tb.reg.cdm(It, Is, gradient_types="rx")  # unknown gradient type
    with pytest.raises(tb.RegbError):
        tb.reg.cdm([It[0]] * 13, [Is[0]] * 13)  # more than 12 modality pairs
