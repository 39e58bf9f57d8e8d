"""Subject preprocessing of the mm_reg pipeline (reg/mm_reg.hpp:14-20,
subject_image_pre): the separable [1 2 1] Gaussian, the Otsu threshold and median,
normalize_otsu_median and the uint8 conversion.  Fixtures: tests/golden/preprocess.npz
(the reference's own code, made by tests/golden/make_golden.py --only preprocess)."""
import numpy as np
import pytest

CASES = range(4)


@pytest.fixture(scope="module")
def pp(golden):
    return golden("preprocess")


@pytest.mark.parametrize("k", CASES)
def test_oracle_matches_reference(orc, pp, k):
    t = pp[f"c{k}_in"]
    assert np.array_equal(orc.gaussian(t), pp[f"c{k}_gauss"])
    assert np.array_equal(orc.gaussian(t, 2), pp[f"c{k}_gauss2"])
    g = pp[f"c{k}_gauss"]
    assert np.float32(orc.otsu_threshold(g)) == pp[f"c{k}_otsu"]
    assert np.float32(orc.otsu_median(g)) == pp[f"c{k}_median"]
    assert np.array_equal(orc.subject_image_pre(t), pp[f"c{k}_pre"])


@pytest.mark.gpu
@pytest.mark.parametrize("k", CASES)
def test_device_bit_exact(pp, k):
    """The device path against the reference's own outputs: the Gaussian (1 and 2
    rounds) and the whole subject_image_pre, bit for bit."""
    import torch

    import tipl_b200 as tb

    t = pp[f"c{k}_in"]
    assert np.array_equal(tb.gaussian(t), pp[f"c{k}_gauss"])
    assert np.array_equal(tb.gaussian(t, 2), pp[f"c{k}_gauss2"])
    assert np.array_equal(tb.subject_image_pre(t), pp[f"c{k}_pre"])
    d = torch.from_numpy(t).cuda()
    assert np.array_equal(tb.subject_image_pre(d).cpu().numpy(), pp[f"c{k}_pre"])


@pytest.mark.gpu
def test_device_full_size_against_oracle(orc):
    """182x218x182 (the median takes the 256-chunk path over millions of values):
    device equals the oracle bit for bit; uint16 storage widened exactly first."""
    from tipl_b200 import phantom as ph

    import tipl_b200 as tb

    rng = np.random.default_rng(ph.seed_for(4, 12))
    t = ph.rician(ph.class_phantom((182, 218, 182), rng), rng)
    assert np.array_equal(tb.subject_image_pre(t), orc.subject_image_pre(t))
    u = np.round(np.clip(t, 0, 4095)).astype(np.uint16)
    assert np.array_equal(tb.subject_image_pre(u), orc.subject_image_pre(u.astype(np.float32)))
