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
