"""Mapping steps of the mm_reg pipeline (reg/mm_reg.hpp:271-345): displacement_to_mapping,
inv_displacement_to_mapping, compose_mapping and correlation(_ygz).  Fixtures:
tests/golden/mapping.npz (the reference's own code, tests/golden/make_golden.py --only mapping)."""
import numpy as np
import pytest

CASES = range(3)


@pytest.fixture(scope="module")
def mp(golden):
    return golden("mapping")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("k", CASES)
def test_oracle_matches_reference(orc, mp, k):
    g = lambda n: mp[f"c{k}_{n}"]
    assert np.array_equal(bits(orc.displacement_to_mapping(g("dis"), g("T"))), bits(g("map")))
    assert np.array_equal(bits(orc.inv_displacement_to_mapping(g("dis"), g("T"), tuple(g("mshape")))), bits(g("inv")))
    assert np.array_equal(orc.compose_mapping(g("img"), g("map")), g("composed"))
    assert orc.correlation(g("x"), g("y")) == g("r")
    assert orc.correlation(g("x"), g("y"), True) == g("r_ygz")


@pytest.mark.gpu
@pytest.mark.parametrize("k", CASES)
def test_device_bit_exact(mp, k):
    import tipl_b200 as tb

    g = lambda n: mp[f"c{k}_{n}"]
    assert np.array_equal(bits(tb.displacement_to_mapping(g("dis"), g("T"))), bits(g("map")))
    assert np.array_equal(bits(tb.inv_displacement_to_mapping(g("dis"), g("T"), tuple(g("mshape")))), bits(g("inv")))
    assert np.array_equal(tb.compose_mapping(g("img"), g("map")), g("composed"))
    assert tb.correlation(g("x"), g("y")) == g("r")
    assert tb.correlation(g("x"), g("y"), masked=True) == g("r_ygz")
