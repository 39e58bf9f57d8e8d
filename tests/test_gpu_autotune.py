"""The launch-shape autotuner (regb_autotune): it picks one of its candidate block sizes
for each cost kernel, and the costs are bit-identical before and after it runs (the
block size only decides which block counts which voxels)."""
import numpy as np
import pytest

import tipl_b200 as tb
from tipl_b200 import phantom as ph

pytestmark = pytest.mark.gpu


def test_autotune_keeps_costs_identical():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(ph.seed_for(2, 77))
    shape = (60, 70, 50)
    t, mv, _ = ph.affine_pair(shape, rng=rng)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(mv)
    Ts = np.array([tb.affine_to_matrix(ph.random_affine(rng, rot_deg=5, trans_vox=2), shape, (1, 1, 1), shape,
                                       (1, 1, 1)) for _ in range(5)])

    def costs():
        return tb.mi_cost(f8, m8, Ts), tb.corr_cost(f8, m8, Ts), tb.mi32_cost(f8, m8, Ts)

    before = costs()
    got = tb.autotune()
    assert got["corr"] in (8192, 16384, 32768, 65536, 131072)
    assert got["mi"] in (16384, 32768, 49152, 60000, 65535)
    assert got["mi32"] in (8192, 16384, 32768, 60000, 131072)
    assert tb.tuning() == {k: got[k] for k in ("corr", "mi", "mi32")}
    after = costs()
    for b, a in zip(before, after):
        assert np.array_equal(np.asarray(b).view(np.uint64), np.asarray(a).view(np.uint64))


def test_autotune_buckets_cache_and_costs(tmp_path):
    """The per-bucket tuner: every bucket's choice is a candidate, costs on grids of
    different buckets are bit-identical before and after, and the table written to the
    cache file is read back (from_cache) unchanged by the next call."""
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(ph.seed_for(2, 78))
    cases = []
    for shape in ((40, 44, 36), (100, 110, 96)):  # buckets 0 and 1
        t, mv, _ = ph.affine_pair(shape, rng=rng)
        f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(mv)
        Ts = np.array([tb.affine_to_matrix(ph.random_affine(rng, rot_deg=5, trans_vox=2), shape, (1, 1, 1), shape,
                                           (1, 1, 1)) for _ in range(4)])
        cases.append((f8, m8, Ts))

    def costs():
        return [(tb.mi_cost(f, m, T), tb.corr_cost(f, m, T), tb.mi32_cost(f, m, T)) for f, m, T in cases]

    before = costs()
    path = tmp_path / "tune" / "autotune.txt"
    got = tb.autotune_buckets(str(path))
    assert not got["from_cache"] and path.exists()
    cand = {"corr": (8192, 16384, 32768, 65536, 131072), "mi": (16384, 32768, 49152, 60000, 65535),
            "mi32": (8192, 16384, 32768, 60000, 131072)}
    for b, row in got["table"].items():
        for k, v in row.items():
            assert v in cand[k], (b, k, v)
    assert tb.tuning_buckets() == got["table"]
    again = tb.autotune_buckets(str(path))
    assert again["from_cache"] and again["table"] == got["table"]
    after = costs()
    for bc, ac in zip(before, after):
        for b, a in zip(bc, ac):
            assert np.array_equal(np.asarray(b).view(np.uint64), np.asarray(a).view(np.uint64))
