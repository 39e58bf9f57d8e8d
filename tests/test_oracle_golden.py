"""Pins the plain-C oracle to the reference: every golden fixture (made by
tests/golden/make_golden.py from the reference's own CPU build) must be reproduced
bit for bit.  When the reference build is present (oracle/_ref), a few fresh seeded
cases are also compared live."""
import os

import numpy as np
import pytest

import oracle


def bits(a):
    a = np.asarray(a)
    return a.view({1: np.uint8, 4: np.uint32, 8: np.uint64}[a.dtype.itemsize])


def same(a, b):
    return np.array_equal(bits(a), bits(b))


def test_transforms(orc, golden):
    g = golden("transforms")
    for p, s, T, Ti in zip(g["params"], g["shapes"], g["T"], g["Tinv"]):
        fs = (s[0], s[1], s[2])
        ts = (s[3], s[4], s[5])
        got = orc.affine_to_matrix(p[:12], fs, p[12:15], ts, p[15:18])
        assert same(got, T)
        assert same(orc.matrix_inverse(T), Ti)


def test_resample(orc, golden):
    g = golden("resample")
    shape = tuple(g["out_shape"])
    for T, o8, of in zip(g["T"], g["out8"], g["outf"]):
        assert same(orc.resample(g["src8"], shape, T), o8)
        assert same(orc.resample(g["srcf"], shape, T), of)


def test_affine_costs(orc, golden):
    g = golden("affine_costs")
    f, m = g["fixed"], g["moving"]
    assert same(orc.histogram(f), g["from_hist"])
    for T, h, mi, c, cs in zip(g["T"], g["hist"], g["mi"], g["corr"], g["corr_swap"]):
        hist = orc.mi_hist(f, m, T)
        assert same(hist, h)
        assert int(hist.sum()) == f.size
        assert orc.mi_cost(f, m, T) == pytest.approx(mi, rel=1e-12)
        assert orc.mi_cost_from_hist(h, g["from_hist"]) == pytest.approx(mi, rel=1e-12)
        assert orc.corr_cost(f, m, T) == c  # exact integer moments: bit-exact
        assert orc.corr_cost(m, f, T) == cs  # roles swapped, transform inverted


@pytest.mark.parametrize("ci", range(3))
def test_mi32_variant(orc, golden, ci):
    """32x32-bin MI: joint counts bit-exact and the cost equal to the reference's own
    steps (quantisation to 31.99, its 256-bin MI on the quantised volumes, times 64)."""
    g = golden("mi32")
    f, m = g[f"c{ci}_fixed"], g[f"c{ci}_moving"]
    for T, h, c in zip(g[f"c{ci}_T"], g[f"c{ci}_hist"], g[f"c{ci}_cost"]):
        cost, hist = orc.mi32_cost(f, m, T, with_hist=True)
        assert same(hist, h)
        assert int(hist.sum()) == f.size
        assert cost == c


def cdm_multi_case(g, ci):
    """Inputs and settings of case ci of the cdm_multi fixture (float cases take the
    stored uint8 values * 0.5 + 0.25, exact in float32)."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import CDM_MULTI_CASES, cdm_f32_of

    dt, _, nmod, gt, res = CDM_MULTI_CASES[ci]
    cv = (lambda v: v) if dt == "u8" else cdm_f32_of
    It = [cv(g[f"c{ci}_It{i}"]) for i in range(nmod)]
    Is = [cv(g[f"c{ci}_Is{i}"]) for i in range(nmod)]
    return It, Is, gt, res


def field_digest(d):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(d, np.float32).tobytes()).hexdigest()


@pytest.mark.parametrize("ci", range(6))
def test_cdm_multi_modality(orc, golden, ci):
    """cdm over modality lists (reg/cdm.hpp:419-435): the field's SHA-256 equals the
    reference's, and every passing case's field moves (at resolution 1 every level
    iterates)."""
    g = golden("cdm_multi")
    It, Is, gt, res = cdm_multi_case(g, ci)
    d, ok, _ = orc.cdm_multi(It, Is, resolution=res, gradient_types=gt)
    assert ok == bool(g[f"c{ci}_ok"])
    if ok:
        assert float(np.abs(d).max()) == pytest.approx(float(g[f"c{ci}_maxabs"]))
        assert float(g[f"c{ci}_maxabs"]) > 0.5
        assert field_digest(d) == str(g[f"c{ci}_sha256"])


@pytest.mark.parametrize("ci", range(4))
def test_cdm_passes(orc, golden, ci):
    g = golden("cdm_passes")
    c = {k.split("_", 1)[1]: g[k] for k in g.files if k.startswith(f"c{ci}_")}
    assert same(orc.compose(c["Is"], c["d"]), c["compose8"])
    assert same(orc.compose(c["Isf"], c["d"]), c["composef"])
    for gt in "rd":
        nd, cost = orc.cdm_gradient(c["Is"], c["It"], gt)
        assert same(nd, c[f"grad8_{gt}"]) and np.float32(cost) == c[f"cost8_{gt}"]
        nd, cost = orc.cdm_gradient(c["Isf"], c["Itf"], gt)
        assert same(nd, c[f"gradf_{gt}"]) and np.float32(cost) == c[f"costf_{gt}"]
    assert same(orc.cdm_poisson(c["d"]), c["poisson"])
    assert np.float32(orc.cdm_max_len(c["d"])) == c["maxlen"]
    assert same(orc.accumulate(c["cd"], c["d"]), c["accumulate"])
    assert same(orc.cdm_smooth(c["d"], 0.4), c["smooth"])
    assert same(orc.downsample(c["Is"]), c["down8"])
    assert same(orc.downsample(c["Isf"]), c["downf"])
    assert same(orc.upsample_field_x2(c["up_in"], c["Is"].shape), c["up"])


def test_cdm_end_to_end(orc, golden):
    g = golden("cdm_e2e")
    d8, ok8, _ = orc.cdm(g["It8"], g["Is8"])
    assert ok8 == bool(g["ok8"]) and same(d8, g["d8"])
    df, okf, _ = orc.cdm(g["Itf"], g["Isf"])
    assert okf == bool(g["okf"]) and same(df, g["df"])


def test_f64_oracle_close_to_f32(orc, golden):
    """The all-double restatement agrees with the FP32 one to FP32 accuracy."""
    g = golden("cdm_passes")
    d = g["c1_d"]
    p32 = orc.cdm_poisson(d)
    p64 = orc.cdm_poisson(d.astype(np.float64))
    assert np.abs(p32 - p64).max() <= 1e-5 * max(1.0, np.abs(p64).max())


@pytest.mark.skipif(not os.path.exists(oracle.REF_SO), reason="reference build not present")
def test_live_against_reference(orc):
    R = oracle.Reference()
    rng = np.random.default_rng(7)
    from tipl_b200 import phantom as ph

    t, m, _ = ph.cdm_pair((24, 22, 20), rng=rng)
    t8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    assert same(t8, R.normalize_to_u8(t))
    a, oka, _ = orc.cdm(t8, m8, min_dimension=8)
    b, okb = R.cdm(t8, m8, min_dimension=8)
    assert oka == okb and same(a, b)
    for k in range(3):
        p = ph.random_affine(rng, rot_deg=15, trans_vox=3)
        T = orc.affine_to_matrix(p, t8.shape, (1, 1, 1), m8.shape, (1, 1, 1))
        assert same(T, R.affine_to_matrix(p, t8.shape, (1, 1, 1), m8.shape, (1, 1, 1)))
        assert same(orc.mi_hist(t8, m8, T), R.mi_hist(t8, m8, T))
        assert orc.corr_cost(t8, m8, T) == R.corr_cost(t8, m8, T)


@pytest.mark.parametrize("name", ["full", "c1_blob", "c1_class", "c1_class_u8"])
def test_oracle_cdm_full_matches_reference(orc, golden, name):
    """The oracle's CDM driver against the reference's own cdm_common at the workloads'
    shapes (cdm_full fixture: the 182x218x182 uint8 pair at min_dimension 32, the 64^3
    blob pair of the plain CDM workload -- the zero field -- and a 64^3 class-phantom
    pair, float and uint8); inputs regenerated from their seeds and checked first."""
    import hashlib
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import CDM_FULL_CASES, cdm_full_inputs

    g = golden("cdm_full")
    gen, dt, kw = {c[0]: (c[1], c[2], c[3]) for c in CDM_FULL_CASES}[name]
    It, Is = cdm_full_inputs(gen, dt)
    dig = lambda a: hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()  # noqa: E731
    assert dig(It) == str(g[f"{name}_It_sha256"]) and dig(Is) == str(g[f"{name}_Is_sha256"])
    d, ok, _ = orc.cdm(It, Is, **kw)
    assert int(ok) == int(g[f"{name}_ok"])
    assert dig(np.ascontiguousarray(d, np.float32)) == str(g[f"{name}_sha256"])


def test_oracle_cdm2d_matches_reference(orc, golden):
    """The oracle's 2-D CDM (oracle_cdm2d.h) against the reference's own
    cdm_common<void, unsigned char, 2> on every cdm2d case: field digests bit for bit,
    ok, and the false return of a zero modality-0 template."""
    import hashlib
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import CDM2D_CASES

    g = golden("cdm2d")
    for k, (shape, res, md, gt, nmod, _) in enumerate(CDM2D_CASES):
        It = [g[f"c{k}_It{i}"] for i in range(nmod)]
        Is = [g[f"c{k}_Is{i}"] for i in range(nmod)]
        d, ok, _ = orc.cdm2d(It, Is, resolution=res, min_dimension=md, gradient_types=gt)
        assert int(ok) == int(g[f"c{k}_ok"]), k
        if ok:
            assert hashlib.sha256(d.tobytes()).hexdigest() == str(g[f"c{k}_sha256"]), k


def mi_from_terms(hist, from_hist):
    """The MI reduction's arithmetic (affine_kernels.cu, mi_reduce_kernel): each non-zero
    bin adds n*ln(n) - n*(ln(row) + ln(col)) in double, a block of 8 rows x 256 columns per
    partial sum, the 32 partials added in block order; the cost is -sum / 65536."""
    h = np.asarray(hist, np.int64).reshape(256, 256)
    col = h.sum(axis=0).astype(np.float64)
    row = np.asarray(from_hist, np.float64)
    lcol = np.where(col > 0, np.log(np.where(col > 0, col, 1.0)), 0.0)
    lrow = np.where(row > 0, np.log(np.where(row > 0, row, 1.0)), 0.0)
    n = h.astype(np.float64)
    nz = h > 0
    terms = np.where(nz, n * np.log(np.where(nz, n, 1.0)) - n * (lrow[:, None] + lcol[None, :]), 0.0)
    parts = [float(np.sum(terms[8 * b:8 * b + 8])) for b in range(32)]
    s = 0.0
    for p in parts:
        s += p
    return -(s / 65536.0)


def test_mi_term_form_within_tolerance(orc, golden):
    """The reduction forms each term as n ln n - n (ln row + ln col) instead of the
    reference's n ln(n / row / col): only rounding differs, and the cost stays within the
    1e-12 relative tolerance of the reference's own costs (fixtures) and of the oracle on a
    full-size 182x218x182 histogram."""
    from tipl_b200 import phantom as ph

    g = golden("affine_costs")
    for h, mi in zip(g["hist"], g["mi"]):
        assert mi_from_terms(h, g["from_hist"]) == pytest.approx(mi, rel=1e-12)
    rng = np.random.default_rng(ph.seed_for(2, 0))
    shape = (182, 218, 182)
    t, m, _ = ph.affine_pair(shape, rng=rng)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    T = np.array([1, 0.02, 0, -0.02, 1, 0, 0, 0, 1, 1.5, -2.0, 0.7], np.float32)
    h = orc.mi_hist(f8, m8, T)
    fh = orc.histogram(f8)
    assert mi_from_terms(h, fh) == pytest.approx(orc.mi_cost_from_hist(h, fh), rel=1e-12)
