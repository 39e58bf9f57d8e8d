"""Storage precision: uint16 / BF16 / float volumes quantised to uint8 on the device
for the affine stage (normalize_upper_lower2, numerical/numerical.hpp:909-927) and
widened exactly to float for the FP32 nonlinear stage; FP32 results against the FP64
restatement in the oracle.  Fixtures: tests/golden/precision.npz (the reference's own
normalize_upper_lower2, made by tests/golden/make_golden.py --only precision)."""
import numpy as np
import pytest

import tipl_b200 as tb
from tipl_b200 import phantom as ph


@pytest.fixture(scope="module")
def pg(golden):
    return golden("precision")


def test_oracle_normalize_matches_reference(orc, pg):
    assert np.array_equal(orc.normalize_to_u8(pg["f32"])[0], pg["q_f32"])
    assert np.array_equal(orc.normalize_to_u8(pg["u16"])[0], pg["q_u16"])
    assert np.array_equal(orc.normalize_to_u8(pg["neg"])[0], pg["q_neg"])
    assert np.array_equal(orc.normalize_to_u8(pg["f32"], 200.0)[0], pg["q_f32_200"])


def test_bf16_storage_round_trip():
    """to_bf16 rounds to nearest even (as torch's float->bfloat16); from_bf16 is exact."""
    import torch

    rng = np.random.default_rng(5)
    x = np.concatenate([rng.normal(0, 1000, 4096), rng.uniform(-1, 1, 4096), [0.0, -0.0, 1.0, 65504.0]]).astype(
        np.float32)
    b = tb.to_bf16(x)
    t = torch.from_numpy(x).to(torch.bfloat16).view(torch.int16).numpy().view(np.uint16)
    assert np.array_equal(np.asarray(b, np.uint16), t)
    back = tb.from_bf16(b)
    assert np.array_equal(back, torch.from_numpy(x).to(torch.bfloat16).to(torch.float32).numpy())


def test_fp64_cost_oracle_close_to_fp32(orc):
    rng = np.random.default_rng(ph.seed_for(4, 1))
    t, m, _ = ph.affine_pair((40, 44, 36), rng=rng)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    p = ph.random_affine(rng, rot_deg=5, trans_vox=2)
    T = orc.affine_to_matrix(p, f8.shape, (1, 1, 1), m8.shape, (1, 1, 1))
    T64 = orc.affine_to_matrix_f64(p.astype(np.float64), f8.shape, (1, 1, 1), m8.shape, (1, 1, 1))
    assert abs(orc.mi_cost(f8, m8, T) - orc.mi_cost_f64(f8, m8, T64)) <= 1e-3 * abs(orc.mi_cost(f8, m8, T))
    assert abs(orc.corr_cost(f8, m8, T) - orc.corr_cost_f64(f8, m8, T64)) <= 1e-3


@pytest.mark.gpu
def test_normalize_device_bit_exact(pg, orc):
    import torch

    for key, upper, want in (("f32", 255.999, "q_f32"), ("u16", 255.999, "q_u16"), ("neg", 255.999, "q_neg"),
                             ("f32", 200.0, "q_f32_200")):
        out, ok = tb.normalize_to_u8(pg[key], upper)
        assert ok and np.array_equal(out, pg[want]), key
    # device views, and BF16 storage (the reference's float path on the widened values)
    b = tb.to_bf16(pg["f32"])
    out, ok = tb.normalize_to_u8(b)
    assert ok and np.array_equal(out, orc.normalize_to_u8(tb.from_bf16(b))[0])
    dev = torch.from_numpy(pg["f32"]).cuda().to(torch.bfloat16)
    out, ok = tb.normalize_to_u8(dev)
    assert ok and np.array_equal(out.cpu().numpy(), orc.normalize_to_u8(dev.float().cpu().numpy())[0])
    # a constant volume: the reference returns without writing
    c = np.full((5, 6, 7), 3.0, np.float32)
    o = np.full(c.shape, 9, np.uint8)
    _, ok = tb.normalize_to_u8(c, out=o)
    assert not ok and np.all(o == 9)


@pytest.mark.gpu
def test_widen_exact():
    import torch

    rng = np.random.default_rng(2)
    u = rng.integers(0, 65536, (9, 10, 11)).astype(np.uint16)
    assert np.array_equal(tb.widen_to_f32(u), u.astype(np.float32))
    x = rng.normal(0, 100, (9, 10, 11)).astype(np.float32)
    b = tb.to_bf16(x)
    assert np.array_equal(tb.widen_to_f32(b), tb.from_bf16(b))
    d = torch.from_numpy(x).cuda().to(torch.bfloat16)
    assert torch.equal(tb.widen_to_f32(d), d.float())


@pytest.mark.gpu
def test_engine_u16_affine_equals_quantised_plain():
    """A uint16 job's affine stage is the plain registration of the device-quantised volumes."""
    rng = np.random.default_rng(ph.seed_for(4, 2))
    t, m, _ = ph.affine_pair((40, 44, 36), rng=rng)
    tu = np.round(t * (4095.0 / t.max())).astype(np.uint16)
    mu = np.round(m * (4095.0 / m.max())).astype(np.uint16)
    q_t, _ = tb.normalize_to_u8(tu)
    q_m, _ = tb.normalize_to_u8(mu)
    cost, arg, _ = tb.reg.linear(q_t, (1, 1, 1), q_m, (1, 1, 1))
    with tb.Engine() as eng:
        tid = eng.add_template(tu)
        r = eng.wait(eng.submit(mu, template=tid))
    assert r["status"] == 0
    assert r["linear_cost"] == np.float32(cost) and np.array_equal(r["arg"], arg)


@pytest.mark.gpu
def test_engine_bf16_cdm_equals_float_plain():
    """A BF16 job's CDM runs in FP32 on the widened volumes: the field equals the plain
    float CDM of the template and the affine-resampled (widened) subject."""
    rng = np.random.default_rng(ph.seed_for(4, 4))
    t, m, _ = ph.cdm_pair((32, 36, 30), rng=rng)
    tb16, mb16 = tb.to_bf16(t), tb.to_bf16(m)
    field = np.zeros(t.shape + (3,), np.float32)
    with tb.Engine() as eng:
        tid = eng.add_template(tb16)
        r = eng.wait(eng.submit(mb16, template=tid, cdm=True, field_out=field))
    assert r["status"] == 0 and r["cdm_ok"]
    tf, mf = tb.from_bf16(tb16), tb.from_bf16(mb16)
    T = tb.affine_to_matrix(r["arg"], t.shape, (1, 1, 1), m.shape, (1, 1, 1))
    Is = tb.resample(mf, t.shape, T)
    want, ok = tb.reg.cdm(tf, Is)
    assert ok and np.array_equal(field.view(np.uint32), want.view(np.uint32))


@pytest.mark.gpu
def test_cdm_fp32_against_fp64_oracle(orc):
    """uint16 storage, FP32 CDM on the device against the FP64 oracle on the same
    values: displacement-field RMS error well below a voxel (1e-6 measured on this
    32^3 pair; on larger pairs the FP32 and FP64 runs can take a different loop
    decision, which the precision report measures at full size)."""
    rng = np.random.default_rng(ph.seed_for(4, 3))
    t, m, _ = ph.cdm_pair((32, 32, 32), rng=rng)
    ut = np.round(t / t.max() * 4095).astype(np.uint16)
    um = np.round(m / m.max() * 4095).astype(np.uint16)
    d32, ok = tb.reg.cdm(tb.widen_to_f32(ut), tb.widen_to_f32(um))
    d64, ok64, _ = orc.cdm(ut.astype(np.float64), um.astype(np.float64))
    assert ok and ok64
    err = np.sqrt(((d32.astype(np.float64) - d64) ** 2).sum(-1).mean())
    assert err < 1e-4, err
