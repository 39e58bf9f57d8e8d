"""GPU parity of the 32x32-bin MI variant (REGB_COST_MI32) through the C ABI.

The reference builds only a 256x256 joint histogram (reg/linear.hpp:84-85); the
32-bin form quantises both volumes to 0..31 with normalize_upper_lower2(v, 31.99)
and then follows the same steps.  tests/golden/mi32.npz pins it to the reference's
own code (its quantisation and its 256-bin MI on the quantised volumes).

Bars: joint counts bit-exact; the cost, a double sum of n*ln(n/(row*col)) reduced in
another order, within 1e-12 relative; a whole affine registration within 1e-5 of the
same search replayed on the CPU with the oracle's costs (tests/cpp/linear_cpu).
"""
import os
import subprocess

import numpy as np
import pytest

import tipl_b200 as tb
from tipl_b200 import phantom as ph

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module", autouse=True)
def _need_gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from tipl_b200 import build

    build.build()


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b))


@pytest.mark.parametrize("ci", range(3))
def test_mi32_golden(golden, ci):
    g = golden("mi32")
    f, m, Ts = g[f"c{ci}_fixed"], g[f"c{ci}_moving"], g[f"c{ci}_T"]
    cost, hist = tb.mi32_cost(f, m, Ts, return_hist=True)
    for k in range(len(Ts)):
        assert same(hist[k], g[f"c{ci}_hist"][k])
        assert cost[k] == pytest.approx(g[f"c{ci}_cost"][k], rel=1e-12)


@pytest.mark.parametrize("shape", [(64, 64, 64), (91, 109, 91), (5, 300, 7)])
def test_mi32_vs_oracle(orc, shape):
    rng = np.random.default_rng(21)
    t, mv, _ = ph.affine_pair(shape, rng=rng) if min(shape) > 8 else (
        rng.random(shape).astype(np.float32), rng.random(shape).astype(np.float32), None)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(mv)
    Ts = np.array([orc.affine_to_matrix(ph.random_affine(rng, rot_deg=6, trans_vox=3), shape, (1, 1, 1), shape,
                                        (1, 1, 1)) for _ in range(5)])
    cost, hist = tb.mi32_cost(f8, m8, Ts, return_hist=True)
    for k, T in enumerate(Ts):
        c, h = orc.mi32_cost(f8, m8, T, with_hist=True)
        assert same(hist[k], h)
        assert cost[k] == pytest.approx(c, rel=1e-12)


def test_mi32_full_size_properties(orc):
    """182x218x182 (the affine workload's grid): every voxel in one bin, counts equal to
    the oracle's, and a K-candidate batch equal to K single calls."""
    shape = (182, 218, 182)
    rng = np.random.default_rng(ph.seed_for(2, 5))
    t, mv, _ = ph.affine_pair(shape, rng=rng)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(mv)
    Ts = np.array([orc.affine_to_matrix(ph.random_affine(rng, rot_deg=4, trans_vox=2), shape, (1, 1, 1), shape,
                                        (1, 1, 1)) for _ in range(4)])
    cost, hist = tb.mi32_cost(f8, m8, Ts, return_hist=True)
    assert (hist.sum(axis=1) == f8.size).all()
    c0, h0 = orc.mi32_cost(f8, m8, Ts[0], with_hist=True)
    assert same(hist[0], h0)
    assert cost[0] == pytest.approx(c0, rel=1e-12)
    single = np.array([tb.mi32_cost(f8, m8, T[None])[0] for T in Ts])
    assert np.array_equal(single, cost)


def test_mi32_edge_cases(orc):
    """A constant volume (quantised to all 0), a transform that maps every voxel off
    the moving volume, and a one-voxel-thick slab."""
    rng = np.random.default_rng(8)
    f8 = (rng.random((20, 21, 22)) * 256).astype(np.uint8)
    zero = np.zeros((20, 21, 22), np.uint8)
    const = np.full((19, 20, 23), 77, np.uint8)
    I = np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32)
    far = I.copy()
    far[9:] = (500, -400, 300)
    for a, b in ((f8, zero), (zero, f8), (f8, const), (const, f8)):
        for T in (I, far):
            cost, hist = tb.mi32_cost(a, b, T[None], return_hist=True)
            c, h = orc.mi32_cost(a, b, T, with_hist=True)
            assert same(hist[0], h)
            assert cost[0] == pytest.approx(c, rel=1e-12)
    slab = (rng.random((1, 30, 40)) * 256).astype(np.uint8)
    cost, hist = tb.mi32_cost(slab, slab, I[None], return_hist=True)
    c, h = orc.mi32_cost(slab, slab, I, with_hist=True)
    assert same(hist[0], h) and cost[0] == pytest.approx(c, rel=1e-12)


def test_linear_mi32_matches_cpu_replay(golden, tmp_path):
    """tipl::reg::linear with the 32-bin MI on the masked pair: the device run and the
    same search replayed on the CPU with the oracle's costs agree."""
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "tests", "cpp"), "linear_cpu"])
    g = golden("mask_init")
    f8, m8 = g["lin_fixed"], g["lin_moving"]
    p = tb.reg.linear_param(cost_type=tb.reg.MI32)
    cost, arg, evals = tb.reg.linear(f8, (1, 1, 1), m8, (1, 1, 1), param=p)
    fp, mp, op = tmp_path / "f.u8", tmp_path / "m.u8", tmp_path / "o.bin"
    f8.tofile(fp)
    m8.tofile(mp)
    z, y, x = f8.shape
    z2, y2, x2 = m8.shape
    exe = os.path.join(ROOT, "tests", "cpp", "linear_cpu")
    subprocess.run([exe, str(x), str(y), str(z), str(fp), str(x2), str(y2), str(z2), str(mp), str(tb.reg.MI32), "0",
                    str(op)], check=True, capture_output=True, timeout=900)
    o = np.fromfile(op, np.uint8)
    c_cpu, a_cpu = o[:4].view(np.float32)[0], o[4:52].view(np.float32)
    assert cost == pytest.approx(float(c_cpu), rel=1e-5), (cost, c_cpu)
    assert np.allclose(arg, a_cpu, atol=1e-3), (arg, a_cpu)
    assert evals > 0


def test_engine_mixes_mi32_with_mi_jobs():
    """Serving: MI32 and 256-bin MI jobs submitted together run in the same batching
    loop (one launch per cost type per round); each result equals the plain call."""
    rng = np.random.default_rng(ph.seed_for(2, 40))
    tmpl = ph.normalize_to_u8(ph.class_phantom((40, 44, 36), rng))
    movs = []
    for s in [(40, 44, 36), (36, 40, 38), (44, 46, 40), (30, 50, 34)]:
        t2 = ph.class_phantom(s, rng)
        T = ph.affine_matrix_f32(ph.random_affine(rng, rot_deg=6, trans_vox=2), s, (1, 1, 1), s, (1, 1, 1))
        movs.append(ph.normalize_to_u8(ph.rician(ph.apply_matrix(t2, T, s), rng)))
    params = [tb.reg.linear_param(cost_type=tb.reg.MI32 if k % 2 == 0 else tb.reg.MI) for k in range(len(movs))]
    plain = [tb.reg.linear(tmpl, (1, 1, 1), m, (1, 1, 1), param=p) for m, p in zip(movs, params)]
    with tb.Engine(max_active=8) as eng:
        tid = eng.add_template(tmpl)
        ids = [eng.submit(m, template=tid, linear_param=p) for m, p in zip(movs, params)]
        res = [eng.wait(i) for i in ids]
        st = eng.stats()
    assert st["affine_tasks"] == sum(p[2] for p in plain)
    for r, (cost, arg, evals) in zip(res, plain):
        assert r["status"] == 0
        assert r["linear_cost"] == np.float32(cost) and cost != 0.0
        assert np.array_equal(r["arg"].view(np.uint32), arg.view(np.uint32))
        assert r["cost_evals"] == evals


def test_engine_rejects_unknown_cost_type():
    tmpl = np.zeros((8, 8, 8), np.uint8)
    with tb.Engine(max_active=1) as eng:
        with pytest.raises(tb.RegbError):
            eng.submit(tmpl, fixed=tmpl, linear_param=tb.reg.linear_param(cost_type=7))
