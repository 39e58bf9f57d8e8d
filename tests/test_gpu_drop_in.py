"""The drop-in boundary end to end: the reference's own tipl::reg::cdm_common and
tipl::reg::linear (compiled with -DTIPL_USE_CUDA by the host compiler) take their GPU
branch through include/tipl_b200/tipl_gpu.hpp on libregb200.so.  The GPU branch's CDM
field must equal the reference CPU branch's bit for bit; the affine search, whose
reference optimiser runs its line search and L-BFGS in racing threads, must reach a
final cost no worse than the CPU branch's runs by more than 1%."""
import os
import subprocess

import numpy as np
import pytest

from tipl_b200 import phantom as ph

pytestmark = pytest.mark.gpu
BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cpp", "tipl_drop_in")


@pytest.fixture(scope="module")
def volumes(tmp_path_factory):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    # the binary is built by __graft_entry__.build() from the reference's headers and the
    # shim; a missing binary is a failure, not a skip, so the boundary check cannot vanish
    assert os.path.exists(BIN), ("tests/cpp/tipl_drop_in is missing: build it with __graft_entry__.build() "
                                 "(make -C tests/cpp REF_ROOT=<reference tree>)")
    d = tmp_path_factory.mktemp("dropin")
    rng = np.random.default_rng(ph.seed_for(6, 0))
    t, m, _ = ph.affine_pair((40, 44, 36), rng=rng)
    f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    f8.tofile(d / "f.u8")
    m8.tofile(d / "m.u8")
    return d, f8.shape


def run(d, shape, what, where):
    out = d / f"{what}_{where}.bin"
    z, y, x = shape
    r = subprocess.run([BIN, what, where, str(x), str(y), str(z), str(d / "f.u8"), str(d / "m.u8"), str(out)],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return np.fromfile(out, dtype=np.uint8)


def test_cdm_common_gpu_branch_equals_cpu_branch(volumes):
    d, shape = volumes
    g = run(d, shape, "cdm", "gpu")
    c = run(d, shape, "cdm", "cpu")
    assert g[:4].view(np.int32)[0] == 1 and c[:4].view(np.int32)[0] == 1
    assert np.array_equal(g, c)


@pytest.mark.parametrize("gtypes", ["", "dr"])
def test_cdm_common_two_modalities_gpu_branch_equals_cpu_branch(volumes, golden, gtypes):
    """cdm_common on two-modality lists (reg/cdm.hpp:419-435): the GPU branch passes
    both pairs through regb_cdm_multi and its field equals the CPU branch's bit for bit
    (inputs: the first case of the cdm_multi fixture, whose field moves)."""
    d, _ = volumes
    g = golden("cdm_multi")
    for i in range(2):
        g[f"c0_It{i}"].tofile(d / f"mm_f{i}.u8")
        g[f"c0_Is{i}"].tofile(d / f"mm_m{i}.u8")
    z, y, x = g["c0_It0"].shape
    res = {}
    for where in ("gpu", "cpu"):
        out = d / f"cdm2_{where}.bin"
        r = subprocess.run([BIN, "cdm2", where, str(x), str(y), str(z), str(d / "mm_f0.u8"), str(d / "mm_m0.u8"),
                            str(out), str(d / "mm_f1.u8"), str(d / "mm_m1.u8"), gtypes],
                           capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        res[where] = np.fromfile(out, dtype=np.uint8)
    assert res["gpu"][:4].view(np.int32)[0] == 1 and res["cpu"][:4].view(np.int32)[0] == 1
    assert np.abs(res["cpu"][4:].view(np.float32)).max() > 0.5  # the field moves
    assert np.array_equal(res["gpu"], res["cpu"])


def test_linear_gpu_branch_close_to_cpu_branch(volumes):
    """The CPU branch's final cost depends on how its line search and L-BFGS threads
    interleave (4.52-4.56 on this pair over runs on one machine; on 23 seeded pairs
    the spread between reference runs reached 12 %).  The GPU branch replays that race
    on a fixed virtual clock and lands in one of the same basins: its final cost must
    be within 2.5 % of the worst of three CPU runs (measured: +1.1 % on this pair)."""
    d, shape = volumes
    g = run(d, shape, "linear", "gpu").view(np.float32)
    c = [run(d, shape, "linear", "cpu").view(np.float32)[0] for _ in range(3)]
    assert g[0] <= max(c) * 1.025, (g[0], c)


def test_linear_two_pairs_gpu_branch_close_to_cpu_branch(volumes):
    """linear on two-pair lists (mm_reg's mm_linear, reg/linear.hpp:421-440): the GPU
    branch passes both pairs through regb_linear_run_multi; its final cost (the pairs'
    summed cost / 4) must be within 2.5 % of the worst of three CPU-branch runs, the same
    bar as the one-pair search.  Second pair: the inverted contrast inside the head."""
    d, shape = volumes
    f = np.fromfile(d / "f.u8", dtype=np.uint8)
    m = np.fromfile(d / "m.u8", dtype=np.uint8)
    np.where(f > 0, 255 - f, 0).astype(np.uint8).tofile(d / "f2.u8")
    np.where(m > 0, 255 - m, 0).astype(np.uint8).tofile(d / "m2.u8")
    z, y, x = shape

    def run2(where):
        out = d / f"linear2_{where}.bin"
        r = subprocess.run([BIN, "linear2", where, str(x), str(y), str(z), str(d / "f.u8"), str(d / "m.u8"), str(out),
                            str(d / "f2.u8"), str(d / "m2.u8")], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        return np.fromfile(out, dtype=np.float32)

    g = run2("gpu")
    c = [run2("cpu")[0] for _ in range(3)]
    assert np.isfinite(g).all()
    assert g[0] <= max(c) * 1.025, (g[0], c)


@pytest.mark.parametrize("k", [0, 2, 3, 5])
def test_cdm_common_2d_gpu_branch_equals_cpu_branch(volumes, golden, k):
    """cdm_common<void, unsigned char, 2> (the reference's cdm_cuda<tipl::out, unsigned
    char, 2> instantiation, reg/cdm_cu.hpp:12-17): its GPU branch runs through the
    shim's 2-D cdm_cuda on regb_cdm2d_multi and its field equals the CPU branch's bit
    for bit (cdm2d fixture cases: default parameters, a 'd' gradient on an odd shape,
    two modalities "rd", 256 x 256)."""
    import sys

    sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
    from make_golden import CDM2D_CASES

    d, _ = volumes
    g = golden("cdm2d")
    (h, w), res, md, gt, nmod, _ = CDM2D_CASES[k]
    for i in range(nmod):
        g[f"c{k}_It{i}"].tofile(d / f"f2d_{i}.u8")
        g[f"c{k}_Is{i}"].tofile(d / f"m2d_{i}.u8")
    res_out = {}
    for where in ("gpu", "cpu"):
        out = d / f"cdm2d_{where}.bin"
        args = [BIN, "cdm2d", where, str(w), str(h), "1", str(d / "f2d_0.u8"), str(d / "m2d_0.u8"), str(out), str(res),
                str(md), gt or "-"]
        if nmod == 2:
            args += [str(d / "f2d_1.u8"), str(d / "m2d_1.u8")]
        r = subprocess.run(args, capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        res_out[where] = np.fromfile(out, dtype=np.uint8)
    assert res_out["gpu"][:4].view(np.int32)[0] == 1 and res_out["cpu"][:4].view(np.int32)[0] == 1
    assert np.abs(res_out["cpu"][4:].view(np.float32)).max() > 0.5  # the field moves
    assert np.array_equal(res_out["gpu"], res_out["cpu"])
