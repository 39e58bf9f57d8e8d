"""NIfTI volumes (io/nifti.hpp): the library's reader and writer against the
reference's gz_nifti.

Fixtures: tests/golden/nifti/ holds files of every datatype the reader takes (RGB as the
reference's packed colour, complex left at 0 like the reference's float read), both
byte orders, NIfTI-1 and -2, .nii / .nii.gz / .hdr+.img, sform and qform-only
geometry, orientations that need flips and each kind of axis swap, scl_slope /
scl_inter, a 4-D file and an MNI-space header; tests/golden/nifti.npz holds what the
reference's reader returns for each (made by tests/golden/make_golden.py --only nifti).

Bars: voxel values, dims, voxel sizes and srow rows bit-exact; the writer's files
byte-identical to the reference writer's."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

import tipl_b200 as tb

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def bits(a):
    a = np.asarray(a)
    return a.view({1: np.uint8, 2: np.uint16, 4: np.uint32, 8: np.uint64}[a.dtype.itemsize])


@pytest.fixture(scope="module")
def ng(golden):
    return golden("nifti")


def cases(g):
    return sorted(k[:-5] for k in g.files if k.endswith("_path"))


def path_of(g, name):
    return os.path.join(GOLDEN, str(g[name + "_path"]))


def oracle_load(orc, path, vol=0, cap=1 << 26):
    out = np.zeros(cap, np.float32)
    dim = np.zeros(3, np.int32)
    vs = np.zeros(3, np.float32)
    srow = np.zeros(12, np.float32)
    steps = np.zeros(8, np.int32)
    ns = C.c_int(0)
    p = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
    ok = orc.lib.orc_nifti_load(str(path).encode(), int(vol), p(out), C.c_longlong(cap), p(dim), p(vs), p(srow),
                                p(steps), C.byref(ns))
    assert ok, path
    x, y, z = (int(v) for v in dim)
    return out[:x * y * z].reshape(z, y, x).copy(), vs, srow, list(steps[:ns.value])


def test_oracle_matches_reference(orc, ng):
    for n in cases(ng):
        I, vs, srow, _ = oracle_load(orc, path_of(ng, n))
        assert I.shape == ng[n + "_I"].shape, n
        assert np.array_equal(bits(I), bits(ng[n + "_I"])), n
        assert np.array_equal(bits(vs), bits(ng[n + "_vs"])), n
        assert np.array_equal(bits(srow), bits(ng[n + "_srow"])), n


def test_header_geometry_matches_reference(orc, ng):
    """regb_nifti_info_read (host only): LPS dims, voxel size, srow, is_mni and the
    reorientation steps equal the reference's."""
    seen_steps = set()
    for n in cases(ng):
        info = tb.nifti_info(path_of(ng, n))
        z, y, x = ng[n + "_I"].shape
        assert info["dim"] == (x, y, z), n
        assert np.array_equal(bits(info["vs"]), bits(ng[n + "_vs"])), n
        assert np.array_equal(bits(info["srow"]), bits(ng[n + "_srow"])), n
        assert info["is_mni"] == bool(ng[n + "_mni"]), n
        _, _, _, steps = oracle_load(orc, path_of(ng, n))
        assert info["steps"] == steps, n
        seen_steps.update(steps)
    assert seen_steps == {0, 1, 2, 3, 4, 5}  # every flip and every swap is exercised
    four = tb.nifti_info(path_of(ng, "i16_4d"))
    assert four["nvolumes"] == 2


def test_reader_errors(tmp_path):
    with pytest.raises(tb.RegbError):
        tb.nifti_info(str(tmp_path / "missing.nii"))
    bad = tmp_path / "bad.nii"
    bad.write_bytes(b"\0" * 400)
    with pytest.raises(tb.RegbError):
        tb.nifti_info(str(bad))


@pytest.mark.parametrize("dtype", [np.uint8, np.float32])
@pytest.mark.parametrize("name", ["v.nii", "v.nii.gz"])
def test_writer_bytes_equal_reference(tmp_path, dtype, name):
    """regb_nifti_save writes the reference writer's file byte for byte (always gzip,
    as the reference's output stream is)."""
    sys.path.insert(0, os.path.dirname(HERE))
    import oracle

    if not os.path.exists(oracle.REF_SO):
        pytest.skip("reference build (oracle/_ref) not present")
    R = oracle.Reference()
    rng = np.random.default_rng(4)
    v = (rng.random((6, 8, 7)) * 200).astype(dtype)
    vs = np.array([1.5, 1.25, 2.0], np.float32)
    srow = np.array([-1.5, 0, 0, 40, 0, -1.25, 0, 30, 0, 0, 2, -20], np.float32)
    for mni in (False, True):
        R.nifti_save(str(tmp_path / ("ref_" + name)), v, vs, srow, mni)
        tb.nifti_save(str(tmp_path / ("our_" + name)), v, vs, srow, is_mni=mni)
        assert (tmp_path / ("ref_" + name)).read_bytes() == (tmp_path / ("our_" + name)).read_bytes()


def test_writer_round_trip_geometry(tmp_path, orc):
    """A uint16 volume (written with the int16 code, as the reference writes uint16)
    and an RAS-oriented float volume come back through the oracle's reader with the
    reference's reorientation."""
    rng = np.random.default_rng(5)
    v = rng.integers(0, 30000, (5, 6, 7)).astype(np.uint16)
    vs = np.array([1.0, 2.0, 3.0], np.float32)
    srow = np.array([-1, 0, 0, 1, 0, -2, 0, 2, 0, 0, 3, 3], np.float32)
    tb.nifti_save(str(tmp_path / "u16.nii"), v, vs, srow)
    I, vs2, srow2, steps = oracle_load(orc, tmp_path / "u16.nii")
    assert steps == [] and np.array_equal(I, v.astype(np.float32))
    assert np.array_equal(vs2, vs) and np.array_equal(srow2, srow)
    f = rng.random((5, 6, 7)).astype(np.float32)
    ras = np.array([1, 0, 0, -3, 0, 1, 0, -4, 0, 0, 1, 5], np.float32)
    tb.nifti_save(str(tmp_path / "ras.nii.gz"), f, (1, 1, 1), ras)
    I, _, srow2, steps = oracle_load(orc, tmp_path / "ras.nii.gz")
    assert steps == [0, 1] and np.array_equal(I, f[:, ::-1, ::-1])
    assert np.array_equal(srow2, np.array([-1, 0, 0, 3, 0, -1, 0, 1, 0, 0, 1, 5], np.float32))


# ----------------------------------------------------------------- device reads
@pytest.mark.gpu
@pytest.mark.parametrize("device", [False, True])
def test_load_matches_reference(ng, device):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    for n in cases(ng):
        I, info = tb.nifti_load(path_of(ng, n), device="cuda" if device else None)
        if device:
            torch.cuda.synchronize()
            I = I.cpu().numpy()
        assert np.array_equal(bits(I), bits(ng[n + "_I"])), n
        assert np.array_equal(bits(info["srow"]), bits(ng[n + "_srow"])), n


@pytest.mark.gpu
def test_load_second_volume(orc, ng):
    I1, _ = tb.nifti_load(path_of(ng, "i16_4d"), volume=1)
    ref, _, _, _ = oracle_load(orc, path_of(ng, "i16_4d"), vol=1)
    assert np.array_equal(bits(I1), bits(ref))
    with pytest.raises(tb.RegbError):
        tb.nifti_load(path_of(ng, "i16_4d"), volume=2)


@pytest.mark.gpu
def test_full_size_volume(orc, tmp_path):
    """182x218x182 int16 RAS file (flips x and y, scaled): the device read equals the
    oracle's read voxel for voxel."""
    sys.path.insert(0, GOLDEN)
    from make_golden import nifti_bytes

    rng = np.random.default_rng(6)
    v = rng.integers(-2000, 30000, (182, 218, 182)).astype(np.int16)
    ras = [1.0, 0, 0, -90.0, 0, 1.0, 0, -126.0, 0, 0, 1.0, -72.0]
    data, _ = nifti_bytes(v, 4, 16, srow=ras, slope=0.75, inter=10.0)
    import gzip

    path = tmp_path / "big.nii.gz"
    with gzip.GzipFile(path, "wb", mtime=0, compresslevel=1) as f:
        f.write(data)
    I, info = tb.nifti_load(str(path), device="cuda")
    ref, _, srow, steps = oracle_load(orc, path, cap=v.size)
    assert steps == [0, 1] and info["steps"] == [0, 1]
    assert np.array_equal(bits(I.cpu().numpy()), bits(ref))
    assert np.array_equal(bits(info["srow"]), bits(srow))


def test_reader_rejects_truncated_and_unsupported(tmp_path):
    """A file shorter than its header says, a zero bitpix (the reference's own error,
    io/nifti.hpp:1052-1057) and a converted datatype whose bitpix does not match its
    element size fail with an error before any device work (so this runs without a
    GPU)."""
    sys.path.insert(0, GOLDEN)
    from make_golden import nifti_bytes

    v = np.arange(5 * 6 * 7, dtype=np.int16).reshape(5, 6, 7)
    data, _ = nifti_bytes(v, 4, 16)
    short = tmp_path / "short.nii"
    short.write_bytes(data[:-10])
    assert tb.nifti_info(str(short))["dim"] == (7, 6, 5)  # the header itself is fine
    with pytest.raises(tb.RegbError):
        tb.nifti_load(str(short))
    for dt, bp in ((64, 0), (4, 8)):
        bad, _ = nifti_bytes(np.zeros((5, 6, 7), np.uint8), dt, bp)
        (tmp_path / "bad.nii").write_bytes(bad)
        with pytest.raises(tb.RegbError):
            tb.nifti_load(str(tmp_path / "bad.nii"))


def test_mm_reg_export_fields_equal_reference_writer(tmp_path):
    """regb_mm_reg_export_fields writes mm_reg::export_nonlinear's dis file (a 4-D float
    NIfTI of f2t's then t2f's x, y, z components, reg/mm_reg.hpp:418-441) byte for byte as
    the reference's writer writes the same 4-D image."""
    sys.path.insert(0, os.path.dirname(HERE))
    import oracle

    if not os.path.exists(oracle.REF_SO):
        pytest.skip("reference build (oracle/_ref) not present")
    R = oracle.Reference()
    rng = np.random.default_rng(9)
    f2t = rng.normal(0, 2, (5, 6, 7, 3)).astype(np.float32)
    t2f = rng.normal(0, 2, (5, 6, 7, 3)).astype(np.float32)
    vs = np.array([1.5, 1.25, 2.0], np.float32)
    srow = np.array([-1.5, 0, 0, 40, 0, -1.25, 0, 30, 0, 0, 2, -20], np.float32)
    buf = np.concatenate([np.moveaxis(f2t, -1, 0), np.moveaxis(t2f, -1, 0)])  # (6, z, y, x)
    assert R.nifti_save4(str(tmp_path / "ref_dis.nii.gz"), buf, vs, srow)
    tb.mm_reg_export_fields(str(tmp_path / "our_dis.nii.gz"), f2t, t2f, vs, srow)
    assert (tmp_path / "ref_dis.nii.gz").read_bytes() == (tmp_path / "our_dis.nii.gz").read_bytes()
