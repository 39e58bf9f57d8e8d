"""Generate the golden fixtures in this folder from the reference's own CPU code.

Run where the reference tree is present (it builds oracle/_ref/libtipl_ref.so from
it):  python tests/golden/make_golden.py [--ref-root PATH]

Every fixture stores its seeded inputs together with the reference's outputs, so
the tests need neither the reference nor the phantom generator to replay them.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tipl_b200 import phantom as ph  # noqa: E402


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(f"{name}: {os.path.getsize(path)} bytes")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=oracle.ref_root_from_env(), required=oracle.ref_root_from_env() is None,
                    help="the reference source tree (default: $TIPL_REF_ROOT)")
    ap.add_argument("--only", default=None,
                    help="make one fixture group: core | mask_init | precision | preprocess | linear_runs"
                         " | mapping | mi32 | nifti | cdm_multi | cdm_full | cdm2d")
    args = ap.parse_args()
    oracle.build(args.ref_root, with_ref=True)
    R = oracle.Reference()
    R.set_threads(1)
    if args.only in (None, "core"):
        core(R)
    if args.only in (None, "mask_init"):
        mask_init(R)
    if args.only in (None, "precision"):
        precision(R)
    if args.only in (None, "preprocess"):
        preprocess(R)
    if args.only in (None, "linear_runs"):
        linear_runs(R)
    if args.only in (None, "mapping"):
        mapping(R)
    if args.only in (None, "mi32"):
        mi32(R)
    if args.only in (None, "nifti"):
        nifti(R)
    if args.only in (None, "cdm_multi"):
        cdm_multi(R)
    if args.only in (None, "cdm_full"):
        cdm_full(R)
    if args.only in (None, "cdm2d"):
        cdm2d(R)


NIFTI_DIR = os.path.join(HERE, "nifti")


def cdm_multi_inputs(shape, nmod, rng):
    """nmod uint8 template contrasts of one anatomy (a class phantom, its inverted
    contrast inside the head, a blob field masked to it) and the subject: every contrast
    warped by one smooth field (sigma 6, max 3 voxels) with Rician noise."""
    base = ph.class_phantom(shape, rng)
    mask = (base > 0).astype(np.float32)
    inv = np.where(base > 0, 4095.0 - base, 0.0).astype(np.float32)
    blobs = (ph.blob_volume(shape, rng, noise=0.0) * mask).astype(np.float32)
    It = [base, inv, blobs][:nmod]
    d = ph.smooth_field(shape, rng, 6.0, 3.0)
    Is = [ph.rician(ph.warp(t, d), rng) for t in It]
    return [ph.normalize_to_u8(t) for t in It], [ph.normalize_to_u8(t) for t in Is]


def cdm_f32_of(v):
    """The float inputs of the float cases: uint8 values * 0.5 + 0.25 (exact in float32)."""
    return v.astype(np.float32) * np.float32(0.5) + np.float32(0.25)


def field_digest(d):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(d, np.float32).tobytes()).hexdigest()


CDM_MULTI_CASES = [("u8", (36, 40, 34), 2, "", 1.0), ("u8", (30, 32, 28), 3, "rd", 1.0),
                   ("f32", (32, 34, 30), 2, "dr", 1.0), ("u8", (18, 18, 18), 2, "", 1.0),
                   ("u8", (36, 40, 34), 1, "", 1.0), ("f32", (36, 40, 34), 1, "d", 1.0)]


def cdm_multi(R):
    """cdm_common over modality lists (reg/cdm.hpp:419-435) through the reference's own
    CPU cdm at resolution 1 (every level iterates): (dtype, shape, modalities,
    gradient_type string, resolution).  Inputs are stored as uint8 (float cases use
    cdm_f32_of); each field as its SHA-256 and max |d|.  c3 has a modality-0 template
    of zeros, so its first partial cost sum is zero and the call returns false; c4 and
    c5 are one-modality lists (the plain cdm_common call) whose fields move."""
    rng = np.random.default_rng(ph.seed_for(3, 44))
    out = {}
    for k, (dt, shape, nmod, gt, res) in enumerate(CDM_MULTI_CASES):
        It, Is = cdm_multi_inputs(shape, nmod, rng)
        if k == 3:
            It[0] = np.zeros_like(It[0])
        cv = (lambda v: v) if dt == "u8" else cdm_f32_of
        d, ok = R.cdm_multi([cv(v) for v in It], [cv(v) for v in Is], resolution=res, gradient_types=gt)
        for i in range(nmod):
            out[f"c{k}_It{i}"], out[f"c{k}_Is{i}"] = It[i], Is[i]
        out[f"c{k}_ok"] = np.array(int(ok))
        out[f"c{k}_sha256"] = np.array(field_digest(d) if ok else "")
        out[f"c{k}_maxabs"] = np.array(float(np.abs(d).max()) if ok else 0.0)
    save("cdm_multi", **out)


def input_digest(v):
    import hashlib

    return hashlib.sha256(np.ascontiguousarray(v).tobytes()).hexdigest()


# (name, generator, dtype, cdm_param overrides): the inputs are regenerated from their
# seeds by the tests, which first check them against the stored input digests.
CDM_FULL_CASES = [("full", "workload", "u8", {"min_dimension": 32}),
                  ("c1_blob", "blob", "f32", {}),
                  ("c1_class", "class", "f32", {}),
                  ("c1_class_u8", "class", "u8", {})]


def cdm_full_inputs(gen, dt):
    """The inputs of a CDM_FULL_CASES entry: 'workload' is the 182x218x182 pair of the
    nonlinear workload, 'blob' the 64^3 float pair of the plain CDM workload (its blob
    generator), 'class' a 64^3 class-phantom pair; 'u8' cases are quantised with
    normalize_upper_lower2 (255.999)."""
    if gen == "workload":
        t, m = ph.cdm_workload_pair((182, 218, 182))
    elif gen == "blob":
        t, m, _ = ph.cdm_pair((64, 64, 64), seed=ph.seed_for(1, 0))
    else:
        t, m = ph.cdm_class_pair((64, 64, 64))
    if dt == "u8":
        return ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    return np.ascontiguousarray(t, np.float32), np.ascontiguousarray(m, np.float32)


def cdm_full(R):
    """The reference's own CPU cdm_common (one thread) at the workloads' shapes: the
    182x218x182 uint8 pair at min_dimension 32 (levels 23/46/91 iterate; the field moves),
    the 64^3 float blob pair of the plain CDM workload at the default cdm_param (the
    reference returns the zero field: it never improves on its first iteration there),
    and a 64^3 class-phantom pair at the default cdm_param, float and uint8 (the field
    moves).  Stored: input digests, the field's SHA-256, max |d|, ok."""
    out = {}
    for name, gen, dt, kw in CDM_FULL_CASES:
        It, Is = cdm_full_inputs(gen, dt)
        d, ok = R.cdm(It, Is, **kw)
        out[f"{name}_It_sha256"] = np.array(input_digest(It))
        out[f"{name}_Is_sha256"] = np.array(input_digest(Is))
        out[f"{name}_ok"] = np.array(int(ok))
        out[f"{name}_sha256"] = np.array(field_digest(d) if ok else "")
        out[f"{name}_maxabs"] = np.array(float(np.abs(d).max()) if ok else 0.0)
        print(name, ok, float(np.abs(d).max()), flush=True)
    save("cdm_full", **out)


# (shape (h, w), resolution, min_dimension, gradient types, modalities, variant)
CDM2D_CASES = [((64, 72), 2.0, 16, "", 1, ""), ((96, 80), 1.0, 16, "", 1, ""), ((33, 47), 1.0, 8, "d", 1, ""),
               ((64, 64), 1.0, 16, "rd", 2, ""), ((128, 120), 2.0, 16, "", 1, ""), ((256, 256), 2.0, 16, "", 1, ""),
               ((40, 2), 1.0, 1, "", 1, ""), ((1, 30), 1.0, 1, "", 1, ""), ((48, 40), 1.0, 16, "", 2, "zero0")]


def cdm2d_inputs(shape, nmod, rng):
    """2-D uint8 pairs: a slice of a class phantom and the same slice warped in-plane by
    a smooth 2-D field (the x, y components of a sigma-4 field, max 3 pixels) with
    Rician noise; the second modality is the inverted contrast inside the head."""
    from scipy import ndimage

    t = ph.class_phantom((3,) + tuple(shape), rng)[1]
    d = ph.smooth_field((3,) + tuple(shape), rng, 4.0, 3.0)[1]
    y, x = np.meshgrid(np.arange(shape[0], dtype=np.float32), np.arange(shape[1], dtype=np.float32), indexing="ij")
    m = ndimage.map_coordinates(t, np.stack([y + d[..., 1], x + d[..., 0]]), order=1, mode="constant")
    m = ph.rician(m.astype(np.float32), rng)
    It, Is = [ph.normalize_to_u8(t)], [ph.normalize_to_u8(m)]
    if nmod > 1:
        It.append(ph.normalize_to_u8(np.where(t > 0, 4095 - t, 0).astype(np.float32)))
        Is.append(ph.normalize_to_u8(np.where(m > 50, 4095 - m, 0).astype(np.float32)))
    return It, Is


def cdm2d(R):
    """cdm_common<void, unsigned char, 2> (reg/cdm.hpp:373-474, 534-558 at dimension 2;
    the reference's CPU branch, one thread) on 2-D uint8 pairs: default and full
    resolution, gradient types 'r' / 'd' / "rd", one and two modalities, odd shapes,
    1- and 2-pixel axes, and a zero modality-0 template (false).  Stored: the inputs,
    the field's SHA-256 and max |d|, ok."""
    rng = np.random.default_rng(ph.seed_for(7, 2))
    out = {}
    for k, (shape, res, md, gt, nmod, var) in enumerate(CDM2D_CASES):
        It, Is = cdm2d_inputs(shape, nmod, rng)
        if var == "zero0":
            It[0] = np.zeros_like(It[0])
        d, ok = R.cdm2d(It, Is, resolution=res, min_dimension=md, gradient_types=gt)
        for i in range(nmod):
            out[f"c{k}_It{i}"], out[f"c{k}_Is{i}"] = It[i], Is[i]
        out[f"c{k}_ok"] = np.array(int(ok))
        out[f"c{k}_sha256"] = np.array(field_digest(d) if ok else "")
        out[f"c{k}_maxabs"] = np.array(float(np.abs(d).max()) if ok else 0.0)
        print(k, shape, ok, float(np.abs(d).max()) if ok else None, flush=True)
    save("cdm2d", **out)


def nifti_bytes(data, datatype, bitpix, srow=None, pixdim=(1.0, 1.0, 1.0), qform=None, big=False, version=1,
                slope=1.0, inter=0.0, magic=None, extra_dims=(), sform_code=1):
    """A NIfTI-1 (348-byte) or NIfTI-2 (540-byte) header followed by the voxels, built
    field by field from the published layouts (header only when magic is 'ni1')."""
    import struct

    e = ">" if big else "<"
    z, y, x = data.shape[:3]  # an RGB array carries its 3 channels last
    dims = [3 + len(extra_dims), x, y, z] + list(extra_dims)
    dims += [1] * (8 - len(dims))
    pix = [1.0, *pixdim, 1.0, 1.0, 1.0, 1.0]
    sform, qform_code = (sform_code, 0) if qform is None else (0, 1)
    if qform is not None:
        pix[0] = qform.get("qfac", 1.0)
    q = qform or {}
    srow = srow if srow is not None else [pixdim[0], 0, 0, 0, 0, pixdim[1], 0, 0, 0, 0, pixdim[2], 0]
    vals = data.astype(data.dtype.newbyteorder(e), copy=False).tobytes()
    if version == 1:
        h = bytearray(352)
        struct.pack_into(e + "i", h, 0, 348)
        struct.pack_into(e + "8h", h, 40, *dims)
        struct.pack_into(e + "hh", h, 70, datatype, bitpix)
        struct.pack_into(e + "8f", h, 76, *pix)
        struct.pack_into(e + "fff", h, 108, 352.0, slope, inter)
        struct.pack_into(e + "hh", h, 252, qform_code, sform)
        struct.pack_into(e + "6f", h, 256, q.get("b", 0.0), q.get("c", 0.0), q.get("d", 0.0), q.get("x", 0.0),
                         q.get("y", 0.0), q.get("z", 0.0))
        struct.pack_into(e + "12f", h, 280, *srow)
        h[344:348] = (magic or b"n+1\0")
        if magic == b"ni1\0":
            return bytes(h[:348]), vals
        return bytes(h) + vals, None
    h = bytearray(544)
    struct.pack_into(e + "i", h, 0, 540)
    h[4:12] = b"n+2\0\r\n\x1a\n"
    struct.pack_into(e + "hh", h, 12, datatype, bitpix)
    struct.pack_into(e + "8q", h, 16, *dims)
    struct.pack_into(e + "8d", h, 104, *pix)
    struct.pack_into(e + "q", h, 168, 544)
    struct.pack_into(e + "dd", h, 176, slope, inter)
    struct.pack_into(e + "ii", h, 344, qform_code, sform)
    struct.pack_into(e + "6d", h, 352, q.get("b", 0.0), q.get("c", 0.0), q.get("d", 0.0), q.get("x", 0.0),
                     q.get("y", 0.0), q.get("z", 0.0))
    struct.pack_into(e + "12d", h, 400, *srow)
    return bytes(h) + vals, None


def nifti_cases():
    """(name, array (z, y, x), datatype, bitpix, keyword arguments of nifti_bytes)."""
    rng = np.random.default_rng(ph.seed_for(6, 1))
    sh = (5, 9, 7)
    lps = [-1.5, 0, 0, 40.0, 0, -1.25, 0, 30.0, 0, 0, 2.0, -20.0]  # already LPS: no steps
    ras = [1.5, 0, 0, -40.0, 0, 1.25, 0, -30.0, 0, 0, 2.0, -20.0]   # flips x and y
    swap_xy = [0, 1.25, 0, -10.0, 1.5, 0, 0, -20.0, 0, 0, 2.0, 5.0]
    swap_xz = [0, 0, -2.0, 3.0, 0, -1.25, 0, 7.0, 1.5, 0, 0, -9.0]
    swap_yz = [-1.5, 0, 0, 1.0, 0, 0, 2.0, 2.0, 0, -1.25, 0, 3.0]
    oblique = [1.4, 0.3, 0.05, -12.0, -0.2, 1.2, 0.4, 8.0, 0.1, -0.35, 1.9, 2.0]
    return [
        ("u8_lps", (rng.random(sh) * 255).astype(np.uint8), 2, 8, dict(srow=lps, pixdim=(1.5, 1.25, 2.0))),
        ("i16_ras_scaled", rng.integers(-3000, 3000, sh).astype(np.int16), 4, 16,
         dict(srow=ras, pixdim=(1.5, 1.25, 2.0), slope=2.5, inter=-3.0)),
        ("f32_be_swapxy", rng.normal(0, 100, sh).astype(np.float32), 16, 32,
         dict(srow=swap_xy, pixdim=(1.25, 1.5, 2.0), big=True)),
        ("f64_nifti2_swapxz", rng.normal(0, 1e3, sh).astype(np.float64), 64, 64,
         dict(srow=swap_xz, pixdim=(2.0, 1.25, 1.5), version=2)),
        ("i32_qform", rng.integers(-2 ** 30, 2 ** 30, sh).astype(np.int32), 8, 32,
         dict(pixdim=(1.1, 1.2, 1.3), qform={"b": 0.0, "c": 0.0, "d": 0.70710677, "x": 5.0, "y": -6.0, "z": 7.0,
                                            "qfac": -1.0})),
        ("u16_pair_swapyz", rng.integers(0, 65535, sh).astype(np.uint16), 512, 16,
         dict(srow=swap_yz, pixdim=(1.5, 2.0, 1.25), magic=b"ni1\0")),
        ("i8_oblique", rng.integers(-128, 127, sh).astype(np.int8), 256, 8, dict(srow=oblique)),
        ("u32_be", rng.integers(0, 2 ** 32 - 1, sh, dtype=np.uint64).astype(np.uint32), 768, 32,
         dict(srow=ras, big=True)),
        ("i64_nifti2_be", rng.integers(-2 ** 60, 2 ** 60, sh, dtype=np.int64), 1024, 64,
         dict(srow=lps, version=2, big=True, slope=0.5)),
        ("u64", rng.integers(0, 2 ** 63, sh, dtype=np.uint64) * np.uint64(2), 1280, 64, dict(srow=ras, inter=1.0)),
        ("i16_4d", rng.integers(-500, 500, (2,) + sh).astype(np.int16).reshape(2 * sh[0], sh[1], sh[2]), 4, 16,
         dict(srow=ras, extra_dims=(2,))),
        ("f32_mni", rng.random(sh).astype(np.float32), 16, 32,
         dict(srow=[-1.0, 0, 0, 90.0, 0, -1.0, 0, 126.0, 0, 0, 1.0, -72.0], sform_code=4)),
        ("rgb_ras", rng.integers(0, 256, sh + (3,)).astype(np.uint8), 128, 24, dict(srow=ras)),
        ("complex64_be_scaled", (rng.normal(0, 10, sh) + 1j * rng.normal(0, 10, sh)).astype(np.complex64), 32, 64,
         dict(srow=lps, big=True, slope=2.0, inter=1.5)),
    ]


def write_nifti_case(name, arr, dt, bp, kw, gz):
    os.makedirs(NIFTI_DIR, exist_ok=True)
    import gzip

    head, img = nifti_bytes(arr, dt, bp, **kw)
    if kw.get("extra_dims"):
        # a NIfTI-1 4-D file: arr stacks the volumes along z; dim[3] is one volume's depth
        import struct

        e = ">" if kw.get("big") else "<"
        hb = bytearray(head)
        struct.pack_into(e + "h", hb, 46, arr.shape[0] // kw["extra_dims"][0])
        head = bytes(hb)
    if img is not None:
        path = os.path.join(NIFTI_DIR, name + ".hdr")
        open(path, "wb").write(head)
        open(os.path.join(NIFTI_DIR, name + ".img"), "wb").write(img)
        return path
    path = os.path.join(NIFTI_DIR, name + (".nii.gz" if gz else ".nii"))
    if gz:
        with gzip.GzipFile(path, "wb", mtime=0) as f:
            f.write(head)
    else:
        open(path, "wb").write(head)
    return path


def nifti(R):
    """NIfTI files of every datatype, byte order and header form, read by the reference's
    gz_nifti (>> I >> vs >> T >> is_mni); the files sit in tests/golden/nifti/."""
    out = {}
    for k, (name, arr, dt, bp, kw) in enumerate(nifti_cases()):
        path = write_nifti_case(name, arr, dt, bp, kw, gz=(k % 2 == 1))
        r = R.nifti_load(path)
        assert r is not None, name
        I, vs, srow, mni = r
        out[name + "_path"] = np.array(os.path.relpath(path, HERE))
        out[name + "_I"] = I
        out[name + "_vs"] = vs
        out[name + "_srow"] = srow
        out[name + "_mni"] = np.array(mni)
    save("nifti", **out)


def mi32(R):
    """The 32x32-bin MI variant through the reference's own steps: normalize_upper_lower2
    to 31.99 (the uint16 instantiation; uint8 values widen exactly), then the reference's
    256x256 get_mutual_info / get_mutual_info_mean on the quantised volumes.  With values
    0..31 every non-zero bin lies in the top-left 32x32 block, in the same order, so the
    32x32 histogram is that block and the 32-bin cost is the 256-bin cost times 64 (the
    mean is over 1024 instead of 65536 bins; both scalings are exact)."""
    rng = np.random.default_rng(ph.seed_for(2, 32))
    out = {}
    for k, (fs, ms) in enumerate([((30, 34, 28), (32, 30, 29)), ((23, 19, 27), (23, 19, 27)),
                                  ((1, 20, 24), (1, 22, 24))]):
        if fs[0] > 1:
            t = ph.class_phantom(fs, rng)
            m = ph.rician(ph.class_phantom(ms, rng), rng)
            f8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
        else:
            f8 = (rng.random(fs) * 256).astype(np.uint8)
            m8 = (rng.random(ms) * 200 + 40).astype(np.uint8)
        Ts = [np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32)]
        for _ in range(3):
            p = ph.random_affine(rng, rot_deg=8, trans_vox=3)
            Ts.append(R.affine_to_matrix(p, fs, (1, 1, 1), ms, (1, 1, 1)))
        qf = R.normalize_u16_to_u8(f8.astype(np.uint16), 32.0 - 0.01)
        qm = R.normalize_u16_to_u8(m8.astype(np.uint16), 32.0 - 0.01)
        out[f"c{k}_fixed"], out[f"c{k}_moving"] = f8, m8
        out[f"c{k}_T"] = np.array(Ts, np.float32)
        out[f"c{k}_hist"] = np.array([R.mi_hist(qf, qm, T).reshape(256, 256)[:32, :32].ravel() for T in Ts], np.int32)
        out[f"c{k}_cost"] = np.array([R.mi_cost(qf, qm, T) * 64.0 for T in Ts], np.float64)
    save("mi32", **out)


def mapping(R):
    """displacement_to_mapping, inv_displacement_to_mapping, compose_mapping, correlation(_ygz)."""
    rng = np.random.default_rng(ph.seed_for(5, 21))
    out = {}
    for k, (shp, mshp) in enumerate([((20, 24, 18), (22, 19, 25)), ((9, 7, 11), (9, 7, 11)), ((1, 12, 14), (3, 10, 15))]):
        dis = rng.normal(0, 1.5, shp + (3,)).astype(np.float32)
        dis.reshape(-1, 3)[::5] = 0
        p = ph.random_affine(rng, rot_deg=8, trans_vox=2)
        T = R.affine_to_matrix(p, shp, (1, 1, 1), mshp, (1, 1, 1))
        img = (rng.random(mshp) * 255).astype(np.uint8)
        m = R.displacement_to_mapping(dis, T)
        x = (rng.random(shp) * 255).astype(np.uint8)
        y = (rng.random(shp) * 255).astype(np.uint8)
        y.flat[::3] = 0
        out.update({f"c{k}_dis": dis, f"c{k}_T": T, f"c{k}_mshape": np.array(mshp), f"c{k}_img": img,
                    f"c{k}_map": m, f"c{k}_inv": R.inv_displacement_to_mapping(dis, T, mshp),
                    f"c{k}_composed": R.compose_mapping(img, m), f"c{k}_x": x, f"c{k}_y": y,
                    f"c{k}_r": np.float64(R.correlation(x, y)), f"c{k}_r_ygz": np.float64(R.correlation(x, y, True))})
    save("mapping", **out)


def linear_pairs():
    """Six seeded 30x34x28 phantom pairs: template, its exact affine resample (masked,
    even k) or that resample with Rician noise (no mask, odd k)."""
    R = oracle.Reference()
    out = []
    for seed in range(6):
        rng = np.random.default_rng(3000 + seed)
        shape = (30, 34, 28)
        f8 = ph.normalize_to_u8(ph.class_phantom(shape, rng))
        T = R.affine_to_matrix(ph.random_affine(rng, rot_deg=10, trans_vox=3), shape, (1, 1, 1), shape, (1, 1, 1))
        m8 = R.resample(f8, shape, T)
        if seed % 2:
            m8 = ph.normalize_to_u8(ph.rician(m8.astype(np.float32), rng))
        out.append((f8, m8))
    return out


def linear_runs(R):
    """The reference linear() (MI) on each pair, four runs with 1, 4, 8 and 16 threads:
    its line search and L-BFGS race in two threads, so the runs differ."""
    pairs = linear_pairs()
    costs = []
    for f8, m8 in pairs:
        row = []
        for th in (1, 4, 8, 16):
            R.set_threads(th)
            row.append(R.linear(f8, (1, 1, 1), m8, (1, 1, 1))[0])
        costs.append(row)
    R.set_threads(1)
    save("linear_runs", fixed=np.array([p[0] for p in pairs]), moving=np.array([p[1] for p in pairs]),
         costs=np.array(costs, np.float32))


def preprocess(R):
    """subject_image_pre of the mm_reg pipeline (gaussian, Otsu median, uint8) and its parts."""
    rng = np.random.default_rng(ph.seed_for(4, 11))
    out = {}
    # shapes: one under the median's 2048-value chunking threshold above Otsu, the rest over
    for k, shp in enumerate([(9, 11, 13), (30, 34, 28), (41, 37, 45), (1, 20, 24)]):
        t = ph.rician(ph.class_phantom(shp, rng), rng) if shp[0] > 1 else rng.random(shp).astype(np.float32) * 90
        g = R.gaussian(t)
        out[f"c{k}_in"] = t
        out[f"c{k}_gauss"] = g
        out[f"c{k}_gauss2"] = R.gaussian(t, 2)
        out[f"c{k}_otsu"] = np.float32(R.otsu_threshold(g))
        out[f"c{k}_median"] = np.float32(R.otsu_median(g))
        out[f"c{k}_pre"] = R.subject_image_pre(t)
    save("preprocess", **out)


def precision(R):
    """normalize_upper_lower2 of float32 and uint16 volumes (the quantisation before linear())."""
    rng = np.random.default_rng(ph.seed_for(4, 9))
    t = ph.class_phantom((26, 30, 22), rng)                       # float32 in [0, 4095]
    u = np.round(t + rng.normal(0, 20, t.shape)).clip(0, 4095).astype(np.uint16)
    neg = (t - 1000.0 + rng.normal(0, 5, t.shape)).astype(np.float32)  # negative values too
    save("precision", f32=t, u16=u, neg=neg, q_f32=R.normalize_to_u8(t), q_u16=R.normalize_u16_to_u8(u),
         q_neg=R.normalize_to_u8(neg), q_f32_200=R.normalize_to_u8(t, 200.0))


def mask_init(R):
    """has_mask, estimate_affine_param, to_affine_param and linear() with the mask start."""
    rng = np.random.default_rng(ph.seed_for(0, 9))
    vols = []
    for shp in [(30, 34, 28), (27, 31, 35)]:
        vols.append(ph.normalize_to_u8(ph.class_phantom(shp, rng)))              # zero background
    vols.append((rng.random((20, 22, 18)) * 200 + 20).astype(np.uint8))          # no zero voxel
    b = np.full((20, 22, 18), 7, np.uint8)
    b[:, :, 0] = 0
    b[:, :, -1] = 0
    vols.append(b)                                                                # box inside along x only
    vols.append(np.zeros((9, 10, 11), np.uint8))                                  # empty
    c = np.zeros((16, 18, 14), np.uint8)
    c[3:11, 5:9, 2:12] = 90
    vols.append(c)                                                                # axis-aligned box
    has = np.array([R.has_mask(v) for v in vols], np.int32)
    flat = np.concatenate([v.ravel() for v in vols])
    shapes = np.array([v.shape for v in vols], np.int32)
    pairs, vss, est = [], [], []
    for (i, j) in [(0, 1), (1, 0), (0, 0), (5, 0), (0, 5), (4, 0), (3, 1)]:
        for vs_pair in [((1, 1, 1), (1, 1, 1)), (tuple(rng.uniform(0.8, 2.0, 3)), tuple(rng.uniform(0.8, 2.0, 3)))]:
            svs, tvs = (np.array(v, np.float32) for v in vs_pair)
            pairs.append((i, j))
            vss.append(np.concatenate([svs, tvs]))
            est.append(R.estimate_affine_param(vols[i], svs, vols[j], tvs))
    Ts, tshapes, tvss, to_param = [], [], [], []
    for k in range(24):
        fs = tuple(int(v) for v in rng.integers(5, 60, 3))
        ts = tuple(int(v) for v in rng.integers(5, 60, 3))
        fvs = rng.uniform(0.7, 2.2, 3).astype(np.float32)
        tvs = rng.uniform(0.7, 2.2, 3).astype(np.float32)
        if k % 4 == 0:
            fvs[:] = 1.0
            tvs[:] = 1.0
        p = ph.random_affine(rng, rot_deg=25, trans_vox=8, vs=fvs)
        p[9:] = rng.uniform(-0.08, 0.08, 3)
        T = R.affine_to_matrix(p, fs, fvs, ts, tvs)
        Ts.append(T)
        tshapes.append(np.array(fs + ts, np.int32))
        tvss.append(np.concatenate([fvs, tvs]))
        to_param.append(R.matrix_to_affine_param(T, fs, fvs, ts, tvs))
    # linear() on a masked pair: the moving volume keeps a zero background
    t = ph.class_phantom((44, 52, 48), rng)
    T = R.affine_to_matrix(ph.random_affine(rng, rot_deg=8, trans_vox=3), t.shape, (1, 1, 1), t.shape, (1, 1, 1))
    f8 = ph.normalize_to_u8(t)
    m8 = R.resample(f8, t.shape, T)
    # the reference's line search and L-BFGS race in two threads: record several runs
    lin_costs = []
    for th in (1, 4, 8, 16):
        R.set_threads(th)
        c, a = R.linear(f8, (1, 1, 1), m8, (1, 1, 1))
        lin_costs.append(c)
        if th == 8:
            lin_cost, lin_arg = c, a
    # narrow bound: one thread, L-BFGS from the given start, reproducible
    starts = np.array([[0, 0, 0, 0, 0, 0, 1, 1, 1, 0, 0, 0],
                       [1, 0.5, -0.5, 0.05, 0.02, -0.03, 1.02, 0.97, 1.0, 0.01, 0, -0.01]], np.float32)
    narrow = [R.linear_bound(f8, (1, 1, 1), m8, (1, 1, 1), arg=st, bound=1, cost_type=ct)
              for st in starts for ct in (1, 0)]
    R.set_threads(1)
    save("mask_init", vols=flat, shapes=shapes, has=has, pairs=np.array(pairs, np.int32),
         vs=np.array(vss, np.float32), est=np.array(est, np.float32), T=np.array(Ts, np.float32),
         tshapes=np.array(tshapes), tvs=np.array(tvss, np.float32), to_param=np.array(to_param, np.float32),
         lin_fixed=f8, lin_moving=m8, lin_cost=np.float32(lin_cost), lin_arg=lin_arg,
         lin_costs=np.array(lin_costs, np.float32), narrow_start=starts,
         narrow_cost=np.array([n[0] for n in narrow], np.float32), narrow_arg=np.array([n[1] for n in narrow]))


def core(R):
    rng = np.random.default_rng(ph.seed_for(0, 1))

    # transformation_matrix(affine_param, ...) and its inverse
    params, shapes, T_out, Ti_out = [], [], [], []
    for k in range(24):
        fs = tuple(int(v) for v in rng.integers(5, 60, 3))
        ts = tuple(int(v) for v in rng.integers(5, 60, 3))
        fvs = rng.uniform(0.7, 2.2, 3).astype(np.float32)
        tvs = rng.uniform(0.7, 2.2, 3).astype(np.float32)
        if k % 4 == 0:
            tvs[:] = 1.0
        p = ph.random_affine(rng, rot_deg=25, trans_vox=8, vs=fvs)
        T = R.affine_to_matrix(p, fs, fvs, ts, tvs)
        params.append(np.concatenate([p, fvs, tvs]))
        shapes.append(np.array(fs + ts, np.int32))
        T_out.append(T)
        Ti_out.append(R.matrix_inverse(T))
    save("transforms", params=np.array(params, np.float32), shapes=np.array(shapes), T=np.array(T_out),
         Tinv=np.array(Ti_out))

    # resample (uint8 and float), including the integer-shift copy path
    src8 = (rng.random((23, 19, 17)) * 256).astype(np.uint8)
    srcf = rng.random((23, 19, 17)).astype(np.float32)
    out_shape = (20, 21, 18)
    Ts = []
    for k in range(6):
        p = ph.random_affine(rng, rot_deg=20, trans_vox=4)
        Ts.append(R.affine_to_matrix(p, out_shape, (1, 1, 1), src8.shape, (1, 1, 1)))
    Ts.append(np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 2, -3, 1], np.float32))  # integer shift: copy path
    Ts.append(np.array([1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0], np.float32))   # identity
    Ts = np.array(Ts, np.float32)
    save("resample", src8=src8, srcf=srcf, out_shape=np.array(out_shape), T=Ts,
         out8=np.array([R.resample(src8, out_shape, T) for T in Ts]),
         outf=np.array([R.resample(srcf, out_shape, T) for T in Ts]))

    # MI joint histogram / MI cost / correlation cost on a small phantom pair
    tmpl, mov, _ = ph.affine_pair((30, 34, 28), rng=rng)
    f8 = ph.normalize_to_u8(tmpl)
    m8 = ph.normalize_to_u8(mov)
    m8b = m8[1:-2, 2:, :-3].copy()  # a moving volume of another shape
    Ts, mi, corr, corr_swap, hists = [], [], [], [], []
    for k in range(5):
        p = ph.random_affine(rng, rot_deg=8, trans_vox=3) if k else np.array([0, 0, 0, 0, 0, 0, 1, 1, 1, 0, 0, 0],
                                                                            np.float32)
        T = R.affine_to_matrix(p, f8.shape, (1, 1, 1), m8b.shape, (1, 1, 1))
        Ts.append(T)
        hists.append(R.mi_hist(f8, m8b, T))
        mi.append(R.mi_cost(f8, m8b, T))
        corr.append(R.corr_cost(f8, m8b, T))
        corr_swap.append(R.corr_cost(m8b, f8, T))
    save("affine_costs", fixed=f8, moving=m8b, T=np.array(Ts), hist=np.array(hists), mi=np.array(mi),
         corr=np.array(corr), corr_swap=np.array(corr_swap), from_hist=R.histogram(f8))

    # CDM passes on odd shapes (flat-index wrap, 1- and 2-voxel axes)
    cases = {}
    for ci, shp in enumerate([(17, 9, 5), (6, 11, 13), (2, 7, 9), (1, 8, 8)]):
        It = (rng.random(shp) * 256).astype(np.uint8)
        Is = (rng.random(shp) * 256).astype(np.uint8)
        It.flat[:: 7] = 0
        Itf = rng.random(shp).astype(np.float32)
        Isf = rng.random(shp).astype(np.float32)
        d = rng.normal(0, 1.5, shp + (3,)).astype(np.float32)
        d.reshape(-1, 3)[::4] = 0
        cd = rng.normal(0, 1.0, shp + (3,)).astype(np.float32)
        c = {"It": It, "Is": Is, "Itf": Itf, "Isf": Isf, "d": d, "cd": cd}
        c["compose8"] = R.compose(Is, d)
        c["composef"] = R.compose(Isf, d)
        for gt in "rd":
            c[f"grad8_{gt}"], c[f"cost8_{gt}"] = R.cdm_gradient(Is, It, gt)
            c[f"gradf_{gt}"], c[f"costf_{gt}"] = R.cdm_gradient(Isf, Itf, gt)
        c["poisson"] = R.cdm_poisson(d)
        c["maxlen"] = np.float32(R.cdm_max_len(d))
        c["accumulate"] = R.accumulate(cd, d)
        c["smooth"] = R.cdm_smooth(d, 0.4)
        c["down8"] = R.downsample(Is)
        c["downf"] = R.downsample(Isf)
        small = d[: (shp[0] + 1) // 2, : (shp[1] + 1) // 2, : (shp[2] + 1) // 2].copy()
        c["up_in"] = small
        c["up"] = R.upsample_field_x2(small, shp)
        for k, v in c.items():
            cases[f"c{ci}_{k}"] = np.asarray(v)
    save("cdm_passes", **cases)

    # CDM end to end (default parameters): uint8 and float, 32^3 blob pair
    t, m, _ = ph.cdm_pair((32, 32, 32), rng=rng)
    t8, m8 = ph.normalize_to_u8(t), ph.normalize_to_u8(m)
    d8, ok8 = R.cdm(t8, m8)
    df, okf = R.cdm(t, m)
    save("cdm_e2e", It8=t8, Is8=m8, d8=d8, ok8=np.array(ok8), Itf=t, Isf=m, df=df, okf=np.array(okf))


if __name__ == "__main__":
    main()
