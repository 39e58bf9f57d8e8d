"""tipl_b200 -- the TIPL registration hot path on B200 (sm_100a).

Python mirror of the reference's calls for this path, over the C ABI of
libregb200.so (include/regb200.h).  Names and argument meaning follow the
reference:

=============================  ===================================================
reference                      here
=============================  ===================================================
tipl::reg::linear              ``reg.linear(from_, from_vs, to, to_vs, arg, ...)``
tipl::reg::cdm_common          ``reg.cdm(It, Is, param)``
tipl::resample                 ``resample(src, out_shape, T)``
tipl::compose_displacement     ``compose_displacement(src, dis)``
tipl::accumulate_displacement  ``accumulate_displacement(dis, new_dis)``
mutual_information / corr      ``mi_cost`` / ``corr_cost`` (K transforms at once); ``mi32_cost``
                               the 32x32-bin MI variant
transformation_matrix(...)     ``affine_to_matrix(param, ...)``
gz_nifti >> I >> vs >> T       ``nifti_load(path)`` / ``nifti_info`` / ``nifti_save``
=============================  ===================================================

Arrays are numpy arrays shaped (z, y, x) (x-fastest memory, the reference's
layout) -- host memory, staged by the library -- or CUDA torch tensors of the same
shape, used in place on the device.  Displacement fields are (z, y, x, 3) float32
with components (dx, dy, dz).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import CdmParam, Field, LinearParam, RegbError, Volume  # noqa: F401

__all__ = ["affine_to_matrix", "affine_to_matrix_f64", "matrix_inverse", "resample", "mi_cost", "mi32_cost",
           "corr_cost", "nifti_info", "nifti_load", "nifti_save", "compose_displacement", "accumulate_displacement",
           "downsample", "upsample_field_x2", "cdm_gradient", "cdm_poisson", "cdm_max_length", "cdm_smooth", "reg",
           "Engine", "RegbError", "version", "autotune", "tuning", "autotune_buckets", "tuning_buckets", "mm_reg_export_fields"]


def version() -> str:
    return _lib.lib().regb_version().decode()


def _is_dev(a) -> bool:
    return hasattr(a, "is_cuda") and a.is_cuda


def _dims(shape):
    z, y, x = shape[:3]
    arr = (C.c_int * 3)(int(x), int(y), int(z))
    return arr


class BF16(np.ndarray):
    """A host volume stored as BF16: a uint16 array holding the upper 16 bits of each
    float32 value (make one with to_bf16).  Device volumes use torch.bfloat16."""

    def __new__(cls, bits):
        return np.ascontiguousarray(bits, dtype=np.uint16).view(cls)


def to_bf16(a) -> BF16:
    """float32 -> BF16 storage, rounding to nearest even."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = (u + 0x7FFF + ((u >> 16) & 1)) >> 16
    return BF16(r.astype(np.uint16))


def from_bf16(b) -> np.ndarray:
    """BF16 storage -> the float32 values it holds (exact)."""
    return (np.asarray(b, dtype=np.uint16).astype(np.uint32) << 16).view(np.float32)


def _dtype_code(a) -> int:
    if isinstance(a, BF16):
        return _lib.BF16
    name = str(a.dtype)
    if name in ("uint8", "torch.uint8"):
        return _lib.U8
    if name in ("float32", "torch.float32"):
        return _lib.F32
    if name in ("uint16", "torch.uint16"):
        return _lib.U16
    if name == "torch.bfloat16":
        return _lib.BF16
    raise TypeError(f"unsupported dtype {a.dtype}")


def _vol(a) -> Volume:
    if _is_dev(a):
        assert a.is_contiguous()
        return Volume(a.data_ptr(), _dims(a.shape), _dtype_code(a), _lib.DEVICE)
    assert a.flags["C_CONTIGUOUS"]
    return Volume(a.ctypes.data, _dims(a.shape), _dtype_code(a), _lib.HOST)


def _field(a) -> Field:
    if _is_dev(a):
        assert a.is_contiguous() and a.shape[-1] == 3
        return Field(a.data_ptr(), _dims(a.shape), _lib.DEVICE)
    assert a.flags["C_CONTIGUOUS"] and a.dtype == np.float32 and a.shape[-1] == 3
    return Field(a.ctypes.data, _dims(a.shape), _lib.HOST)


def _like(a, shape, dtype=None):
    if _is_dev(a):
        import torch

        return torch.zeros(tuple(shape), dtype=dtype or a.dtype, device=a.device)
    return np.zeros(tuple(shape), dtype=dtype or a.dtype)


def _host(a, dtype):
    if _is_dev(a):
        return a
    return np.ascontiguousarray(a, dtype=dtype)


def _fptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _stream(stream):
    if stream is None:
        return None
    return C.c_void_p(int(getattr(stream, "cuda_stream", stream)))


# ---------------------------------------------------------------- transforms
def affine_to_matrix(param, from_shape, from_vs, to_shape, to_vs) -> np.ndarray:
    """transformation_matrix(affine_param, from, from_vs, to, to_vs) as 12 floats."""
    p = np.ascontiguousarray(param, np.float32)
    T = np.zeros(12, np.float32)
    fd = np.array(list(_dims(from_shape)), np.int32)
    td = np.array(list(_dims(to_shape)), np.int32)
    _lib.check(_lib.lib().regb_affine_to_matrix(_fptr(p), _fptr(fd), _fptr(np.asarray(from_vs, np.float32)),
                                                _fptr(td), _fptr(np.asarray(to_vs, np.float32)), _fptr(T)))
    return T


def affine_to_matrix_f64(param, from_shape, from_vs, to_shape, to_vs) -> np.ndarray:
    p = np.ascontiguousarray(param, np.float64)
    T = np.zeros(12, np.float64)
    fd = np.array(list(_dims(from_shape)), np.int32)
    td = np.array(list(_dims(to_shape)), np.int32)
    _lib.check(_lib.lib().regb_affine_to_matrix_f64(_fptr(p), _fptr(fd), _fptr(np.asarray(from_vs, np.float64)),
                                                    _fptr(td), _fptr(np.asarray(to_vs, np.float64)), _fptr(T)))
    return T


def matrix_inverse(T) -> np.ndarray:
    M = np.ascontiguousarray(T, np.float32).copy()
    _lib.check(_lib.lib().regb_matrix_inverse(_fptr(M)), allow=(_lib.REGB_OK, _lib.REGB_FALSE))
    return M


def matrix_to_affine_param(T, from_shape, from_vs, to_shape, to_vs) -> np.ndarray:
    """transformation_matrix::to_affine_param: the 12 parameters of a from -> to matrix."""
    M = np.ascontiguousarray(T, np.float32)
    a = np.zeros(12, np.float32)
    fd = np.array(list(_dims(from_shape)), np.int32)
    td = np.array(list(_dims(to_shape)), np.int32)
    _lib.check(_lib.lib().regb_matrix_to_affine_param(_fptr(M), _fptr(fd), _fptr(np.asarray(from_vs, np.float32)),
                                                      _fptr(td), _fptr(np.asarray(to_vs, np.float32)), _fptr(a)))
    return a


def normalize_to_u8(img, upper=255.999, out=None, stream=None):
    """normalize_upper_lower2(img, out, upper) on the device: uint8 of (v - min) * upper / (max - min).
    Returns (out, ok); ok is False (out untouched) for a constant volume."""
    if out is None:
        if _is_dev(img):
            import torch

            out = torch.zeros(tuple(img.shape), dtype=torch.uint8, device=img.device)
        else:
            out = np.zeros(img.shape, np.uint8)
    st = _lib.check(_lib.lib().regb_normalize_to_u8(C.byref(_vol(img)), C.byref(_vol(out)), float(upper),
                                                    _stream(stream)), allow=(_lib.REGB_OK, _lib.REGB_FALSE))
    return out, st == _lib.REGB_OK


def widen_to_f32(img, out=None, stream=None):
    """Exact widening of a uint8 / uint16 / BF16 volume to float32."""
    if out is None:
        if _is_dev(img):
            import torch

            out = torch.zeros(tuple(img.shape), dtype=torch.float32, device=img.device)
        else:
            out = np.zeros(img.shape, np.float32)
    _lib.check(_lib.lib().regb_widen_to_f32(C.byref(_vol(img)), C.byref(_vol(out)), _stream(stream)))
    return out


def displacement_to_mapping(dis, T, stream=None):
    """displacement_to_mapping(dis, mapping, T): mapping(x) = T(x + dis(x))."""
    out = _like(dis, dis.shape)
    _lib.check(_lib.lib().regb_displacement_to_mapping(C.byref(_field(dis)), _fptr(np.ascontiguousarray(T, np.float32)),
                                                       C.byref(_field(out)), _stream(stream)))
    return out


def inv_displacement_to_mapping(inv_dis, T, map_shape, stream=None):
    """inv_displacement_to_mapping: over map_shape, p = T^-1(x), p + trilinear(inv_dis, p)."""
    out = _like(inv_dis, tuple(map_shape) + (3,))
    _lib.check(_lib.lib().regb_inv_displacement_to_mapping(C.byref(_field(inv_dis)),
                                                           _fptr(np.ascontiguousarray(T, np.float32)),
                                                           C.byref(_field(out)), _stream(stream)))
    return out


def compose_mapping(img, mapping, stream=None):
    """compose_mapping(from, mapping) of a uint8 volume."""
    out = _like(img, mapping.shape[:3])
    _lib.check(_lib.lib().regb_compose_mapping(C.byref(_vol(img)), C.byref(_field(mapping)), C.byref(_vol(out)),
                                               _stream(stream)))
    return out


def match_fov(It, T, moving_shape, stream=None):
    """mm_reg's It_match_fov: It with 0 where T(x) falls outside a volume of moving_shape."""
    out = _like(It, It.shape)
    md = (C.c_int * 3)(*[int(v) for v in (moving_shape[2], moving_shape[1], moving_shape[0])])
    _lib.check(_lib.lib().regb_match_fov(C.byref(_vol(It)), _fptr(np.ascontiguousarray(T, np.float32)), md,
                                         C.byref(_vol(out)), _stream(stream)))
    return out


def correlation(x, y, masked=False) -> float:
    """Pearson r of two uint8 volumes (exact integer moments); masked: over y > 0 only."""
    r = C.c_double(0.0)
    _lib.check(_lib.lib().regb_correlation(C.byref(_vol(x)), C.byref(_vol(y)), int(bool(masked)), C.byref(r)))
    return r.value


def gaussian(img, bandwidth=1, out=None, stream=None):
    """filter::gaussian of a float32 volume (separable [1 2 1], bandwidth rounds)."""
    if out is None:
        out = _like(img, img.shape)
    _lib.check(_lib.lib().regb_gaussian(C.byref(_vol(img)), C.byref(_vol(out)), int(bandwidth), _stream(stream)))
    return out


def subject_image_pre(img, out=None, stream=None):
    """reg::subject_image_pre: gaussian, Otsu-median normalisation to [0, 255.99], uint8."""
    if out is None:
        if _is_dev(img):
            import torch

            out = torch.zeros(tuple(img.shape), dtype=torch.uint8, device=img.device)
        else:
            out = np.zeros(img.shape, np.uint8)
    _lib.check(_lib.lib().regb_subject_image_pre(C.byref(_vol(img)), C.byref(_vol(out)), _stream(stream)))
    return out


def has_mask(img) -> bool:
    """tipl::has_mask of a uint8 volume (numpy or device tensor)."""
    out = C.c_int(0)
    _lib.check(_lib.lib().regb_has_mask(C.byref(_vol(img)), C.byref(out)))
    return bool(out.value)


def estimate_affine_param(source, source_vs, target, target_vs) -> np.ndarray:
    """tipl::estimate_affine_param: initial parameters from the masks' centroids and axes."""
    a = np.zeros(12, np.float32)
    _lib.check(_lib.lib().regb_estimate_affine_param(C.byref(_vol(source)), _fptr(np.asarray(source_vs, np.float32)),
                                                     C.byref(_vol(target)), _fptr(np.asarray(target_vs, np.float32)),
                                                     _fptr(a)), allow=(_lib.REGB_OK, _lib.REGB_FALSE))
    return a


# ---------------------------------------------------------------- resample / costs
def resample(src, out_shape, T, allow_shift_copy=True, out=None, stream=None):
    """tipl::resample<linear>(src, out_shape, T)."""
    out = _like(src, out_shape) if out is None else out
    Tm = np.ascontiguousarray(T, np.float32)
    _lib.check(_lib.lib().regb_resample(C.byref(_vol(src)), C.byref(_vol(out)), _fptr(Tm), int(allow_shift_copy),
                                        _stream(stream)))
    return out


def mi_cost(fixed, moving, Ts, return_hist=False, stream=None):
    """-MI of the 256x256 joint histogram for each of K transforms (reference MI functor)."""
    Tm = np.ascontiguousarray(Ts, np.float32).reshape(-1, 12)
    K = Tm.shape[0]
    cost = np.zeros(K, np.float64)
    hist = np.zeros((K, 65536), np.int32) if return_hist else None
    _lib.check(_lib.lib().regb_mi_cost(C.byref(_vol(fixed)), C.byref(_vol(moving)), _fptr(Tm), K, _fptr(cost),
                                       _fptr(hist) if hist is not None else None, _stream(stream)))
    return (cost, hist) if return_hist else cost


def mi32_cost(fixed, moving, Ts, return_hist=False, stream=None):
    """-MI of the 32x32 joint histogram for each of K transforms, both volumes first
    quantised to 0..31 by normalize_upper_lower2(v, 31.99) (a variant of the reference
    MI functor, whose histogram is fixed at 256x256)."""
    Tm = np.ascontiguousarray(Ts, np.float32).reshape(-1, 12)
    K = Tm.shape[0]
    cost = np.zeros(K, np.float64)
    hist = np.zeros((K, 1024), np.int32) if return_hist else None
    _lib.check(_lib.lib().regb_mi32_cost(C.byref(_vol(fixed)), C.byref(_vol(moving)), _fptr(Tm), K, _fptr(cost),
                                         _fptr(hist) if hist is not None else None, _stream(stream)))
    return (cost, hist) if return_hist else cost


def corr_cost(fixed, moving, Ts, stream=None):
    """1 - r^2 for each of K transforms (reference correlation functor)."""
    Tm = np.ascontiguousarray(Ts, np.float32).reshape(-1, 12)
    K = Tm.shape[0]
    cost = np.zeros(K, np.float64)
    _lib.check(_lib.lib().regb_corr_cost(C.byref(_vol(fixed)), C.byref(_vol(moving)), _fptr(Tm), K, _fptr(cost),
                                         _stream(stream)))
    return cost


# ---------------------------------------------------------------- launch-shape autotuner
_COST_NAMES = ("corr", "mi", "mi32")


def autotune() -> dict:
    """Times the batched cost kernels on this device for a few block sizes and keeps the
    fastest (costs are identical under every choice); returns the choices (minimum voxels
    per block, by cost) and the seconds the tuning took."""
    tuned = np.zeros(3, np.int32)
    sec = C.c_double(0.0)
    _lib.check(_lib.lib().regb_autotune(_fptr(tuned), C.byref(sec)))
    return {**{k: int(v) for k, v in zip(_COST_NAMES, tuned)}, "seconds": sec.value}


def tuning() -> dict:
    """The block sizes in use for a 182x218x182 grid (defaults until autotune runs)."""
    tuned = np.zeros(3, np.int32)
    _lib.check(_lib.lib().regb_tuning_get(_fptr(tuned)))
    return {k: int(v) for k, v in zip(_COST_NAMES, tuned)}


TUNE_BUCKETS = ("64^3", "128^3", "182x218x182", "256^3")


def autotune_buckets(cache_path: str | None = "") -> dict:
    """The autotuner per size bucket of the fixed grid (regb_autotune_buckets): returns
    {bucket: {cost: minimum voxels per block}}, the seconds taken and whether the table
    came from the cache file (cache_path None = no file, "" = the default file)."""
    tuned = np.zeros(12, np.int32)
    sec = C.c_double(0.0)
    hit = C.c_int(0)
    path = None if cache_path is None else str(cache_path).encode()
    _lib.check(_lib.lib().regb_autotune_buckets(path, _fptr(tuned), C.byref(sec), C.byref(hit)))
    table = {b: {k: int(tuned[3 * i + c]) for c, k in enumerate(_COST_NAMES)} for i, b in enumerate(TUNE_BUCKETS)}
    return {"table": table, "seconds": sec.value, "from_cache": bool(hit.value)}


def tuning_buckets() -> dict:
    """The block sizes in use per size bucket."""
    tuned = np.zeros(12, np.int32)
    _lib.check(_lib.lib().regb_tuning_get_buckets(_fptr(tuned)))
    return {b: {k: int(tuned[3 * i + c]) for c, k in enumerate(_COST_NAMES)} for i, b in enumerate(TUNE_BUCKETS)}


# ---------------------------------------------------------------- NIfTI volumes (io/nifti.hpp)
def mm_reg_export_fields(path, f2t, t2f, vs, srow):
    """mm_reg::export_nonlinear's displacement file (reg/mm_reg.hpp:418-441): a 4-D float
    NIfTI (w, h, d, 6) of f2t's then t2f's x, y, z components, with the template's voxel
    size and srow rows."""
    _lib.check(_lib.lib().regb_mm_reg_export_fields(str(path).encode(), C.byref(_field(_host(f2t, np.float32))),
                                                    C.byref(_field(_host(t2f, np.float32))),
                                                    _fptr(np.asarray(vs, np.float32)),
                                                    _fptr(np.asarray(srow, np.float32))))


def nifti_info(path) -> dict:
    """The geometry tipl::io::gz_nifti reports for a .nii / .nii.gz / .hdr file after its
    LPS reorientation: dims (x, y, z), voxel size, srow rows, and the reorientation steps."""
    info = _lib.NiftiInfo()
    _lib.check(_lib.lib().regb_nifti_info_read(str(path).encode(), C.byref(info)))
    return _info_dict(info)


def _info_dict(info) -> dict:
    return {"dim": tuple(info.dim), "vs": np.array(info.vs, np.float32), "srow": np.array(info.srow, np.float32),
            "file_dim": tuple(info.file_dim), "datatype": info.datatype, "bitpix": info.bitpix,
            "nvolumes": info.nvolumes, "scl_slope": info.scl_slope, "scl_inter": info.scl_inter,
            "sform_code": info.sform_code, "is_mni": bool(info.is_mni), "big_endian": bool(info.big_endian),
            "nifti2": bool(info.nifti2), "steps": list(info.steps[:info.n_steps]),
            "descrip": info.descrip.decode(errors="replace")}


def nifti_load(path, volume=0, device=None, stream=None):
    """nii >> I >> vs >> T: volume `volume` as a float32 (z, y, x) array in LPS
    orientation -- a CUDA torch tensor when device is given, else a numpy array -- and
    the info dict (vs, srow, ...).  The conversion and reorientation run on the GPU."""
    info = nifti_info(path)
    x, y, z = info["dim"]
    if device is not None:
        import torch

        out = torch.zeros((z, y, x), dtype=torch.float32, device=device)
    else:
        out = np.zeros((z, y, x), np.float32)
    _lib.check(_lib.lib().regb_nifti_load(str(path).encode(), int(volume), C.byref(_vol(out)), None,
                                          _stream(stream)))
    return out, info


def nifti_save(path, vol, vs=(1.0, 1.0, 1.0), srow=None, is_mni=False, descrip=None):
    """nii << vs << T << I: writes a uint8 / uint16 / float32 (z, y, x) volume (host
    array or CUDA tensor) as NIfTI-1, gzip-compressed when path ends in .gz."""
    if srow is None:
        srow = np.array([vs[0], 0, 0, 0, 0, vs[1], 0, 0, 0, 0, vs[2], 0], np.float32)
    v = vol if _is_dev(vol) else np.ascontiguousarray(vol)
    _lib.check(_lib.lib().regb_nifti_save(str(path).encode(), C.byref(_vol(v)),
                                          _fptr(np.ascontiguousarray(vs, np.float32)),
                                          _fptr(np.ascontiguousarray(srow, np.float32)), int(bool(is_mni)),
                                          descrip.encode() if descrip else None))


# ---------------------------------------------------------------- displacement algebra / CDM passes
def compose_displacement(src, dis, stream=None):
    out = _like(src, src.shape)
    _lib.check(_lib.lib().regb_compose_displacement(C.byref(_vol(src)), C.byref(_field(_host(dis, np.float32))),
                                                    C.byref(_vol(out)), _stream(stream)))
    return out


def accumulate_displacement(dis, new_dis, stream=None):
    """Returns dis composed with new_dis (the reference updates new_dis in place)."""
    nd = new_dis.clone() if _is_dev(new_dis) else np.array(new_dis, np.float32, copy=True)
    _lib.check(_lib.lib().regb_accumulate_displacement(C.byref(_field(_host(dis, np.float32))), C.byref(_field(nd)),
                                                       _stream(stream)))
    return nd


def downsample(img, stream=None):
    z, y, x = img.shape
    out = _like(img, ((z + 1) // 2, (y + 1) // 2, (x + 1) // 2))
    _lib.check(_lib.lib().regb_downsample(C.byref(_vol(img)), C.byref(_vol(out)), _stream(stream)))
    return out


def upsample_field_x2(d, out_shape, stream=None):
    out = _like(d, tuple(out_shape) + (3,), dtype=None)
    _lib.check(_lib.lib().regb_upsample_field_x2(C.byref(_field(_host(d, np.float32))), C.byref(_field(out)),
                                                 _stream(stream)))
    return out


def cdm_gradient(Js, It, gradient_type="r", stream=None):
    nd = _like(Js, tuple(Js.shape) + (3,), dtype=_f32_like(Js))
    c = C.c_float(0)
    _lib.check(_lib.lib().regb_cdm_gradient(C.byref(_vol(Js)), C.byref(_vol(It)), C.byref(_field(nd)),
                                            ord(gradient_type), C.byref(c), _stream(stream)))
    return nd, float(c.value)


def _f32_like(a):
    if _is_dev(a):
        import torch

        return torch.float32
    return np.float32


def cdm_poisson(d, stream=None):
    nd = d.clone() if _is_dev(d) else np.array(d, np.float32, copy=True)
    _lib.check(_lib.lib().regb_cdm_poisson(C.byref(_field(nd)), _stream(stream)))
    return nd


def cdm_max_length(d, stream=None) -> float:
    c = C.c_float(0)
    _lib.check(_lib.lib().regb_cdm_max_length(C.byref(_field(_host(d, np.float32))), C.byref(c), _stream(stream)))
    return float(c.value)


def cdm_smooth(d, smoothing, out=None, stream=None):
    src = _host(d, np.float32)
    dd = _like(src, src.shape) if out is None else out
    _lib.check(_lib.lib().regb_cdm_smooth(C.byref(_field(src)), C.byref(_field(dd)), float(smoothing),
                                          _stream(stream)))
    return dd


# ---------------------------------------------------------------- whole registrations
class reg:
    """tipl::reg entry points."""

    AFFINE, RIGID_BODY, TRANSLOCATION = 15, 3, 1
    CORR, MI, MI32 = 0, 1, 2  # MI32: the 32x32-bin MI variant

    @staticmethod
    def linear_param(reg_type=15, cost_type=1, bound=0, search_count=16, absolute_bound=1) -> LinearParam:
        return LinearParam(reg_type, cost_type, bound, search_count, absolute_bound)

    @staticmethod
    def cdm_param(resolution=2.0, speed=0.3, smoothing=0.05, min_dimension=16, gradient_type="r") -> CdmParam:
        return CdmParam(resolution, speed, smoothing, min_dimension, ord(gradient_type))

    @staticmethod
    def linear(from_, from_vs, to, to_vs, arg=None, param: LinearParam | None = None, terminated=None):
        """tipl::reg::linear: returns (cost, arg[12], cost_evaluations).  from_ / to are
        one volume each or lists of image pairs (make_list(It), make_list(I) of mm_reg's
        mm_linear); the longer list is cut to the shorter one's length."""
        fl = list(from_) if isinstance(from_, (list, tuple)) else [from_]
        tl = list(to) if isinstance(to, (list, tuple)) else [to]
        n = min(len(fl), len(tl))  # run_optimize: min(from.size(), to.size()) cost functions
        if n < 1:
            raise ValueError("linear: empty image list")
        a = (np.array([0, 0, 0, 0, 0, 0, 1, 1, 1, 0, 0, 0], np.float32) if arg is None
             else np.array(arg, np.float32, copy=True))
        p = param or reg.linear_param()
        cost = C.c_float(0)
        evals = C.c_longlong(0)
        term = None if terminated is None else C.cast(terminated, C.c_void_p)
        vf = (_lib.Volume * n)(*[_vol(v) for v in fl[:n]])
        vt = (_lib.Volume * n)(*[_vol(v) for v in tl[:n]])
        st = _lib.lib().regb_linear_multi(vf, _fptr(np.asarray(from_vs, np.float32)), vt,
                                          _fptr(np.asarray(to_vs, np.float32)), n, _fptr(a), C.byref(p), term,
                                          C.byref(cost), C.byref(evals))
        _lib.check(st, allow=(_lib.REGB_OK, _lib.REGB_CANCELLED))
        return float(cost.value), a, int(evals.value)

    @staticmethod
    def cdm(It, Is, param: CdmParam | None = None, terminated=None, out=None, gradient_types=None):
        """tipl::reg::cdm_common: returns (field, ok).  It / Is are one volume each or
        equal-length lists of modality pairs (make_list(J), make_list(It) in mm_reg);
        gradient_types is cdm_param::gradient_type, one 'r' / 'd' per modality ('r'
        past its end; None = param.gradient_type for the first modality).  2-D uint8
        images (shape (h, w)) take the reference's dimension-2 path; their field has
        shape (h, w, 2)."""
        multi = isinstance(It, (list, tuple))
        Its = list(It) if multi else [It]
        Iss = list(Is) if isinstance(Is, (list, tuple)) else [Is]
        n = min(len(Its), len(Iss))  # cdm_common truncates the longer list (reg/cdm.hpp:542-545)
        if n < 1:
            raise ValueError("cdm: empty modality list")
        two_d = len(Its[0].shape) == 2
        p = param or reg.cdm_param()
        term = None if terminated is None else C.cast(terminated, C.c_void_p)
        gt = None if gradient_types is None else str(gradient_types).encode()
        if two_d:
            h, w = Its[0].shape
            d = _like(Its[0], (h, w, 2), dtype=_f32_like(Its[0])) if out is None else out

            def vol2(a):  # a 2-D image as a volume of dims (w, h, 1)
                return _vol(a.reshape(1, *a.shape))

            vt = (_lib.Volume * n)(*[vol2(a) for a in Its[:n]])
            vs = (_lib.Volume * n)(*[vol2(a) for a in Iss[:n]])
            if _is_dev(d):
                assert d.is_contiguous() and tuple(d.shape) == (h, w, 2)
                f = _lib.Field(d.data_ptr(), (C.c_int * 3)(w, h, 1), _lib.DEVICE)
            else:
                assert d.flags["C_CONTIGUOUS"] and d.dtype == np.float32 and d.shape == (h, w, 2)
                f = _lib.Field(d.ctypes.data, (C.c_int * 3)(w, h, 1), _lib.HOST)
            st = _lib.lib().regb_cdm2d_multi(vt, vs, n, C.byref(f), C.byref(p), gt, term)
            _lib.check(st, allow=(_lib.REGB_OK, _lib.REGB_FALSE, _lib.REGB_CANCELLED))
            return d, st != _lib.REGB_FALSE
        d = _like(Its[0], tuple(Its[0].shape) + (3,), dtype=_f32_like(Its[0])) if out is None else out
        vt = (_lib.Volume * n)(*[_vol(a) for a in Its[:n]])
        vs = (_lib.Volume * n)(*[_vol(a) for a in Iss[:n]])
        st = _lib.lib().regb_cdm_multi(vt, vs, n, C.byref(_field(d)), C.byref(p), gt, term)
        _lib.check(st, allow=(_lib.REGB_OK, _lib.REGB_FALSE, _lib.REGB_CANCELLED))
        return d, st != _lib.REGB_FALSE


# ---------------------------------------------------------------- serving engine
class Engine:
    """Continuous-batching registration server on one GPU (regb_engine_* in the C ABI).

    Jobs run concurrently: their affine probe sets share launches and their CDM
    levels iterate together.  Host arrays passed to submit() are kept alive here
    until the job is released."""

    def __init__(self, hbm_budget_bytes=0, max_active=64, gather_us=10, cdm_iters_per_round=4, affine_workers=3):
        L = _lib.lib()
        cfg = _lib.EngineConfig()
        L.regb_engine_config_default(C.byref(cfg))
        cfg.hbm_budget_bytes = int(hbm_budget_bytes)
        cfg.max_active = int(max_active)
        cfg.gather_us = int(gather_us)
        cfg.cdm_iters_per_round = int(cdm_iters_per_round)
        cfg.affine_workers = int(affine_workers)
        h = C.c_void_p()
        _lib.check(L.regb_engine_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._keep = {}
        self._tkeep = []

    def add_template(self, vol, vs=(1.0, 1.0, 1.0)) -> int:
        tid = C.c_int(-1)
        v = _vol(vol)
        _lib.check(_lib.lib().regb_engine_add_template(self._h, C.byref(v), _fptr(np.asarray(vs, np.float32)),
                                                       C.byref(tid)))
        self._tkeep.append(vol)
        return tid.value

    def submit(self, moving, moving_vs=(1.0, 1.0, 1.0), template=None, fixed=None, fixed_vs=(1.0, 1.0, 1.0),
               linear=True, linear_param: LinearParam | None = None, arg=None, cdm=False,
               cdm_param: CdmParam | None = None, field_out=None, subject_pre=False, mm_reg=False,
               field_rev_out=None, mapping_out=None, inv_mapping_out=None, prev_field=None,
               prev_field_rev=None) -> int:
        L = _lib.lib()
        j = _lib.Job()
        L.regb_job_default(C.byref(j))
        keep = [moving]
        if template is not None:
            j.template_id = int(template)
        else:
            j.template_id = -1
            j.fixed = _vol(fixed)
            keep.append(fixed)
        j.fixed_vs[:] = [float(v) for v in fixed_vs]
        j.moving = _vol(moving)
        j.moving_vs[:] = [float(v) for v in moving_vs]
        j.run_linear = int(bool(linear))
        if linear_param is None and mm_reg:
            # the mm_reg class registers with correlation by default (reg/mm_reg.hpp:53)
            linear_param = reg.linear_param(cost_type=reg.CORR)
        if linear_param is not None:
            j.linear = linear_param
        if arg is not None:
            j.arg[:] = [float(v) for v in arg]
        j.run_cdm = int(bool(cdm))
        j.subject_pre = int(bool(subject_pre))
        j.mm_reg = int(bool(mm_reg))
        if cdm_param is not None:
            j.cdm = cdm_param
        if field_out is not None:
            if _is_dev(field_out):
                j.field_out = field_out.data_ptr()
                j.field_location = _lib.DEVICE
            else:
                assert field_out.dtype == np.float32 and field_out.flags["C_CONTIGUOUS"]
                j.field_out = field_out.ctypes.data
                j.field_location = _lib.HOST
            keep.append(field_out)
        for name, buf in (("field_rev_out", field_rev_out), ("mapping_out", mapping_out),
                          ("inv_mapping_out", inv_mapping_out)):
            if buf is not None:
                # same location as field_out (host numpy or device tensor)
                setattr(j, name, buf.data_ptr() if _is_dev(buf) else buf.ctypes.data)
                if field_out is None:
                    j.field_location = _lib.DEVICE if _is_dev(buf) else _lib.HOST
                keep.append(buf)
        if prev_field is not None and prev_field_rev is not None:
            # an earlier registration's fields, at field_out's location (mm_reg's previous_t2f / f2t)
            for name, buf in (("prev_field", prev_field), ("prev_field_rev", prev_field_rev)):
                if not _is_dev(buf):
                    buf = np.ascontiguousarray(buf, np.float32)
                setattr(j, name, buf.data_ptr() if _is_dev(buf) else buf.ctypes.data)
                keep.append(buf)
        jid = C.c_uint64(0)
        _lib.check(L.regb_engine_submit(self._h, C.byref(j), C.byref(jid)))
        self._keep[jid.value] = keep
        return jid.value

    @staticmethod
    def _res(r):
        return {"status": r.status, "linear_cost": r.linear_cost, "arg": np.array(r.arg[:], np.float32),
                "cost_evals": r.cost_evals, "cdm_ok": bool(r.cdm_ok), "cdm_iterations": r.cdm_iterations,
                "queued_ms": r.queued_ms, "run_ms": r.run_ms, "cdm_rev_ok": bool(r.cdm_rev_ok),
                "r_linear": r.r_linear, "r_nonlinear": r.r_nonlinear}

    def poll(self, jid):
        r = _lib.Result()
        st = _lib.lib().regb_engine_poll(self._h, C.c_uint64(jid), C.byref(r))
        if st == _lib.REGB_PENDING:
            return None
        _lib.check(st)
        return self._res(r)

    def wait(self, jid, release=True):
        r = _lib.Result()
        _lib.check(_lib.lib().regb_engine_wait(self._h, C.c_uint64(jid), C.byref(r)))
        if release:
            _lib.lib().regb_engine_release_job(self._h, C.c_uint64(jid))
            self._keep.pop(jid, None)
        return self._res(r)

    def cancel(self, jid):
        _lib.check(_lib.lib().regb_engine_cancel(self._h, C.c_uint64(jid)))

    def stats(self):
        s = _lib.EngineStats()
        _lib.check(_lib.lib().regb_engine_get_stats(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in s._fields_}

    def close(self):
        if self._h:
            _lib.lib().regb_engine_destroy(self._h)
            self._h = None
            self._keep.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
