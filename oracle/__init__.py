"""Test infrastructure only: ctypes wrappers over the two CPU checkers.

* ``Oracle`` -- oracle/liboracle.so, the plain-C restatement of the reference's CPU
  hot path (oracle/oracle.c + oracle_core.h/oracle_field.h/oracle_cdm.h).
* ``Reference`` -- oracle/_ref/libtipl_ref.so, the reference's own header-only C++
  compiled from its sources by oracle/Makefile (present only where it was built).
* ``ReferenceGPU`` -- oracle/_ref/libtipl_ref_gpu.so, the reference's own CUDA path
  (nvcc, sm_100a), timed by bench.py as a secondary figure.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import this
package; the product path (tipl_b200) never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libtipl_ref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libtipl_ref_gpu.so")


def ref_root_from_env() -> str | None:
    """The reference source tree named by TIPL_REF_ROOT (None when unset)."""
    return os.environ.get("TIPL_REF_ROOT") or None


def build(ref_root: str | None = None, with_ref: bool = True) -> None:
    """Compile liboracle.so and, with with_ref, the reference driver from the source tree
    ref_root (or TIPL_REF_ROOT).  Asking for the reference build without naming a tree
    that holds the reference's reg/ headers is an error."""
    subprocess.check_call(["make", "-s", "-C", HERE, "oracle"])
    if not with_ref:
        return
    root = ref_root or ref_root_from_env()
    if not root or not os.path.isdir(os.path.join(root, "reg")):
        raise RuntimeError(f"reference source tree not found (ref_root={root!r}); pass ref_root or set "
                           "TIPL_REF_ROOT to the directory that holds reg/linear.hpp")
    subprocess.check_call(["make", "-s", "-C", HERE, "ref", "refgpu", f"REF_ROOT={root}"])


_P = C.c_void_p


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _dims(shape) -> np.ndarray:
    """numpy (z, y, x) shape -> reference (w, h, d) int array."""
    z, y, x = shape[:3]
    return np.array([x, y, z], dtype=np.int32)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u8(a):
    return np.ascontiguousarray(a, dtype=np.uint8)


class _Lib:
    _pfx = ""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = C.CDLL(path)

    def _fn(self, name):
        return getattr(self.lib, self._pfx + name)

    # -- mapping steps of the mm_reg pipeline (reg/mm_reg.hpp:271-345)
    def displacement_to_mapping(self, dis, T):
        d = np.ascontiguousarray(dis, np.float32)
        out = np.zeros_like(d)
        self._fn("displacement_to_mapping" + ("" if self._pfx == "tiplref_" else "_f32"))(
            _ptr(d), _ptr(_dims(d.shape)), _ptr(_f32(T)), _ptr(out))
        return out

    def inv_displacement_to_mapping(self, inv_dis, T, map_shape):
        d = np.ascontiguousarray(inv_dis, np.float32)
        out = np.zeros(tuple(map_shape) + (3,), np.float32)
        self._fn("inv_displacement_to_mapping" + ("" if self._pfx == "tiplref_" else "_f32"))(
            _ptr(d), _ptr(_dims(d.shape)), _ptr(_f32(T)), _ptr(_dims(map_shape)), _ptr(out))
        return out

    def compose_mapping(self, img, mapping):
        m = np.ascontiguousarray(mapping, np.float32)
        out = np.zeros(m.shape[:3], np.uint8)
        self._fn("compose_mapping_u8")(_ptr(_u8(img)), _ptr(_dims(img.shape)), _ptr(m), _ptr(_dims(m.shape)),
                                       _ptr(out))
        return out

    def match_fov(self, It, T, moving_shape):
        out = np.zeros(It.shape, np.uint8)
        self.lib.orc_match_fov_u8(_ptr(_u8(It)), _ptr(_dims(It.shape)), _ptr(_f32(T)), _ptr(_dims(moving_shape)),
                                  _ptr(out))
        return out

    def correlation(self, x, y, masked=False):
        f = self._fn("correlation_ygz_u8" if masked else "correlation_u8")
        f.restype = C.c_double
        return f(_ptr(_u8(x)), _ptr(_u8(y)), C.c_longlong(x.size))

    # -- subject preprocessing of the mm_reg pipeline (reg/mm_reg.hpp:14-20)
    def gaussian(self, img, bandwidth=1):
        out = np.ascontiguousarray(img, np.float32).copy()
        self._fn("gaussian" if self._pfx == "tiplref_" else "gaussian_f32")(_ptr(out), _ptr(_dims(out.shape)),
                                                                           C.c_int(bandwidth))
        return out

    def subject_image_pre(self, img):
        out = np.zeros(img.shape, np.uint8)
        self._fn("subject_image_pre" if self._pfx == "tiplref_" else "subject_image_pre_f32")(
            _ptr(np.ascontiguousarray(img, np.float32)), _ptr(_dims(img.shape)), _ptr(out))
        return out

    def otsu_threshold(self, img):
        a = np.ascontiguousarray(img, np.float32)
        if self._pfx == "tiplref_":
            f = self.lib.tiplref_otsu_threshold
            f.restype = C.c_float
            return f(_ptr(a), _ptr(_dims(a.shape)))
        f = self.lib.orc_otsu_threshold_f32
        f.restype = C.c_float
        return f(_ptr(a), C.c_longlong(a.size))

    def otsu_median(self, img):
        a = np.ascontiguousarray(img, np.float32)
        if self._pfx == "tiplref_":
            f = self.lib.tiplref_otsu_median
            f.restype = C.c_float
            return f(_ptr(a), _ptr(_dims(a.shape)))
        f = self.lib.orc_otsu_median_f32
        f.restype = C.c_float
        return f(_ptr(a), C.c_longlong(a.size))

    # -- mask-moment initialisation of linear() (reg/linear.hpp:658-684)
    def has_mask(self, img) -> bool:
        return bool(self._fn("has_mask" if self._pfx == "tiplref_" else "has_mask_u8")(_ptr(_u8(img)),
                                                                                        _ptr(_dims(img.shape))))

    def estimate_affine_param(self, src, src_vs, tgt, tgt_vs) -> np.ndarray:
        a = np.zeros(12, np.float32)
        self._fn("estimate_affine_param" + ("" if self._pfx == "tiplref_" else "_u8"))(
            _ptr(_u8(src)), _ptr(_dims(src.shape)), _ptr(_f32(src_vs)), _ptr(_u8(tgt)), _ptr(_dims(tgt.shape)),
            _ptr(_f32(tgt_vs)), _ptr(a))
        return a

    def matrix_to_affine_param(self, T, from_shape, from_vs, to_shape, to_vs) -> np.ndarray:
        a = np.zeros(12, np.float32)
        self._fn("matrix_to_affine_param")(_ptr(_f32(T)), _ptr(_dims(from_shape)), _ptr(_f32(from_vs)),
                                           _ptr(_dims(to_shape)), _ptr(_f32(to_vs)), _ptr(a))
        return a

    def eigen_sym3(self, A):
        A = np.ascontiguousarray(A, np.float64).reshape(9)
        V, d = np.zeros(9), np.zeros(3)
        self._fn("eigen_sym3")(_ptr(A), _ptr(V), _ptr(d))
        return V, d


class Oracle(_Lib):
    """Plain-C restatement.  Volumes are numpy arrays shaped (z, y, x); fields (z, y, x, 3)."""

    _pfx = "orc_"

    def __init__(self, path: str = ORACLE_SO):
        super().__init__(path)
        L = self.lib
        L.orc_mi_cost_from_hist.restype = C.c_double
        L.orc_mi_cost_u8.restype = C.c_double
        L.orc_mi32_cost_u8.restype = C.c_double
        L.orc_corr_cost_u8.restype = C.c_double
        L.orc_mi_cost_u8_f64.restype = C.c_double
        L.orc_corr_cost_u8_f64.restype = C.c_double
        for n in ("orc_cdm_gradient_u8", "orc_cdm_gradient_f32", "orc_cdm_max_len_f32"):
            getattr(L, n).restype = C.c_float
        for n in ("orc_cdm_gradient_f64", "orc_cdm_max_len_f64"):
            getattr(L, n).restype = C.c_double
        L.orc_cdm_smooth_f32.argtypes = [_P, _P, _P, C.c_float]
        L.orc_cdm_smooth_f64.argtypes = [_P, _P, _P, C.c_double]
        for sfx in ("u8", "f32", "f64"):
            getattr(L, f"orc_cdm_level_{sfx}").argtypes = [_P, _P, _P, _P, C.c_float, C.c_float, C.c_float,
                                                          C.c_uint, C.c_int, _P]
            getattr(L, f"orc_cdm_multi_{sfx}").argtypes = [_P, _P, C.c_int, _P, _P, C.c_float, C.c_float,
                                                          C.c_float, C.c_uint, C.c_char_p, _P]

    def normalize_to_u8(self, img, upper=255.999):
        """normalize_upper_lower2 of a float32 or uint16 volume; (out, ok)."""
        out = np.zeros(img.shape, np.uint8)
        if img.dtype == np.uint16:
            ok = self.lib.orc_normalize_to_u8_u16(_ptr(np.ascontiguousarray(img)), C.c_longlong(img.size), _ptr(out),
                                                  C.c_float(upper))
        else:
            ok = self.lib.orc_normalize_to_u8_f32(_ptr(_f32(img)), C.c_longlong(img.size), _ptr(out), C.c_float(upper))
        return out, bool(ok)

    # -- transforms
    def affine_to_matrix(self, param, from_shape, from_vs, to_shape, to_vs) -> np.ndarray:
        T = np.zeros(12, np.float32)
        self.lib.orc_affine_to_matrix(_ptr(_f32(param)), _ptr(_dims(from_shape)), _ptr(_f32(from_vs)),
                                      _ptr(_dims(to_shape)), _ptr(_f32(to_vs)), _ptr(T))
        return T

    def affine_to_matrix_f64(self, param, from_shape, from_vs, to_shape, to_vs) -> np.ndarray:
        T = np.zeros(12, np.float64)
        p = np.ascontiguousarray(param, np.float64)
        self.lib.orc_affine_to_matrix_f64(_ptr(p), _ptr(_dims(from_shape)),
                                          _ptr(np.ascontiguousarray(from_vs, np.float64)), _ptr(_dims(to_shape)),
                                          _ptr(np.ascontiguousarray(to_vs, np.float64)), _ptr(T))
        return T

    def matrix_inverse(self, T) -> np.ndarray:
        T = _f32(T).copy()
        self.lib.orc_matrix_inverse(_ptr(T))
        return T

    # -- resample / costs
    def resample(self, src, out_shape, T, allow_crop=True):
        if src.dtype == np.uint8:
            out = np.zeros(out_shape, np.uint8)
            self.lib.orc_resample_u8(_ptr(_u8(src)), _ptr(_dims(src.shape)), _ptr(out), _ptr(_dims(out_shape)),
                                     _ptr(_f32(T)), int(allow_crop))
        else:
            out = np.zeros(out_shape, np.float32)
            self.lib.orc_resample_f32(_ptr(_f32(src)), _ptr(_dims(src.shape)), _ptr(out), _ptr(_dims(out_shape)),
                                      _ptr(_f32(T)), int(allow_crop))
        return out

    def histogram(self, img) -> np.ndarray:
        h = np.zeros(256, np.int32)
        self.lib.orc_histogram_u8(_ptr(_u8(img)), C.c_longlong(img.size), _ptr(h))
        return h

    def mi_hist(self, fixed, moving, T) -> np.ndarray:
        h = np.zeros(65536, np.int32)
        self.lib.orc_mi_hist_u8(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                _ptr(_dims(moving.shape)), _ptr(_f32(T)), _ptr(h))
        return h

    def mi_cost_from_hist(self, hist, from_hist) -> float:
        return self.lib.orc_mi_cost_from_hist(_ptr(np.ascontiguousarray(hist, np.int32)),
                                              _ptr(np.ascontiguousarray(from_hist, np.int32)))

    def mi_cost(self, fixed, moving, T) -> float:
        return self.lib.orc_mi_cost_u8(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                       _ptr(_dims(moving.shape)), _ptr(_f32(T)))

    def mi32_cost(self, fixed, moving, T, with_hist=False):
        """MI on a 32x32 joint histogram of the volumes quantised to 0..31; with_hist
        also returns the 1024 joint counts."""
        h = np.zeros(1024, np.int32)
        c = self.lib.orc_mi32_cost_u8(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                      _ptr(_dims(moving.shape)), _ptr(_f32(T)), _ptr(h))
        return (c, h) if with_hist else c

    def mi_cost_f64(self, fixed, moving, T64) -> float:
        """MI cost with the transform and interpolation in double (error reporting)."""
        return self.lib.orc_mi_cost_u8_f64(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                           _ptr(_dims(moving.shape)), _ptr(np.ascontiguousarray(T64, np.float64)))

    def corr_cost_f64(self, fixed, moving, T64) -> float:
        return self.lib.orc_corr_cost_u8_f64(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                             _ptr(_dims(moving.shape)), _ptr(np.ascontiguousarray(T64, np.float64)))

    def corr_cost(self, fixed, moving, T) -> float:
        return self.lib.orc_corr_cost_u8(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                         _ptr(_dims(moving.shape)), _ptr(_f32(T)))

    # -- CDM passes
    @staticmethod
    def _sfx(a):
        return {np.dtype(np.uint8): "u8", np.dtype(np.float32): "f32", np.dtype(np.float64): "f64"}[a.dtype]

    @staticmethod
    def _fdt(sfx):
        return np.float64 if sfx == "f64" else np.float32

    def compose(self, Is, dis):
        s = self._sfx(Is)
        out = np.zeros_like(Is)
        d = np.ascontiguousarray(dis, self._fdt(s))
        getattr(self.lib, f"orc_compose_{s}")(_ptr(np.ascontiguousarray(Is)), _ptr(_dims(Is.shape)), _ptr(d),
                                              _ptr(out))
        return out

    def cdm_gradient(self, Js, It, gradient_type="r"):
        s = self._sfx(Js)
        nd = np.zeros(Js.shape + (3,), self._fdt(s))
        c = getattr(self.lib, f"orc_cdm_gradient_{s}")(_ptr(np.ascontiguousarray(Js)),
                                                      _ptr(np.ascontiguousarray(It, Js.dtype)),
                                                      _ptr(_dims(Js.shape)), _ptr(nd), ord(gradient_type))
        return nd, c

    def _fs(self, d):
        return "f64" if d.dtype == np.float64 else "f32"

    def cdm_poisson(self, new_d, sweeps=12):
        s = self._fs(new_d)
        d = np.ascontiguousarray(new_d, self._fdt(s)).copy()
        getattr(self.lib, f"orc_cdm_poisson_{s}")(_ptr(d), _ptr(_dims(d.shape)), sweeps)
        return d

    def cdm_max_len(self, d):
        s = self._fs(d)
        d = np.ascontiguousarray(d, self._fdt(s))
        return getattr(self.lib, f"orc_cdm_max_len_{s}")(_ptr(d), _ptr(_dims(d.shape)))

    def accumulate(self, cur_d, new_d):
        s = self._fs(new_d)
        nd = np.ascontiguousarray(new_d, self._fdt(s)).copy()
        cd = np.ascontiguousarray(cur_d, self._fdt(s))
        getattr(self.lib, f"orc_accumulate_{s}")(_ptr(cd), _ptr(nd), _ptr(_dims(nd.shape)))
        return nd

    def cdm_smooth(self, d, smoothing, out=None):
        s = self._fs(d)
        d = np.ascontiguousarray(d, self._fdt(s))
        dd = np.zeros_like(d) if out is None else np.ascontiguousarray(out, self._fdt(s)).copy()
        getattr(self.lib, f"orc_cdm_smooth_{s}")(_ptr(d), _ptr(dd), _ptr(_dims(d.shape)), smoothing)
        return dd

    def downsample(self, img):
        s = self._sfx(img)
        z, y, x = img.shape
        out = np.zeros(((z + 1) // 2, (y + 1) // 2, (x + 1) // 2), img.dtype)
        getattr(self.lib, f"orc_downsample_{s}")(_ptr(np.ascontiguousarray(img)), _ptr(_dims(img.shape)), _ptr(out))
        return out

    def upsample_field_x2(self, d, out_shape):
        s = self._fs(d)
        d = np.ascontiguousarray(d, self._fdt(s))
        out = np.zeros(tuple(out_shape) + (3,), self._fdt(s))
        getattr(self.lib, f"orc_upsample_field_x2_{s}")(_ptr(d), _ptr(_dims(d.shape)), _ptr(out),
                                                        _ptr(_dims(out_shape)))
        return out

    def cdm(self, It, Is, resolution=2.0, speed=0.3, smoothing=0.05, min_dimension=16, gradient_type="r"):
        """The reference's cdm() driver for one modality; returns (field, ok, iterations)."""
        s = self._sfx(It)
        d = np.zeros(It.shape + (3,), self._fdt(s))
        iters = C.c_int(0)
        ok = getattr(self.lib, f"orc_cdm_level_{s}")(_ptr(np.ascontiguousarray(It)),
                                                    _ptr(np.ascontiguousarray(Is, It.dtype)), _ptr(_dims(It.shape)),
                                                    _ptr(d), resolution, speed, smoothing, min_dimension,
                                                    ord(gradient_type), C.byref(iters))
        return d, bool(ok), iters.value

    def cdm2d(self, It, Is, resolution=2.0, speed=0.3, smoothing=0.05, min_dimension=16, gradient_types=""):
        """The reference's cdm() driver at dimension 2 over lists of uint8 image pairs of
        shape (h, w); returns (field (h, w, 2), ok, iterations)."""
        It = [np.ascontiguousarray(a, np.uint8) for a in It]
        Is = [np.ascontiguousarray(a, np.uint8) for a in Is]
        h, w = It[0].shape
        pt = (C.c_void_p * len(It))(*[a.ctypes.data for a in It])
        ps = (C.c_void_p * len(Is))(*[a.ctypes.data for a in Is])
        d = np.zeros((h, w, 2), np.float32)
        iters = C.c_int(0)
        fn = self.lib.orc2_cdm_multi_u8
        fn.argtypes = [_P, _P, C.c_int, _P, _P, C.c_float, C.c_float, C.c_float, C.c_uint, C.c_char_p, _P]
        ok = fn(pt, ps, len(It), _ptr(np.array([w, h], np.int32)), _ptr(d), resolution, speed, smoothing,
                min_dimension, gradient_types.encode(), C.byref(iters))
        return d, bool(ok), iters.value

    def cdm_multi(self, It, Is, resolution=2.0, speed=0.3, smoothing=0.05, min_dimension=16, gradient_types=""):
        """The reference's cdm() driver over lists of modality pairs (reg/cdm.hpp:419-435);
        returns (field, ok, iterations)."""
        s = self._sfx(It[0])
        It = [np.ascontiguousarray(a, It[0].dtype) for a in It]
        Is = [np.ascontiguousarray(a, It[0].dtype) for a in Is]
        pt = (C.c_void_p * len(It))(*[a.ctypes.data for a in It])
        ps = (C.c_void_p * len(Is))(*[a.ctypes.data for a in Is])
        d = np.zeros(It[0].shape + (3,), self._fdt(s))
        iters = C.c_int(0)
        ok = getattr(self.lib, f"orc_cdm_multi_{s}")(pt, ps, len(It), _ptr(_dims(It[0].shape)), _ptr(d), resolution,
                                                    speed, smoothing, min_dimension, gradient_types.encode(),
                                                    C.byref(iters))
        return d, bool(ok), iters.value


class Reference(_Lib):
    """The reference's own CPU implementation (compiled from its headers)."""

    _pfx = "tiplref_"

    def __init__(self, path: str = REF_SO):
        super().__init__(path)
        L = self.lib
        for n in ("tiplref_mi_cost", "tiplref_corr_cost"):
            getattr(L, n).restype = C.c_double
        for n in ("tiplref_cdm_gradient_u8", "tiplref_cdm_gradient_f32", "tiplref_cdm_max_len", "tiplref_linear",
                  "tiplref_linear_bound"):
            getattr(L, n).restype = C.c_float
        L.tiplref_cdm_smooth.argtypes = [_P, _P, _P, C.c_float]
        for n in ("tiplref_cdm_u8", "tiplref_cdm_f32"):
            getattr(L, n).argtypes = [_P, _P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_uint]
        L.tiplref_normalize_to_u8.argtypes = [_P, _P, _P, C.c_float]

    def set_threads(self, n: int) -> None:
        self.lib.tiplref_set_threads(int(n))

    def affine_to_matrix(self, param, from_shape, from_vs, to_shape, to_vs):
        T = np.zeros(12, np.float32)
        self.lib.tiplref_affine_to_matrix(_ptr(_f32(param)), _ptr(_dims(from_shape)), _ptr(_f32(from_vs)),
                                          _ptr(_dims(to_shape)), _ptr(_f32(to_vs)), _ptr(T))
        return T

    def matrix_inverse(self, T):
        T = _f32(T).copy()
        self.lib.tiplref_matrix_inverse(_ptr(T))
        return T

    def resample(self, src, out_shape, T):
        if src.dtype == np.uint8:
            out = np.zeros(out_shape, np.uint8)
            self.lib.tiplref_resample_u8(_ptr(_u8(src)), _ptr(_dims(src.shape)), _ptr(out), _ptr(_dims(out_shape)),
                                         _ptr(_f32(T)))
        else:
            out = np.zeros(out_shape, np.float32)
            self.lib.tiplref_resample_f32(_ptr(_f32(src)), _ptr(_dims(src.shape)), _ptr(out),
                                          _ptr(_dims(out_shape)), _ptr(_f32(T)))
        return out

    def histogram(self, img):
        h = np.zeros(256, np.int32)
        self.lib.tiplref_histogram_u8(_ptr(_u8(img)), _ptr(_dims(img.shape)), _ptr(h))
        return h

    def mi_hist(self, fixed, moving, T):
        h = np.zeros(65536, np.int32)
        self.lib.tiplref_mi_hist(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                 _ptr(_dims(moving.shape)), _ptr(_f32(T)), _ptr(h))
        return h

    def mi_cost(self, fixed, moving, T):
        return self.lib.tiplref_mi_cost(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                        _ptr(_dims(moving.shape)), _ptr(_f32(T)))

    def corr_cost(self, fixed, moving, T):
        return self.lib.tiplref_corr_cost(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_u8(moving)),
                                          _ptr(_dims(moving.shape)), _ptr(_f32(T)))

    def compose(self, Is, dis):
        out = np.zeros_like(Is)
        fn = self.lib.tiplref_compose_u8 if Is.dtype == np.uint8 else self.lib.tiplref_compose_f32
        fn(_ptr(np.ascontiguousarray(Is)), _ptr(_dims(Is.shape)), _ptr(_f32(dis)), _ptr(out))
        return out

    def cdm_gradient(self, Js, It, gradient_type="r"):
        nd = np.zeros(Js.shape + (3,), np.float32)
        fn = self.lib.tiplref_cdm_gradient_u8 if Js.dtype == np.uint8 else self.lib.tiplref_cdm_gradient_f32
        c = fn(_ptr(np.ascontiguousarray(Js)), _ptr(np.ascontiguousarray(It, Js.dtype)), _ptr(_dims(Js.shape)),
               _ptr(nd), ord(gradient_type))
        return nd, c

    def cdm_poisson(self, new_d):
        d = _f32(new_d).copy()
        self.lib.tiplref_cdm_poisson(_ptr(d), _ptr(_dims(d.shape)))
        return d

    def cdm_max_len(self, d):
        d = _f32(d)
        return self.lib.tiplref_cdm_max_len(_ptr(d), _ptr(_dims(d.shape)))

    def accumulate(self, cur_d, new_d):
        nd = _f32(new_d).copy()
        self.lib.tiplref_accumulate(_ptr(_f32(cur_d)), _ptr(nd), _ptr(_dims(nd.shape)))
        return nd

    def cdm_smooth(self, d, smoothing):
        d = _f32(d)
        dd = np.zeros_like(d)
        self.lib.tiplref_cdm_smooth(_ptr(d), _ptr(dd), _ptr(_dims(d.shape)), smoothing)
        return dd

    def downsample(self, img):
        z, y, x = img.shape
        out = np.zeros(((z + 1) // 2, (y + 1) // 2, (x + 1) // 2), img.dtype)
        fn = self.lib.tiplref_downsample_u8 if img.dtype == np.uint8 else self.lib.tiplref_downsample_f32
        fn(_ptr(np.ascontiguousarray(img)), _ptr(_dims(img.shape)), _ptr(out))
        return out

    def upsample_field_x2(self, d, out_shape):
        d = _f32(d)
        out = np.zeros(tuple(out_shape) + (3,), np.float32)
        self.lib.tiplref_upsample_field_x2(_ptr(d), _ptr(_dims(d.shape)), _ptr(out), _ptr(_dims(out_shape)))
        return out

    def cdm(self, It, Is, resolution=2.0, speed=0.3, smoothing=0.05, min_dimension=16):
        d = np.zeros(It.shape + (3,), np.float32)
        fn = self.lib.tiplref_cdm_u8 if It.dtype == np.uint8 else self.lib.tiplref_cdm_f32
        ok = fn(_ptr(np.ascontiguousarray(It)), _ptr(np.ascontiguousarray(Is, It.dtype)), _ptr(_dims(It.shape)),
                _ptr(d), resolution, speed, smoothing, min_dimension)
        return d, bool(ok)

    def cdm2d(self, It, Is, resolution=2.0, speed=0.3, smoothing=0.05, min_dimension=16, gradient_types=""):
        """cdm_common<void, unsigned char, 2> over lists of uint8 image pairs of shape
        (h, w); returns (field (h, w, 2), ok)."""
        It = [np.ascontiguousarray(a, np.uint8) for a in It]
        Is = [np.ascontiguousarray(a, np.uint8) for a in Is]
        h, w = It[0].shape
        pt = (C.c_void_p * len(It))(*[a.ctypes.data for a in It])
        ps = (C.c_void_p * len(Is))(*[a.ctypes.data for a in Is])
        d = np.zeros((h, w, 2), np.float32)
        fn = self.lib.tiplref_cdm2d_multi_u8
        fn.argtypes = [_P, _P, C.c_int, _P, _P, C.c_float, C.c_float, C.c_float, C.c_uint, C.c_char_p]
        ok = fn(pt, ps, len(It), _ptr(np.array([w, h], np.int32)), _ptr(d), resolution, speed, smoothing,
                min_dimension, gradient_types.encode())
        return d, bool(ok)

    def cdm_multi(self, It, Is, resolution=2.0, speed=0.3, smoothing=0.05, min_dimension=16, gradient_types=""):
        """cdm_common over lists of modality pairs; returns (field, ok)."""
        u8 = It[0].dtype == np.uint8
        It = [np.ascontiguousarray(a, It[0].dtype) for a in It]
        Is = [np.ascontiguousarray(a, It[0].dtype) for a in Is]
        pt = (C.c_void_p * len(It))(*[a.ctypes.data for a in It])
        ps = (C.c_void_p * len(Is))(*[a.ctypes.data for a in Is])
        d = np.zeros(It[0].shape + (3,), np.float32)
        fn = self.lib.tiplref_cdm_multi_u8 if u8 else self.lib.tiplref_cdm_multi_f32
        fn.argtypes = [_P, _P, C.c_int, _P, _P, C.c_float, C.c_float, C.c_float, C.c_uint, C.c_char_p]
        ok = fn(pt, ps, len(It), _ptr(_dims(It[0].shape)), _ptr(d), resolution, speed, smoothing, min_dimension,
                gradient_types.encode())
        return d, bool(ok)

    def linear(self, fixed, fixed_vs, moving, moving_vs, arg=None, reg_type=15, cost_type=1):
        """tipl::reg::linear (affine by default, MI by default); returns (cost, 12 params)."""
        a = np.array([0, 0, 0, 0, 0, 0, 1, 1, 1, 0, 0, 0], np.float32) if arg is None else _f32(arg).copy()
        c = self.lib.tiplref_linear(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_f32(fixed_vs)),
                                    _ptr(_u8(moving)), _ptr(_dims(moving.shape)), _ptr(_f32(moving_vs)), _ptr(a),
                                    int(reg_type), int(cost_type))
        return float(c), a

    def linear_bound(self, fixed, fixed_vs, moving, moving_vs, arg=None, reg_type=15, cost_type=1, bound=0):
        """tipl::reg::linear with bound table 0 reg, 1 narrow (single-threaded L-BFGS from arg), 2 large."""
        a = np.array([0, 0, 0, 0, 0, 0, 1, 1, 1, 0, 0, 0], np.float32) if arg is None else _f32(arg).copy()
        c = self.lib.tiplref_linear_bound(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_f32(fixed_vs)),
                                          _ptr(_u8(moving)), _ptr(_dims(moving.shape)), _ptr(_f32(moving_vs)),
                                          _ptr(a), int(reg_type), int(cost_type), int(bound))
        return float(c), a

    def nifti_load(self, path, cap=1 << 28):
        """gz_nifti(path) >> I >> vs >> T >> is_mni: (I float32 (z, y, x), vs, srow[12], is_mni),
        or None when the reference fails to read the file."""
        dim = np.zeros(3, np.int32)
        vs = np.zeros(3, np.float32)
        srow = np.zeros(12, np.float32)
        mni = C.c_int(0)
        buf = np.zeros(int(cap), np.float32)
        ok = self.lib.tiplref_nifti_load(str(path).encode(), _ptr(dim), _ptr(vs), _ptr(srow), _ptr(buf),
                                         C.c_longlong(int(cap)), C.byref(mni))
        if not ok:
            return None
        x, y, z = (int(v) for v in dim)
        return buf[:x * y * z].reshape(z, y, x).copy(), vs, srow, bool(mni.value)

    def nifti_save(self, path, vol, vs, srow, is_mni=False):
        """gz_nifti(path, out) << vs << T << is_mni << I for a float32 or uint8 volume."""
        v = np.ascontiguousarray(vol)
        assert v.dtype in (np.float32, np.uint8)
        return bool(self.lib.tiplref_nifti_save(str(path).encode(), _ptr(v), int(v.dtype == np.uint8),
                                                _ptr(_dims(v.shape)), _ptr(_f32(vs)), _ptr(_f32(srow)), int(is_mni)))

    def nifti_save4(self, path, vol4, vs, srow):
        """gz_nifti(path, out) << vs << T << I for a float32 array (t, z, y, x)."""
        v = np.ascontiguousarray(vol4, np.float32)
        t, z, y, x = v.shape
        return bool(self.lib.tiplref_nifti_save4(str(path).encode(), _ptr(v), _ptr(np.array([x, y, z, t], np.int32)),
                                                 _ptr(_f32(vs)), _ptr(_f32(srow))))

    def normalize_u16_to_u8(self, img, upper=255.999):
        out = np.zeros(img.shape, np.uint8)
        self.lib.tiplref_normalize_u16_to_u8(_ptr(np.ascontiguousarray(img, np.uint16)), _ptr(_dims(img.shape)),
                                             _ptr(out), C.c_float(upper))
        return out

    def normalize_to_u8(self, img, upper=255.999):
        out = np.zeros(img.shape, np.uint8)
        self.lib.tiplref_normalize_to_u8(_ptr(_f32(img)), _ptr(_dims(img.shape)), _ptr(out), upper)
        return out


class ReferenceGPU(_Lib):
    """The reference's own CUDA path (tipl::reg::linear / cdm_common with cuda = true)."""

    _pfx = "tiplrefgpu_"

    def __init__(self, path: str = REF_GPU_SO):
        super().__init__(path)
        L = self.lib
        L.tiplrefgpu_linear.restype = C.c_float
        L.tiplrefgpu_cdm.argtypes = [_P, _P, _P, _P, C.c_float, C.c_float, C.c_float, C.c_uint]

    def set_threads(self, n: int) -> None:
        self.lib.tiplrefgpu_set_threads(int(n))

    def linear(self, fixed, fixed_vs, moving, moving_vs, arg=None, reg_type=15, cost_type=1):
        a = np.array([0, 0, 0, 0, 0, 0, 1, 1, 1, 0, 0, 0], np.float32) if arg is None else _f32(arg).copy()
        c = self.lib.tiplrefgpu_linear(_ptr(_u8(fixed)), _ptr(_dims(fixed.shape)), _ptr(_f32(fixed_vs)),
                                       _ptr(_u8(moving)), _ptr(_dims(moving.shape)), _ptr(_f32(moving_vs)), _ptr(a),
                                       int(reg_type), int(cost_type))
        return float(c), a

    def cdm(self, It, Is, resolution=2.0, speed=0.3, smoothing=0.05, min_dimension=16):
        d = np.zeros(It.shape + (3,), np.float32)
        ok = self.lib.tiplrefgpu_cdm(_ptr(_u8(It)), _ptr(_u8(Is)), _ptr(_dims(It.shape)), _ptr(d), resolution, speed,
                                     smoothing, min_dimension)
        return d, bool(ok)
