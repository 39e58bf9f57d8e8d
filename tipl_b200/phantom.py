"""Seeded synthetic volumes for the registration workloads (no datasets ship here).

Shapes are numpy order (z, y, x); the device and C-ABI use x-fastest storage, which
is the same memory layout.  Seeds follow ``20261203 + 1000*config + job``.

* ``blob_volume``        -- sum of isotropic Gaussian blobs + N(0, noise) (CDM workload).
* ``smooth_field``       -- white noise Gaussian-smoothed, scaled to a max length.
* ``warp``               -- a volume warped by a displacement (compose semantics).
* ``class_phantom``      -- three-class blob phantom inside a smoothed ellipsoid,
                            scaled to [0, 4095] (the affine workloads).
* ``random_affine``      -- a random 12-parameter affine in the reference's
                            parameter layout (translation, rotation, scaling, shear).
* ``normalize_to_u8``    -- the reference's template_image_pre quantisation,
                            (v - min) * (255.999 / range) truncated
                            (reg/mm_reg.hpp:28-34, numerical/numerical.hpp:909-927).
"""
from __future__ import annotations

import numpy as np
from scipy import ndimage

SEED_BASE = 20261203


def seed_for(config: int, job: int = 0) -> int:
    return SEED_BASE + 1000 * config + job


def _grid(shape):
    z, y, x = np.meshgrid(*(np.arange(n, dtype=np.float32) for n in shape), indexing="ij")
    return z, y, x


def blob_volume(shape, rng: np.random.Generator, n_blobs=32, sigma=(3.0, 8.0), amp=(0.2, 1.0),
                noise=0.01) -> np.ndarray:
    """Sum of ``n_blobs`` isotropic Gaussians with centres U(0, shape), sigma and amplitude
    uniform in the given ranges, plus N(0, noise)."""
    shape = tuple(int(s) for s in shape)
    out = np.zeros(shape, np.float32)
    axes = [np.arange(n, dtype=np.float32) for n in shape]
    for _ in range(n_blobs):
        c = [rng.uniform(0, n) for n in shape]
        s = rng.uniform(*sigma)
        a = rng.uniform(*amp)
        g = [np.exp(-((ax - ci) ** 2) / (2 * s * s)).astype(np.float32) for ax, ci in zip(axes, c)]
        out += a * (g[0][:, None, None] * g[1][None, :, None] * g[2][None, None, :])
    if noise:
        out += rng.normal(0.0, noise, shape).astype(np.float32)
    return out


def smooth_field(shape, rng: np.random.Generator, sigma=6.0, max_len=3.0) -> np.ndarray:
    """Displacement field (z, y, x, 3) with components (dx, dy, dz): white N(0,1) noise
    smoothed with a Gaussian of ``sigma`` voxels, scaled so max |d| = ``max_len``."""
    shape = tuple(int(s) for s in shape)
    comps = [ndimage.gaussian_filter(rng.normal(0, 1, shape).astype(np.float32), sigma, mode="reflect")
             for _ in range(3)]
    d = np.stack(comps, axis=-1).astype(np.float32)
    m = float(np.sqrt((d * d).sum(-1)).max())
    if m > 0:
        d *= np.float32(max_len / m)
    return d


def warp(vol: np.ndarray, disp: np.ndarray) -> np.ndarray:
    """out(x) = trilinear(vol, x + d(x)), 0 outside (compose_displacement semantics)."""
    z, y, x = _grid(vol.shape)
    coords = np.stack([z + disp[..., 2], y + disp[..., 1], x + disp[..., 0]])
    return ndimage.map_coordinates(vol, coords, order=1, mode="constant", cval=0.0).astype(vol.dtype)


def ellipsoid_mask(shape, radii_frac=(0.42, 0.42, 0.42), smooth=2.0) -> np.ndarray:
    z, y, x = _grid(shape)
    c = [(n - 1) / 2.0 for n in shape]
    r = [f * n for f, n in zip(radii_frac, shape)]
    q = ((z - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((x - c[2]) / r[2]) ** 2
    m = (q <= 1.0).astype(np.float32)
    return ndimage.gaussian_filter(m, smooth) if smooth else m


def class_phantom(shape, rng: np.random.Generator) -> np.ndarray:
    """Three intensity classes: background 0 outside a smoothed ellipsoid, inside it
    a level U(800,1200) and, where the blob field is high, a level U(2500,3200);
    returned as float32 in [0, 4095]."""
    blobs = blob_volume(shape, rng, noise=0.0)
    blobs /= max(float(blobs.max()), 1e-6)
    mask = ellipsoid_mask(shape)
    lo = rng.uniform(800, 1200)
    hi = rng.uniform(2500, 3200)
    t = np.clip((blobs - 0.35) / 0.2, 0.0, 1.0)
    img = mask * (lo + (hi - lo) * t)
    img = ndimage.gaussian_filter(img.astype(np.float32), 1.0)
    return np.clip(img, 0, 4095).astype(np.float32)


def random_affine(rng: np.random.Generator, rot_deg=10.0, trans_vox=10.0, scale=(0.9, 1.1), shear=0.05,
                  vs=(1.0, 1.0, 1.0)) -> np.ndarray:
    """12 parameters in the reference's affine_param order: translocation[3] (mm),
    rotation[3] (rad), scaling[3], affine (shear)[3] (numerical/transformation.hpp:428-438)."""
    p = np.zeros(12, np.float32)
    p[0:3] = rng.uniform(-trans_vox, trans_vox, 3) * np.asarray(vs, np.float32)
    p[3:6] = np.deg2rad(rng.uniform(-rot_deg, rot_deg, 3))
    p[6:9] = rng.uniform(scale[0], scale[1], 3)
    p[9:12] = rng.uniform(-shear, shear, 3)
    return p


def apply_matrix(vol: np.ndarray, T: np.ndarray, out_shape) -> np.ndarray:
    """out(x) = trilinear(vol, sr*x + shift) for a reference transformation_matrix T
    (T[0:9] row-major sr acting on (x, y, z), T[9:12] shift); 0 outside."""
    z, y, x = _grid(out_shape)
    sr = np.asarray(T[:9], np.float32).reshape(3, 3)
    sh = np.asarray(T[9:12], np.float32)
    px = sr[0, 0] * x + sr[0, 1] * y + sr[0, 2] * z + sh[0]
    py = sr[1, 0] * x + sr[1, 1] * y + sr[1, 2] * z + sh[1]
    pz = sr[2, 0] * x + sr[2, 1] * y + sr[2, 2] * z + sh[2]
    return ndimage.map_coordinates(vol, np.stack([pz, py, px]), order=1, mode="constant",
                                   cval=0.0).astype(np.float32)


def rician(img: np.ndarray, rng: np.random.Generator, frac=0.02) -> np.ndarray:
    s = frac * float(img.max())
    a = img + rng.normal(0, s, img.shape).astype(np.float32)
    b = rng.normal(0, s, img.shape).astype(np.float32)
    return np.sqrt(a * a + b * b).astype(np.float32)


def normalize_to_u8(img: np.ndarray, upper: float = 255.999) -> np.ndarray:
    """(v - min) * (upper / (max - min)) in float32, truncated to uint8."""
    f = np.ascontiguousarray(img, np.float32)
    mn = np.float32(f.min())
    mx = np.float32(f.max())
    rng_ = np.float32(mx - mn)
    if rng_ == 0:
        return np.zeros(f.shape, np.uint8)
    scale = np.float32(np.float32(upper) / rng_)
    return ((f - mn) * scale).astype(np.uint8)


def cdm_pair(shape=(64, 64, 64), seed=None, rng=None):
    """Template/moving float32 pair of the plain CDM workload: blob template; moving =
    template warped by a smooth field (sigma 6, max 3 voxels) plus fresh N(0, 0.01)."""
    rng = rng or np.random.default_rng(seed if seed is not None else seed_for(1))
    tmpl = blob_volume(shape, rng)
    d = smooth_field(shape, rng, 6.0, 3.0)
    mov = warp(tmpl, d) + rng.normal(0, 0.01, tmpl.shape).astype(np.float32)
    return tmpl.astype(np.float32), mov.astype(np.float32), d


def affine_pair(shape=(182, 218, 182), seed=None, rng=None, vs=(1.0, 1.0, 1.0)):
    """Template/moving uint16 pair of the affine workload: class phantom; moving = the
    template under a random affine, resampled trilinearly, with 2% Rician noise.
    Returns (template_u16, moving_u16, true_params)."""
    rng = rng or np.random.default_rng(seed if seed is not None else seed_for(2))
    tmpl = class_phantom(shape, rng)
    p = random_affine(rng, vs=vs)
    T = affine_matrix_f32(p, shape, vs, shape, vs)
    mov = rician(apply_matrix(tmpl, T, shape), rng)
    return (np.clip(tmpl, 0, 4095).astype(np.uint16), np.clip(mov, 0, 4095).astype(np.uint16), p)


def affine_matrix_f32(p, from_shape, from_vs, to_shape, to_vs) -> np.ndarray:
    """The reference's transformation_matrix(affine_param, ...) composition
    (numerical/transformation.hpp:636-675) evaluated in numpy float32; used only to
    make synthetic data (the product path computes it in its own host code)."""
    p = np.asarray(p, np.float32)
    f32 = np.float32
    sx, cx = np.sin(p[3], dtype=f32), np.cos(p[3], dtype=f32)
    sy, cy = np.sin(p[4], dtype=f32), np.cos(p[4], dtype=f32)
    sz, cz = np.sin(p[5], dtype=f32), np.cos(p[5], dtype=f32)
    m = np.array([cy * cz, cy * sz, -sy,
                  -cx * sz + sx * cz * sy, cx * cz + sx * sz * sy, sx * cy,
                  sx * sz + cx * cz * sy, -sx * cz + cx * sz * sy, cx * cy], f32)
    m = m.reshape(3, 3) * p[6:9, None]
    a = p[9:12]
    m[0] += m[1] * a[0] + m[2] * a[1]
    m[1] += m[2] * a[2]
    fz, fy, fx = from_shape
    t = np.array([fx, fy, fz], f32) * f32(-0.5) * np.asarray(from_vs, f32) + p[0:3]
    sh = m @ t
    m = m * np.asarray(from_vs, f32)[None, :]
    tvs = np.asarray(to_vs, f32)
    m = m / tvs[:, None]
    sh = sh / tvs
    tz, ty, tx = to_shape
    sh = sh + np.array([tx, ty, tz], f32) * f32(0.5)
    return np.concatenate([m.reshape(-1), sh]).astype(np.float32)


def cdm_workload_pair(shape=(182, 218, 182), seed=None):
    """Template/moving float32 pair of the nonlinear workloads: a class phantom and the
    same phantom warped by a smooth field (sigma 6, max 4 voxels) with 2% Rician noise.
    At 182x218x182 with min_dimension 32 its CDM iterates the 23, 46 and 91 levels and
    the field moves (max |d| about 2 voxels)."""
    rng = np.random.default_rng(seed if seed is not None else seed_for(4))
    t = class_phantom(shape, rng)
    d = smooth_field(shape, rng, 6.0, 4.0)
    m = rician(warp(t, d), rng)
    return t.astype(np.float32), m.astype(np.float32)


def cdm_class_pair(shape=(64, 64, 64), seed=None):
    """Config-1-shaped CDM pair whose field moves at the default cdm_param: a class
    phantom and the same phantom warped by a smooth field (sigma 6, max 3 voxels) with
    2% Rician noise, float32.  (The blob pair of cdm_pair has smooth, nearly linear 5^3
    windows everywhere, and the reference's CDM never improves on its first iteration
    there: it returns the zero field.)"""
    rng = np.random.default_rng(seed if seed is not None else seed_for(1, 100))
    t = class_phantom(shape, rng)
    d = smooth_field(shape, rng, 6.0, 3.0)
    m = rician(warp(t, d), rng)
    return t.astype(np.float32), m.astype(np.float32)
