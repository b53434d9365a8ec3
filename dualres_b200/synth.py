"""Seeded synthetic dual-resolution volumes.

No public dataset is involved: every volume is drawn from a seeded Gaussian
process, using the same circulant embedding that the sampler inverts. The
volumes follow the layout of the reference's NIfTI inputs:

* images are float32 arrays of shape ``(nz, ny, nx)`` in C order, so the flat
  index is ``x + nx * (y + ny * z)`` (the column-major ``ijk`` order of
  ``include/dualres/impl/nifti_manipulation.inl:335-360``);
* qforms are 4x4 row-major float32 matrices (``nifti_manipulation.h:34``);
* zero voxels carry no data.

The generated geometry keeps the kriging neighbourhood away from the image
border. The latent box sits inside a zero border at least ``ceil(radius /
voxel)`` wide, so the reference's flat-offset-only bounds check
(``kriging_matrix.h:263-266``) never wraps a row. Std-res voxel centres sit
half a high-res voxel from a grid point, so the truncation at
``kriging_matrix.h:255`` is never borderline.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Volume:
    """One dual-resolution problem in image form (what ``dualgpmf`` reads)."""

    highres: np.ndarray          # (nz, ny, nx) float32, 0 = no data
    qform_hr: np.ndarray         # (4, 4) float32 row-major
    stdres: np.ndarray | None    # (sz, sy, sx) float32 or None
    qform_sr: np.ndarray | None
    theta: tuple                 # (variance, bandwidth, exponent)
    radius: float                # kriging neighbourhood (mm)
    latent: np.ndarray = field(repr=False, default=None)  # true field on the high-res image grid
    name: str = ""
    hmask: np.ndarray | None = None
    omask: np.ndarray | None = None


def embedding_dims(g):
    """E_d = 2^ceil(log2(2 (g_d - 1))) (``MultiResParameters.h:191-206``)."""
    out = []
    for gd in g:
        if gd <= 1:
            raise ValueError("grid dimension must be > 1")
        t = 2 * (gd - 1)
        p = 1
        while p < t:
            p <<= 1
        out.append(p)
    return tuple(out)


def rbf(d, theta):
    v, b, e = theta
    return v * np.exp(-b * np.abs(d) ** e)


def circulant_spectrum(E, voxel_mm, theta):
    """FP64 eigenvalues of the wrapped covariance base on an E grid (shape (E2, E1, E0))."""
    axes = []
    for n, h in zip(E, voxel_mm):
        t = np.arange(n)
        axes.append(np.where(t <= n // 2, t, n - t) * h)
    ox, oy, oz = axes
    d = np.sqrt(oz[:, None, None] ** 2 + oy[None, :, None] ** 2 + ox[None, None, :] ** 2)
    return np.fft.fftn(rbf(d, theta)).real


def _latent_field(g, voxel_mm, theta, rng):
    """Stationary GP draw on a g grid via its circulant embedding (negative modes clipped)."""
    E = embedding_dims(g)
    lam = np.clip(circulant_spectrum(E, voxel_mm, theta), 0.0, None)
    N = lam.size
    w = rng.standard_normal(lam.shape) + 1j * rng.standard_normal(lam.shape)
    f = np.fft.fftn(np.sqrt(lam / N) * w)
    return f.real[: g[2], : g[1], : g[0]].astype(np.float64)


def _ellipsoid_mask(g, coverage, rng):
    c = np.array([(n - 1) / 2.0 for n in g])  # (x, y, z) centre
    z, y, x = np.meshgrid(np.arange(g[2]), np.arange(g[1]), np.arange(g[0]), indexing="ij")
    shape = 1.0 + 0.08 * rng.uniform(-1, 1, size=3)
    lo, hi = 0.3, 3.0
    for _ in range(60):
        s = 0.5 * (lo + hi)
        ax = shape * s * np.array(g) / 2.0
        r2 = ((x - c[0]) / ax[0]) ** 2 + ((y - c[1]) / ax[1]) ** 2 + ((z - c[2]) / ax[2]) ** 2
        frac = float((r2 <= 1.0).mean())
        if frac < coverage:
            lo = s
        else:
            hi = s
    m = r2 <= 1.0
    # keep the bounding box equal to the full latent grid
    for sl in [(0, slice(None), slice(None)), (-1, slice(None), slice(None))]:
        pass
    return m


def _smooth_noise_mask(g, coverage, rng, sigma_vox=3.0):
    z = rng.standard_normal((g[2], g[1], g[0]))
    k = np.fft.fftfreq
    fz, fy, fx = np.meshgrid(k(g[2]), k(g[1]), k(g[0]), indexing="ij")
    filt = np.exp(-2 * (math.pi * sigma_vox) ** 2 * (fx ** 2 + fy ** 2 + fz ** 2))
    s = np.fft.ifftn(np.fft.fftn(z) * filt).real
    thr = np.quantile(s, 1.0 - coverage)
    return s > thr


def make_volume(latent_dims=(32, 32, 32), voxel_mm=1.0, theta=(0.806, 0.132, 1.0),
                noise_hr=0.5, noise_sr=0.3, radius=6.9, mask="ellipsoid", coverage=0.60,
                seed=0, dual=True, name=""):
    """Build one synthetic volume.

    ``latent_dims`` is (nx, ny, nz) in high-res voxels. The std-res grid has
    twice the voxel size (2x2x2 block averages of the latent field plus noise),
    as in the reference's README example. A std voxel is kept iff its block
    centre lies inside the high-res mask.
    """
    rng = np.random.default_rng(seed)
    g = tuple(int(v) for v in latent_dims)
    h = float(voxel_mm)
    latent = _latent_field(g, (h, h, h), theta, rng)
    if mask == "ellipsoid":
        m = _ellipsoid_mask(g, coverage, rng)
    elif mask == "smooth":
        m = _smooth_noise_mask(g, coverage, rng)
    elif mask == "full":
        m = np.ones((g[2], g[1], g[0]), dtype=bool)
    else:
        raise ValueError(mask)
    # the mask's bounding box must span the latent grid so that g is as stated
    m[0, 0, 0] = m[-1, -1, -1] = True
    m[0, -1, -1] = m[-1, 0, 0] = True

    border = int(math.ceil(radius / h)) + 1
    border += border % 2  # keep the std grid aligned (2:1)
    nx, ny, nz = g[0] + 2 * border, g[1] + 2 * border, g[2] + 2 * border
    hr = np.zeros((nz, ny, nx), dtype=np.float32)
    lat_img = np.zeros((nz, ny, nx), dtype=np.float32)
    sl = (slice(border, border + g[2]), slice(border, border + g[1]), slice(border, border + g[0]))
    yh = latent + noise_hr * rng.standard_normal(latent.shape)
    yh = np.where(m, yh, 0.0).astype(np.float32)
    yh[(yh == 0) & m] = np.float32(1e-7)
    hr[sl] = yh
    lat_img[sl] = latent.astype(np.float32)
    Qh = np.array([[h, 0, 0, 0], [0, h, 0, 0], [0, 0, h, 0], [0, 0, 0, 1]], dtype=np.float32)

    sr = None
    Qs = None
    if dual:
        gs = tuple((n + 1) // 2 for n in g)
        bs = border // 2
        sx, sy, sz = nx // 2, ny // 2, nz // 2
        sr = np.zeros((sz, sy, sx), dtype=np.float32)
        pad = np.zeros((gs[2] * 2, gs[1] * 2, gs[0] * 2))
        pad[: g[2], : g[1], : g[0]] = latent
        blk = pad.reshape(gs[2], 2, gs[1], 2, gs[0], 2).mean(axis=(1, 3, 5))
        # block centre inside the high-res mask?
        mpad = np.zeros_like(pad, dtype=bool)
        mpad[: g[2], : g[1], : g[0]] = m
        keep = mpad[::2, ::2, ::2] & mpad[1::2, 1::2, 1::2]
        ys = blk + noise_sr * rng.standard_normal(blk.shape)
        ys = np.where(keep, ys, 0.0).astype(np.float32)
        ys[(ys == 0) & keep] = np.float32(1e-7)
        sr[bs: bs + gs[2], bs: bs + gs[1], bs: bs + gs[0]] = ys
        # std voxel s has its centre at high-res coordinate 2 s + 0.5
        Qs = np.array([[2 * h, 0, 0, 0.5 * h], [0, 2 * h, 0, 0.5 * h], [0, 0, 2 * h, 0.5 * h],
                       [0, 0, 0, 1]], dtype=np.float32)
    return Volume(highres=hr, qform_hr=Qh, stdres=sr, qform_sr=Qs, theta=tuple(float(t) for t in theta),
                  radius=float(radius), latent=lat_img, name=name)


def rotated(vol, quatern=(0.2895, -0.866, -0.2865), voxel=(1.8, 1.8, 2.3), qfac=-1.0, offset=(-90.0, 120.0, -40.0)):
    """The same images under a scanner-like geometry: the high-res qform becomes a
    rotation (unit quaternion b, c, d) of anisotropic voxels with qfac, and the
    std-res qform keeps its index map to the high-res grid (centre of std voxel s
    at high-res index 2 s + 0.5), so the kriging neighbourhoods are rotated
    balls of the new voxel geometry."""
    import dataclasses
    from .nifti import quatern_to_qform
    Qh = quatern_to_qform(*quatern, voxel, offset, qfac).astype(np.float64)
    Qs = None
    if vol.stdres is not None:
        M = np.array([[2, 0, 0, 0.5], [0, 2, 0, 0.5], [0, 0, 2, 0.5], [0, 0, 0, 1]], np.float64)
        Qs = (Qh @ M).astype(np.float32)
    return dataclasses.replace(vol, qform_hr=Qh.astype(np.float32), qform_sr=Qs, name=vol.name + "_rotated")


# The workloads named by the reference's benchmark configurations.
def config_c1(seed=1):
    """32^3 latent at 1 mm, RBF(0.806, 0.132, 1) -> 64^3 embedding, ellipsoid mask ~60%."""
    return make_volume((32, 32, 32), 1.0, (0.806, 0.132, 1.0), 0.5, 0.3, 6.9, "ellipsoid", 0.60, seed, name="c1")


def config_c2(seed=2):
    """64x64x48 latent at 1.5 mm, RBF(1.0, 0.4, 1.5) -> 128^3 embedding, smoothed-noise mask ~55%."""
    return make_volume((64, 64, 48), 1.5, (1.0, 0.4, 1.5), 0.7, 0.35, 6.9, "smooth", 0.55, seed, name="c2")


C4_SIZES = [(32, 32, 32), (48, 48, 40), (64, 64, 48), (80, 80, 64)]


def config_c4_volume(index, seed=4):
    """One volume of the uneven batch: size uniform over C4_SIZES, e ~ U[1,2], b ~ U[0.1,0.6], noise ~ U[0.3,1]."""
    rng = np.random.default_rng([seed, index])
    size = C4_SIZES[int(rng.integers(len(C4_SIZES)))]
    e = float(rng.uniform(1.0, 2.0))
    b = float(rng.uniform(0.1, 0.6))
    nh = float(rng.uniform(0.3, 1.0))
    ns = float(rng.uniform(0.3, 1.0))
    return make_volume(size, 1.0, (1.0, b, e), nh, ns, 6.9, "ellipsoid", 0.60, int(rng.integers(1 << 30)),
                       name=f"c4_{index}")


def small_volume(seed=7, dims=(10, 9, 7), radius=3.2, theta=(0.8, 0.3, 1.0), dual=True):
    """A small case for oracle-speed parity tests."""
    return make_volume(dims, 1.0, theta, 0.5, 0.3, radius, "ellipsoid", 0.7, seed, dual=dual, name="small")
