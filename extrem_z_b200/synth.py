"""Seeded synthetic scalar fields and their SZ3-style decompressed copies.

The reference is exercised on real simulation outputs (QMCPack, NYX, S3D) that
are not available here.  These fields stand in for them with the same shapes,
value ranges and tie structure:

* ``f`` (x fastest, index ``x + y*W + z*W*H``) is a sum of ``G`` anisotropic
  Gaussians ``a * exp(-1/2 * sum_d ((x_d - c_d) / s_d)^2)`` with centres
  uniform in the box, ``s_d`` uniform in [2, 10] voxels and ``a`` uniform in
  [-1, 1], plus power-law noise whose power spectrum is ``k^-alpha``
  (``k = 0`` removed) rescaled to an RMS of 0.05.
* The random stream is ``numpy.random.default_rng(seed)`` and is drawn in the
  order: all centres, all widths, all amplitudes, then the noise.
* ``decp`` emulates SZ3's linear quantiser: ``round(f / (2 eb)) * 2 eb`` in
  float64, cast to the field dtype, with ``eb = rel * (max f - min f)``.  If the
  cast breaks ``|f - decp| <= eb`` the value is stepped one ulp toward ``f``.
  The quantiser creates plateaus, so ties are resolved by vertex index.

The reference computes its absolute bound the same way
(``src/ExtreM_cuda.cu:229-232``: ``bound = (maxValue - minValue) * er``), so the
returned ``eb`` is the corrector's ``bound``.
"""

from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Field:
    """One correction job: original field, decompressed copy and bound."""

    f: np.ndarray          # original values, shape (D, H, W), dtype T
    decp: np.ndarray       # decompressed values, same shape and dtype
    eb: float              # absolute error bound (float64)
    seed: int
    rel: float

    @property
    def shape_whd(self):
        d, h, w = self.f.shape
        return w, h, d


def gaussian_field(w: int, h: int, d: int, n_gauss: int, seed: int,
                   alpha: float = 2.0, noise_rms: float = 0.05) -> np.ndarray:
    """Float64 field of shape (d, h, w): Gaussian sum plus power-law noise."""
    rng = np.random.default_rng(seed)
    dims = np.array([w, h, d], dtype=np.float64)
    centres = rng.uniform(0.0, 1.0, size=(n_gauss, 3)) * dims
    sigmas = rng.uniform(2.0, 10.0, size=(n_gauss, 3))
    amps = rng.uniform(-1.0, 1.0, size=n_gauss)

    # Each Gaussian is separable, so the sum is a rank-G contraction of three
    # 1-D profile matrices; evaluate it slice by slice as a matrix product.
    xs = np.arange(w, dtype=np.float64)
    ys = np.arange(h, dtype=np.float64)
    zs = np.arange(d, dtype=np.float64)
    gx = np.exp(-0.5 * ((xs[None, :] - centres[:, 0:1]) / sigmas[:, 0:1]) ** 2)
    gy = np.exp(-0.5 * ((ys[None, :] - centres[:, 1:2]) / sigmas[:, 1:2]) ** 2)
    gz = np.exp(-0.5 * ((zs[None, :] - centres[:, 2:3]) / sigmas[:, 2:3]) ** 2)
    out = np.empty((d, h, w), dtype=np.float64)
    gy_t = np.ascontiguousarray(gy.T)
    for z in range(d):
        wz = amps * gz[:, z]
        out[z] = (gy_t * wz[None, :]) @ gx

    noise = rng.standard_normal((d, h, w))
    spec = np.fft.rfftn(noise)
    fz = np.fft.fftfreq(d)[:, None, None]
    fy = np.fft.fftfreq(h)[None, :, None]
    fx = np.fft.rfftfreq(w)[None, None, :]
    k = np.sqrt(fx * fx + fy * fy + fz * fz)
    amp = np.zeros_like(k)
    nz = k > 0
    amp[nz] = k[nz] ** (-alpha / 2.0)
    spec *= amp
    noise = np.fft.irfftn(spec, s=(d, h, w), axes=(0, 1, 2))
    rms = math.sqrt(float(np.mean(noise * noise)))
    if rms > 0:
        noise *= noise_rms / rms
    out += noise
    return out


def quantise(f: np.ndarray, rel: float):
    """SZ3 linear-quantiser stand-in.  Returns (decp, eb)."""
    f64 = f.astype(np.float64)
    eb = float(rel) * (float(f64.max()) - float(f64.min()))
    if eb <= 0.0:
        return f.copy(), eb
    q = np.round(f64 / (2.0 * eb)) * (2.0 * eb)
    decp = q.astype(f.dtype)
    bad = np.abs(f64 - decp.astype(np.float64)) > eb
    if np.any(bad):
        decp[bad] = np.nextafter(decp[bad], f[bad])
    return decp, eb


def make_field(w: int, h: int, d: int, *, n_gauss: int, seed: int, rel: float,
               dtype=np.float64, alpha: float = 2.0) -> Field:
    """Original field cast to ``dtype`` plus its quantised copy."""
    f = gaussian_field(w, h, d, n_gauss, seed, alpha=alpha).astype(dtype)
    decp, eb = quantise(f, rel)
    return Field(f=f, decp=decp, eb=eb, seed=seed, rel=rel)


# ---------------------------------------------------------------------------
# Named workloads (shapes, Gaussian counts, seeds and bounds of the benchmark
# configurations).
# ---------------------------------------------------------------------------

def plain_64(dtype=np.float32) -> Field:
    """64^3, 64 Gaussians, seed 0, rel 1e-3, k^-2 noise."""
    return make_field(64, 64, 64, n_gauss=64, seed=0, rel=1e-3, dtype=dtype)


def plain_256(dtype=np.float64) -> Field:
    """256^3, 512 Gaussians, seed 1, rel 1e-4, k^-2 noise."""
    return make_field(256, 256, 256, n_gauss=512, seed=1, rel=1e-4, dtype=dtype)


def plain_512() -> Field:
    """512^3 float64, 4096 Gaussians, seed 2, rel 1e-5, k^-5/3 noise."""
    return make_field(512, 512, 512, n_gauss=4096, seed=2, rel=1e-5,
                      dtype=np.float64, alpha=5.0 / 3.0)


def mixed_batch_specs(n_fields: int = 64, first_seed: int = 100,
                      slice_fraction: float = 0.25):
    """Specs of the mixed batch: uneven shapes, dtypes and bounds.

    Edge lengths are log-uniform in [32, 192]; a quarter of the fields are 2-D
    slices (D = 1); dtype float32/float64 50/50; rel log-uniform in
    [1e-5, 1e-2]; G = max(8, round(512 * N / 256^3)).  Each field's parameters
    come from its own seed.
    """
    specs = []
    for i in range(n_fields):
        seed = first_seed + i
        r = np.random.default_rng(seed ^ 0x5EED)
        edges = np.exp(r.uniform(math.log(32), math.log(192), size=3)).round().astype(int)
        w, h, d = int(edges[0]), int(edges[1]), int(edges[2])
        if r.uniform() < slice_fraction:
            d = 1
        dtype = np.float32 if r.uniform() < 0.5 else np.float64
        rel = float(math.exp(r.uniform(math.log(1e-5), math.log(1e-2))))
        n = w * h * d
        g = max(8, int(round(512 * n / 256 ** 3)))
        specs.append(dict(w=w, h=h, d=d, n_gauss=g, seed=seed, rel=rel, dtype=dtype))
    return specs


def serving_request_spec(request_id: int):
    """Spec of one serving request: voxels log-uniform in [32^3, 384^3]."""
    seed = 10000 + request_id
    r = np.random.default_rng(seed ^ 0x5EED)
    n = math.exp(r.uniform(math.log(32 ** 3), math.log(384 ** 3)))
    edge = n ** (1.0 / 3.0)
    jit = np.exp(r.uniform(-0.15, 0.15, size=3))
    w, h, d = (max(8, int(round(edge * j))) for j in jit)
    dtype = np.float32 if r.uniform() < 0.5 else np.float64
    rel = float(math.exp(r.uniform(math.log(1e-5), math.log(1e-2))))
    g = max(8, int(round(512 * w * h * d / 256 ** 3)))
    return dict(w=w, h=h, d=d, n_gauss=g, seed=seed, rel=rel, dtype=dtype)


def make_field_device(w: int, h: int, d: int, *, n_gauss: int, seed: int, rel: float,
                      dtype=np.float64, alpha: float = 2.0, noise_rms: float = 0.05,
                      device="cuda"):
    """The generator of ``make_field`` evaluated on a CUDA device with torch.

    Centres, widths and amplitudes come from the same numpy stream as
    ``gaussian_field``; the white noise comes from torch's CUDA generator
    seeded with ``seed``, so values differ from ``make_field`` while the
    distribution is the same.  For request streams too large to generate on
    the host in a benchmark's time.  Returns (f, decp, eb) with f and decp
    CUDA tensors of shape (d, h, w).
    """
    import torch
    rng = np.random.default_rng(seed)
    dims = np.array([w, h, d], dtype=np.float64)
    centres = rng.uniform(0.0, 1.0, size=(n_gauss, 3)) * dims
    sigmas = rng.uniform(2.0, 10.0, size=(n_gauss, 3))
    amps = rng.uniform(-1.0, 1.0, size=n_gauss)
    dev = torch.device(device)
    f64 = torch.float64
    c = torch.as_tensor(centres, dtype=f64, device=dev)
    s = torch.as_tensor(sigmas, dtype=f64, device=dev)
    a = torch.as_tensor(amps, dtype=f64, device=dev)

    def profile(n, axis):
        t = torch.arange(n, dtype=f64, device=dev)
        return torch.exp(-0.5 * ((t[None, :] - c[:, axis:axis + 1]) / s[:, axis:axis + 1]) ** 2)

    gx, gy, gz = profile(w, 0), profile(h, 1), profile(d, 2)
    wz = (gz * a[:, None]).T.contiguous()           # (d, G)
    out = torch.empty((d, h, w), dtype=f64, device=dev)
    cy = max(1, min(h, (1 << 25) // max(1, n_gauss * w)))
    for y0 in range(0, h, cy):
        y1 = min(h, y0 + cy)
        kron = (gy[:, y0:y1, None] * gx[:, None, :]).reshape(n_gauss, -1)
        out[:, y0:y1, :] = (wz @ kron).reshape(d, y1 - y0, w)

    gen = torch.Generator(device=dev)
    gen.manual_seed(int(seed))
    noise = torch.randn((d, h, w), generator=gen, dtype=f64, device=dev)
    spec = torch.fft.rfftn(noise)
    fz = torch.fft.fftfreq(d, device=dev, dtype=f64)[:, None, None]
    fy = torch.fft.fftfreq(h, device=dev, dtype=f64)[None, :, None]
    fx = torch.fft.rfftfreq(w, device=dev, dtype=f64)[None, None, :]
    k = torch.sqrt(fx * fx + fy * fy + fz * fz)
    amp = torch.where(k > 0, k.clamp_min(1e-300) ** (-alpha / 2.0), torch.zeros_like(k))
    noise = torch.fft.irfftn(spec * amp, s=(d, h, w), dim=(0, 1, 2))
    rms = float(torch.sqrt(torch.mean(noise * noise)))
    if rms > 0:
        noise *= noise_rms / rms
    out += noise
    del noise, spec

    tdt = torch.float32 if np.dtype(dtype) == np.float32 else torch.float64
    f = out.to(tdt)
    fv = f.to(f64)
    eb = float(rel) * (float(fv.max()) - float(fv.min()))
    if eb <= 0.0:
        return f, f.clone(), eb
    q = torch.round(fv / (2.0 * eb)) * (2.0 * eb)
    decp = q.to(tdt)
    bad = (fv - decp.to(f64)).abs() > eb
    if bool(bad.any()):
        decp = torch.where(bad, torch.nextafter(decp, f), decp)
    return f, decp, eb
