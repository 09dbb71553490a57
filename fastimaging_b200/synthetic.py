"""Seeded synthetic snapshots with the shapes of the benchmark workloads.

Visibilities of a point-source sky follow the reference's model
(src/stp/visibility/visibility.cpp:15-28):
    vis = flux * n * exp(+2 pi i (u l + v m + w (n - 1))),  n = sqrt(1 - l^2 - m^2)
plus complex Gaussian noise; extended sources are elliptical Gaussians.
No public dataset is involved: every array is generated from a fixed seed.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def arcsec_to_rad(v):
    return (v / 3600.0) * (math.pi / 180.0)


@dataclass
class Snapshot:
    vis: np.ndarray      # (n,) complex128 or complex64
    weights: np.ndarray  # (n,) float64
    uvw: np.ndarray      # (n, 3) float64, Fortran order (u, v, w columns)
    image_size: int
    cell_size: float     # arcsec
    sources: np.ndarray  # (k, 3): l, m, flux


def _uv_disk(rng, n, radius):
    r = radius * np.sqrt(rng.random(n))
    t = 2 * math.pi * rng.random(n)
    return r * np.cos(t), r * np.sin(t)


def _uv_gauss(rng, n, radius, sigma_frac):
    u = np.empty(0)
    v = np.empty(0)
    while u.size < n:
        k = int((n - u.size) * 1.2) + 16
        a = rng.normal(0.0, sigma_frac * radius, size=k)
        b = rng.normal(0.0, sigma_frac * radius, size=k)
        keep = a * a + b * b < radius * radius
        u = np.concatenate([u, a[keep]])
        v = np.concatenate([v, b[keep]])
    return u[:n], v[:n]


def point_source_vis(u, v, w, sources, chunk=1 << 20):
    """sum_k flux_k n_k exp(2 pi i (u l + v m + w (n-1)))."""
    out = np.zeros(u.size, dtype=np.complex128)
    for s in range(0, u.size, chunk):
        e = min(u.size, s + chunk)
        uu, vv, ww = u[s:e], v[s:e], w[s:e]
        acc = np.zeros(e - s, dtype=np.complex128)
        for l, m, f in sources:
            nn = math.sqrt(1.0 - l * l - m * m)
            acc += f * nn * np.exp(2j * math.pi * (uu * l + vv * m + ww * (nn - 1.0)))
        out[s:e] = acc
    return out


def gaussian_source_vis(u, v, l, m, flux, sig_u, sig_v, pa):
    """Elliptical Gaussian (pixel widths already converted to uv widths)."""
    cu, su = math.cos(pa), math.sin(pa)
    up = u * cu + v * su
    vp = -u * su + v * cu
    amp = flux * np.exp(-2 * math.pi ** 2 * (sig_u ** 2 * up ** 2 + sig_v ** 2 * vp ** 2))
    return amp * np.exp(2j * math.pi * (u * l + v * m))


def make_snapshot(seed, n_vis, image_size, cell_arcsec=1.0, n_src=5, flux=(1.0, 10.0), log_flux=False,
                  noise_sigma=0.1, uv_frac=0.9, w_range=(0.0, 0.0), density="disk", gauss_sigma=0.25,
                  n_extended=0, ext_sigma_px=(2.0, 6.0), vis_dtype=np.complex128, src_frac=0.8):
    """One snapshot.  uv extent: radius uv_frac * (N/2) * du with du = 1/(N cell)."""
    rng = np.random.default_rng(seed)
    cell = arcsec_to_rad(cell_arcsec)
    du = 1.0 / (image_size * cell)
    radius = uv_frac * (image_size / 2) * du
    if density == "disk":
        u, v = _uv_disk(rng, n_vis, radius)
    else:
        u, v = _uv_gauss(rng, n_vis, radius, gauss_sigma)
    if w_range[1] > w_range[0]:
        w = rng.uniform(w_range[0], w_range[1], size=n_vis)
    else:
        w = np.zeros(n_vis)
    half = int(image_size * src_frac / 2)
    px = rng.integers(-half, half, size=(n_src, 2))
    if log_flux:
        f = np.exp(rng.uniform(math.log(flux[0]), math.log(flux[1]), size=n_src))
    else:
        f = rng.uniform(flux[0], flux[1], size=n_src)
    src = np.column_stack([px[:, 0] * cell, px[:, 1] * cell, f])
    vis = point_source_vis(u, v, w, src)
    for _ in range(n_extended):
        ex = rng.integers(-half, half, size=2)
        sx, sy = rng.uniform(*ext_sigma_px, size=2)
        fx = rng.uniform(flux[0], flux[1])
        vis += gaussian_source_vis(u, v, ex[0] * cell, ex[1] * cell, fx * 2 * math.pi * sx * sy, sx * cell, sy * cell,
                                   rng.uniform(0, math.pi))
    if noise_sigma > 0:
        vis += noise_sigma * (rng.normal(size=n_vis) + 1j * rng.normal(size=n_vis))
    uvw = np.asfortranarray(np.column_stack([u, v, w]))
    return Snapshot(vis.astype(vis_dtype), np.ones(n_vis), uvw, image_size, cell_arcsec, src)


# Benchmark workloads (sizes of the reference's headline configurations).
def config1(seed=1):
    """Plain imager: 2048^2, 1 arcsec cells, 100k vis, w = 0, 5 sources 1-10 Jy, noise 0.1 Jy;
    Gaussian-Sinc S=3 os=8."""
    return make_snapshot(seed, 100_000, 2048, 1.0, n_src=5, flux=(1.0, 10.0), noise_sigma=0.1)


def config2(seed=2):
    """W-projection imager: 4096^2, 1M vis, w ~ U[-2000, 2000] lambda, 20 sources log-uniform 0.1-10 Jy,
    noise 0.05 Jy; 32 planes, W-kernel support <= 16, os 8."""
    return make_snapshot(seed, 1_000_000, 4096, 1.0, n_src=20, flux=(0.1, 10.0), log_flux=True, noise_sigma=0.05,
                         w_range=(-2000.0, 2000.0))


def config3(seed=3):
    """Precision study: 8192^2, 4M complex64 vis, uv Gaussian-concentrated (sigma 0.25 of the uv radius);
    PSWF S=4 os=16."""
    return make_snapshot(seed, 4_000_000, 8192, 1.0, n_src=20, flux=(0.1, 10.0), log_flux=True, noise_sigma=0.05,
                         density="gauss", gauss_sigma=0.25, vis_dtype=np.complex64)


CONFIG2_IMAGER = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, gridding_correction=True,
                      analytic_gcf=False, num_wplanes=32, max_wpconv_support=16, undersampling_opt=1,
                      kernel_trunc_perc=1.0)
CONFIG1_IMAGER = dict(kernel_func=4, kernel_support=3, kernel_exact=False, oversampling=8, gridding_correction=True,
                      analytic_gcf=False)
CONFIG3_IMAGER = dict(kernel_func=5, kernel_support=4, kernel_exact=False, oversampling=16, gridding_correction=True,
                      analytic_gcf=True)


def config4(seed=4, n_snapshots=64, n_src=5):
    """Batched snapshots: visibility counts log-uniform in 50k-2M, image sizes from {1024, 2048, 4096, 8192},
    w ~ U[-w_max, w_max] with w_max ~ U[0, 2000] lambda per snapshot, kernels alternating GaussianSinc / PSWF by a
    seeded coin; W-projection with 16 planes, W-kernel support <= 16 (1 % truncation), os 8.
    Returns [(Snapshot, imager keywords)]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_snapshots):
        n_vis = int(round(math.exp(rng.uniform(math.log(5e4), math.log(2e6)))))
        size = int(rng.choice([1024, 2048, 4096, 8192]))
        w_max = float(rng.uniform(0.0, 2000.0))
        kf = 4 if rng.random() < 0.5 else 5
        s = make_snapshot(seed * 1000 + i, n_vis, size, 1.0, n_src=n_src, flux=(0.5, 10.0), noise_sigma=0.05,
                          w_range=(-w_max, w_max))
        kw = dict(image_size=size, cell_size=1.0, kernel_func=kf, kernel_support=3, kernel_exact=False,
                  oversampling=8, gridding_correction=True, analytic_gcf=False, num_wplanes=16,
                  max_wpconv_support=16, undersampling_opt=1, kernel_trunc_perc=1.0)
        out.append((s, kw))
    return out


def config5_pool(seed=5, n_templates=12):
    """Request templates of the serving workload: snapshot sizes drawn as in config4 (visibility counts
    log-uniform 50k-2M, image sizes from {1024, 2048, 4096, 8192}, W-projection 16 planes), each sky with
    50 point sources plus 5 extended elliptical Gaussians (sigma 2-6 px).  Requests sample this pool.
    Returns [(Snapshot, imager keywords)]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_templates):
        n_vis = int(round(math.exp(rng.uniform(math.log(5e4), math.log(2e6)))))
        size = int(rng.choice([1024, 2048, 4096, 8192]))
        w_max = float(rng.uniform(0.0, 2000.0))
        kf = 4 if rng.random() < 0.5 else 5
        s = make_snapshot(seed * 1000 + i, n_vis, size, 1.0, n_src=50, flux=(0.5, 10.0), noise_sigma=0.05,
                          w_range=(-w_max, w_max), n_extended=5)
        kw = dict(image_size=size, cell_size=1.0, kernel_func=kf, kernel_support=3, kernel_exact=False,
                  oversampling=8, gridding_correction=True, analytic_gcf=False, num_wplanes=16,
                  max_wpconv_support=16, undersampling_opt=1, kernel_trunc_perc=1.0)
        out.append((s, kw))
    return out
