"""Seeded synthetic parallel-beam sinograms for the gridrec path.

The reference ships no datasets; these analytic phantoms stand in for its
inputs with the sizes and value ranges of the configured workloads:

* ``shepp_logan_sinogram`` -- the modified (Toft) Shepp-Logan phantom, ten
  ellipses with the usual intensities, scaled so the largest line integral is
  2.0, then Poisson counts at 1e4 incident photons and ``-log``.
* ``random_ellipse_sinogram`` -- 5..20 random ellipses per slice drawn from
  ``numpy.random.default_rng(seed)`` (semi-axes U[0.02, 0.4], densities
  U[-0.2, 1.0], rotations U[0, pi), centres uniform in the disk of radius 0.5).
* ``raw_counts`` -- uint16 detector counts ``flat * exp(-p) + dark`` with
  Poisson noise and per-pixel flats (mean 40000 +-5 %) and darks (mean 100),
  the input of the fused flat/dark + -log load.

Geometry: detector pixel k sits at t = k - center (pixels); a projection at
angle theta is the line integral along x*cos(theta) + y*sin(theta) = t, the
convention under which gridrec's Fourier-slice mapping (gridrec/GPU/gridrec.cu:
540-541, U = scale*j*cos + M/2) holds.  Phantom coordinates are in units of the
half detector width, so the unit disk spans the detector.

Line integrals are evaluated in float64 with numpy, or on a CUDA device with
torch (``device=`` argument) for large batches; the ellipse parameters come from
numpy in both cases, so only the Poisson noise draw differs between backends.
"""
from __future__ import annotations

import math

import numpy as np

# Modified Shepp-Logan (Toft): intensity, semi-axis a, semi-axis b, x0, y0, phi(deg)
_SHEPP_LOGAN_TOFT = (
    (1.0, 0.69, 0.92, 0.0, 0.0, 0.0),
    (-0.8, 0.6624, 0.874, 0.0, -0.0184, 0.0),
    (-0.2, 0.11, 0.31, 0.22, 0.0, -18.0),
    (-0.2, 0.16, 0.41, -0.22, 0.0, 18.0),
    (0.1, 0.21, 0.25, 0.0, 0.35, 0.0),
    (0.1, 0.046, 0.046, 0.0, 0.1, 0.0),
    (0.1, 0.046, 0.046, 0.0, -0.1, 0.0),
    (0.1, 0.046, 0.023, -0.08, -0.605, 0.0),
    (0.1, 0.023, 0.023, 0.0, -0.606, 0.0),
    (0.1, 0.023, 0.046, 0.06, -0.605, 0.0),
)


def shepp_logan_ellipses() -> np.ndarray:
    """Rows (rho, a, b, x0, y0, phi_rad) of the modified Shepp-Logan phantom."""
    e = np.array(_SHEPP_LOGAN_TOFT, dtype=np.float64)
    e[:, 5] = np.deg2rad(e[:, 5])
    return e


def random_ellipses(seed: int) -> np.ndarray:
    """5..20 random ellipses (rho, a, b, x0, y0, phi) from default_rng(seed)."""
    rng = np.random.default_rng(seed)
    k = int(rng.integers(5, 21))
    a = rng.uniform(0.02, 0.4, k)
    b = rng.uniform(0.02, 0.4, k)
    rho = rng.uniform(-0.2, 1.0, k)
    r = 0.5 * np.sqrt(rng.uniform(0.0, 1.0, k))
    t = rng.uniform(0.0, 2.0 * np.pi, k)
    phi = rng.uniform(0.0, np.pi, k)
    return np.stack([rho, a, b, r * np.cos(t), r * np.sin(t), phi], axis=1)


def angles_deg(n_ang: int) -> np.ndarray:
    """n_ang angles evenly spaced on [0, 180) degrees: theta_i = 180 i / n_ang."""
    return (180.0 * np.arange(n_ang, dtype=np.float64) / n_ang).astype(np.float32)


def line_integrals(ellipses: np.ndarray, n_det: int, theta_deg: np.ndarray,
                   center: float, device=None):
    """Exact line integrals p[angle, k] of a sum of ellipses (float64).

    With ``device`` set (a torch CUDA device), the evaluation runs on that
    device and a float64 torch tensor is returned; otherwise a numpy array.
    """
    half = n_det / 2.0
    th = np.deg2rad(np.asarray(theta_deg, dtype=np.float64))
    if device is not None:
        import torch
        t = (torch.arange(n_det, dtype=torch.float64, device=device) - center) / half
        thd = torch.as_tensor(th, device=device)
        c, s = torch.cos(thd)[:, None], torch.sin(thd)[:, None]
        p = torch.zeros((len(th), n_det), dtype=torch.float64, device=device)
        for rho, a, b, x0, y0, phi in ellipses.tolist():
            sh = t[None, :] - (x0 * c + y0 * s)
            cp = torch.cos(thd - phi)[:, None]
            sp = torch.sin(thd - phi)[:, None]
            a2 = (a * cp) ** 2 + (b * sp) ** 2
            d = a2 - sh * sh
            p += torch.where(d > 0, 2.0 * rho * a * b * torch.sqrt(d.clamp_min(0)) / a2,
                             torch.zeros_like(d))
        return p * half  # lengths in pixels of the detector grid
    t = (np.arange(n_det, dtype=np.float64) - center) / half
    c, s = np.cos(th)[:, None], np.sin(th)[:, None]
    p = np.zeros((len(th), n_det), dtype=np.float64)
    for rho, a, b, x0, y0, phi in ellipses:
        sh = t[None, :] - (x0 * c + y0 * s)
        cp = np.cos(th - phi)[:, None]
        sp = np.sin(th - phi)[:, None]
        a2 = (a * cp) ** 2 + (b * sp) ** 2
        d = a2 - sh * sh
        p += np.where(d > 0, 2.0 * rho * a * b * np.sqrt(np.clip(d, 0, None)) / a2, 0.0)
    return p * half


def poisson_log(p, photons: float = 1e4, seed: int = 0):
    """-log(max(Poisson(photons*exp(-p)), 1)/photons), float32 (numpy or torch)."""
    if isinstance(p, np.ndarray):
        rng = np.random.default_rng(seed)
        counts = rng.poisson(photons * np.exp(-p)).astype(np.float64)
        return (-np.log(np.maximum(counts, 1.0) / photons)).astype(np.float32)
    import torch
    g = torch.Generator(device=p.device)
    g.manual_seed(int(seed))
    counts = torch.poisson(photons * torch.exp(-p), generator=g)
    return (-torch.log(counts.clamp_min(1.0) / photons)).to(torch.float32)


def shepp_logan_sinogram(n_det: int = 512, n_ang: int = 360, center: float = 256.3,
                         noise_seed: int = 0, photons: float = 1e4, max_atten: float = 2.0):
    """Noisy -log sinogram (n_ang x n_det float32) of the modified Shepp-Logan phantom."""
    th = angles_deg(n_ang)
    p = line_integrals(shepp_logan_ellipses(), n_det, th, center)
    p *= max_atten / p.max()
    return poisson_log(p, photons, noise_seed)


def random_ellipse_sinogram(seed: int, n_det: int = 2048, n_ang: int = 1500,
                            center: float | None = None, photons: float = 1e4,
                            device=None):
    """Noisy -log sinogram of the random-ellipse slice `seed`; returns (sino, center).

    The centre defaults to n_det/2 + U[-2, 2] drawn after the ellipses from the
    same generator (so it depends only on the seed).
    """
    ell = random_ellipses(seed)
    if center is None:
        rng = np.random.default_rng(seed + 1_000_003)
        center = n_det / 2.0 + float(rng.uniform(-2.0, 2.0))
    p = line_integrals(ell, n_det, angles_deg(n_ang), center, device=device)
    # densities are per unit half-width; keep attenuation O(1) at any n_det
    p = p / (n_det / 2.0)
    return poisson_log(p, photons, seed), center


def random_ellipse_raw(seed: int, n_det: int, n_ang: int, device, flat_mean: float = 40000.0,
                       flat_spread: float = 0.05, dark_mean: float = 100.0):
    """Raw uint16 counts of the random-ellipse slice `seed` on a torch device:
    Poisson(flat * exp(-p)) + dark, with this slice's own flat (flat_mean
    +-flat_spread per pixel) and dark (dark_mean + N(0, 2)) rows.

    Returns (raw as an int16 tensor view of the uint16 bits, flat, dark, center)."""
    import torch
    ell = random_ellipses(seed)
    rng = np.random.default_rng(seed + 1_000_003)
    center = n_det / 2.0 + float(rng.uniform(-2.0, 2.0))
    p = line_integrals(ell, n_det, angles_deg(n_ang), center, device=device) / (n_det / 2.0)
    g = torch.Generator(device=device)
    g.manual_seed(int(seed) + 7)
    u = torch.rand(n_det, generator=g, device=device, dtype=torch.float64)
    flat = flat_mean * (1.0 + flat_spread * (2.0 * u - 1.0))
    dark = dark_mean + 2.0 * torch.randn(n_det, generator=g, device=device, dtype=torch.float64)
    counts = torch.poisson(flat[None, :] * torch.exp(-p), generator=g) + torch.round(dark)[None, :]
    raw = counts.clamp(0, 65535).to(torch.int32)
    raw = torch.where(raw > 32767, raw - 65536, raw).to(torch.int16)  # uint16 bits
    return raw, flat.to(torch.float32), dark.to(torch.float32), center


def raw_counts(p, seed: int = 0, flat_mean: float = 40000.0, flat_spread: float = 0.05,
               dark_mean: float = 100.0):
    """uint16 counts Poisson(flat*exp(-p)) + dark, plus the flat and dark rows.

    Returns (raw[n_ang, n_det] uint16, flat[n_det] float32, dark[n_det] float32).
    """
    rng = np.random.default_rng(seed)
    n_det = p.shape[-1]
    flat = flat_mean * (1.0 + flat_spread * rng.uniform(-1.0, 1.0, n_det))
    dark = dark_mean + rng.normal(0.0, 2.0, n_det)
    raw = rng.poisson(flat[None, :] * np.exp(-p)) + np.round(dark)[None, :]
    raw = np.clip(raw, 0, 65535).astype(np.uint16)
    return raw, flat.astype(np.float32), dark.astype(np.float32)


def psnr(img: np.ndarray, ref: np.ndarray) -> float:
    """Peak signal-to-noise ratio of img against ref (peak = max |ref|)."""
    mse = float(np.mean((img.astype(np.float64) - ref) ** 2))
    peak = float(np.max(np.abs(ref)))
    return math.inf if mse == 0 else 10.0 * math.log10(peak * peak / mse)


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b||_2 / ||b||_2 in float64."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
