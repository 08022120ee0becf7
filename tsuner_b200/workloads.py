"""Seeded synthetic inputs with the shapes of the benchmark configurations.

No public dataset is involved: the reference's own example inputs are
NetCDF4/HDF5 files that cannot be read in this image, and the benchmark
configurations are defined synthetically.  Every generator is deterministic
(numpy integer arithmetic / PCG64 with a fixed seed), so tests, the oracle,
the reference build and the CUDA path all see bit-identical inputs.

State convention (GPU/main_TSUNER.cu:104-111): planes h, qx, qy, H, hc with
H = depth of the bed below the datum = -z_b; eta = h - H.

Each generator returns a Workload with:
  p      SimParams            sw   TsuSwitches (FP64 plain form)
  V      (5, npy, npx) float64 initial state (hc = 0)
  mask   (npy, npx) int32      1 = erodible
  CC,tCC boundary series or None (see boundary_series)
"""
from dataclasses import dataclass
from typing import Optional

import numpy as np

from .abi import make_params, make_switches

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(seed, n):
    """n consecutive outputs of SplitMix64 started at `seed` (uint64)."""
    with np.errstate(over="ignore"):
        k = np.arange(1, n + 1, dtype=np.uint64)
        z = np.uint64(seed) + k * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def gaussian_noise(seed, n):
    """Standard normals: SplitMix64 uniforms -> Box-Muller (pairs)."""
    m = (n + 1) // 2
    z = splitmix64(seed, 2 * m)
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    u1, u2 = u[0::2], u[1::2]
    r = np.sqrt(-2.0 * np.log1p(-u1))
    th = 2.0 * np.pi * u2
    return np.stack([r * np.cos(th), r * np.sin(th)], axis=1).reshape(-1)[:n]


@dataclass
class Workload:
    name: str
    p: object
    sw: object
    V: np.ndarray
    mask: np.ndarray
    CC: Optional[np.ndarray] = None
    tCC: Optional[np.ndarray] = None
    slr: float = 0.0
    steps: int = 0

    @property
    def ncells(self):
        return self.p.npx * self.p.npy


def centres(n, d):
    return (np.arange(n, dtype=np.float64) + 0.5) * d


def expired_series(npx, npy):
    """A CC series that is never active (t < tCC[timeCC-2] never holds), so a
    Read_files == 1 build treats every boundary as a wall
    (GPU/VolumeSolver.cu:249-254)."""
    nseg = 2 * npx + 2 * npy
    return np.zeros((2, nseg, 4)), np.array([-2.0, -1.0])


def hump(npx=512, npy=512, dx=10.0, steps=2000, seed=1, amp=2.0, sigma=500.0):
    """Config 1: cini-style Gaussian free-surface hump over a sloping,
    noisy bed.  z_b = -50 + 0.02 x + N(0, 0.1^2) (SplitMix64/Box-Muller,
    seed 1), eta0 = amp exp(-r^2 / (2 sigma^2)) about the domain centre,
    h = max(eta0 - z_b, 0), zero velocity, walls, erodible everywhere."""
    x = centres(npx, dx)[None, :]
    y = centres(npy, dx)[:, None]
    zb = -50.0 + 0.02 * x + 0.1 * gaussian_noise(seed, npx * npy).reshape(npy, npx)
    H = -zb
    xc, yc = 0.5 * npx * dx, 0.5 * npy * dx
    eta0 = amp * np.exp(-((x - xc) ** 2 + (y - yc) ** 2) / (2.0 * sigma ** 2))
    h = np.maximum(eta0 + H, 0.0)
    V = np.zeros((5, npy, npx))
    V[0], V[3] = h, H
    p = make_params(npx, npy, dx, dx)
    sw = make_switches(order=2, wbc=1, read_files=0)
    return Workload("hump%dx%d" % (npx, npy), p, sw, V, np.ones((npy, npx), np.int32), steps=steps)


def fractal_field(npx, npy, rng, slope=-3.0, std=1.5):
    """Gaussian random field with power spectrum ~ k^slope, zero mean, given std."""
    kx = np.fft.rfftfreq(npx)[None, :]
    ky = np.fft.fftfreq(npy)[:, None]
    k = np.sqrt(kx * kx + ky * ky)
    k[0, 0] = 1.0
    amp = k ** (slope / 2.0)
    amp[0, 0] = 0.0
    spec = (rng.standard_normal((npy, npx // 2 + 1)) + 1j * rng.standard_normal((npy, npx // 2 + 1))) * amp
    f = np.fft.irfft2(spec, s=(npy, npx))
    f -= f.mean()
    f *= std / f.std()
    return f


def shelf_bathymetry(npx, npy, dx, rng, slr, dry_fraction=0.2, std=1.5):
    """1:50 shelf-to-beach ramp rising to the east plus a fractal field,
    offset so `dry_fraction` of the cells lie above the raised sea level."""
    x = centres(npx, dx)[None, :]
    z = x / 50.0 + fractal_field(npx, npy, rng, std=std)
    z -= np.quantile(z, 1.0 - dry_fraction)
    zb = z + slr
    return -zb


def harbour_mask(npx, npy, rng, nblocks=3):
    """Binary mask (1 erodible) with `nblocks` seeded non-erodible rectangles."""
    m = np.ones((npy, npx), np.int32)
    for _ in range(nblocks):
        w = int(rng.integers(max(1, npx // 20), max(2, npx // 8)))
        hgt = int(rng.integers(max(1, npy // 20), max(2, npy // 8)))
        i0 = int(rng.integers(npx // 3, max(npx // 3 + 1, npx - w)))
        j0 = int(rng.integers(0, max(1, npy - hgt)))
        m[j0:j0 + hgt, i0:i0 + w] = 0
    return m


def boundary_series(H, slr, t_end, dt_cc=10.0, amp=0.0, period=600.0, g=9.81):
    """CC[t][seg][4] = (eta, u, v, H) in the reference layout
    (interpolations.cxx:533-774; segments bottom i | right npx+j |
    top npx+npy+i | left 2npx+npy+j).  The west (left) side carries an
    N-wave eta(t) = amp sin(2 pi t / period) for t <= period (crest then
    trough) with the long-wave velocity u = eta sqrt(g / h0); the other
    sides hold still water at the raised level slr.  On dry boundary cells
    eta = -H, so the ghost depth eta + H is zero."""
    npy, npx = H.shape
    nseg = 2 * npx + 2 * npy
    nt = int(np.ceil(t_end / dt_cc)) + 2
    tCC = np.arange(nt, dtype=np.float64) * dt_cc
    Hs = np.concatenate([H[0, :], H[:, npx - 1], H[npy - 1, :], H[:, 0]])
    CC = np.zeros((nt, nseg, 4))
    CC[:, :, 3] = Hs[None, :]
    still = np.maximum(slr, -Hs)
    CC[:, :, 0] = still[None, :]
    west = slice(2 * npx + npy, nseg)
    eta = amp * np.sin(2.0 * np.pi * tCC / period) * (tCC <= period)
    h0 = np.maximum(slr + Hs[west], 0.0)
    wet = h0 > 1.0
    CC[:, west, 0] = np.where(wet[None, :], slr + eta[:, None], still[west][None, :])
    CC[:, west, 1] = np.where(wet[None, :], eta[:, None] * np.sqrt(g / np.maximum(h0, 1.0))[None, :], 0.0)
    return CC, tCC


def nwave_shelf(npx=4096, npy=4096, dx=5.0, steps=5000, seed=2, slr=0.5, amp=3.0, period=600.0,
                t_series=None):
    """Config 2: fractal (k^-3) bathymetry over a 1:50 shelf-to-beach ramp,
    ~20 % dry after a +0.5 m sea-level rise, 3 seeded non-erodible
    rectangles, west-boundary N-wave (3 m, 600 s) through the CC series,
    sediment on."""
    rng = np.random.default_rng(seed)
    H = shelf_bathymetry(npx, npy, dx, rng, slr)
    mask = harbour_mask(npx, npy, rng)
    V = np.zeros((5, npy, npx))
    V[0] = np.maximum(slr + H, 0.0)
    V[3] = H
    if t_series is None:
        t_series = 2000.0
    CC, tCC = boundary_series(H, slr, t_series, amp=amp, period=period)
    p = make_params(npx, npy, dx, dx)
    sw = make_switches(order=2, wbc=1, read_files=1, eta0=slr)
    return Workload("nwave%dx%d" % (npx, npy), p, sw, V, mask, CC, tCC, slr=slr, steps=steps)


def humps_shelf(npx=8192, npy=8192, dx=5.0, steps=2000, seed=3, slr=0.0, nhumps=8):
    """Config 3: the same bathymetry/mask generators, source = `nhumps` seeded
    Gaussian humps (amplitude 0.5-4 m, sigma 200-2000 m), walls."""
    rng = np.random.default_rng(seed)
    H = shelf_bathymetry(npx, npy, dx, rng, slr)
    mask = harbour_mask(npx, npy, rng)
    x = centres(npx, dx)[None, :]
    y = centres(npy, dx)[:, None]
    eta = np.zeros((npy, npx))
    for _ in range(nhumps):
        a = rng.uniform(0.5, 4.0)
        s = rng.uniform(200.0, 2000.0)
        xc = rng.uniform(0.1, 0.6) * npx * dx
        yc = rng.uniform(0.1, 0.9) * npy * dx
        eta += a * np.exp(-((x - xc) ** 2 + (y - yc) ** 2) / (2.0 * s * s))
    V = np.zeros((5, npy, npx))
    V[0] = np.maximum(slr + eta + H, 0.0)
    V[3] = H
    p = make_params(npx, npy, dx, dx)
    sw = make_switches(order=2, wbc=1, read_files=0, eta0=slr)
    return Workload("humps%dx%d" % (npx, npy), p, sw, V, mask, slr=slr, steps=steps)


def ensemble(nmembers=256, lo=256, hi=2048, seed=4, dx=5.0, slr=0.5, t_series=400.0):
    """Config 4: `nmembers` members on square grids whose sides are drawn
    log-uniform in [lo, hi] (seed 4), each with its own seeded shelf
    bathymetry, harbour mask and west-boundary N-wave (amplitude 1-5 m,
    period 300-1200 s); FP32 precision form."""
    rng = np.random.default_rng(seed)
    sides = np.exp(rng.uniform(np.log(lo), np.log(hi), nmembers)).astype(int)
    amps = rng.uniform(1.0, 5.0, nmembers)
    periods = rng.uniform(300.0, 1200.0, nmembers)
    seeds = rng.integers(0, 2 ** 31, nmembers)
    out = []
    for k in range(nmembers):
        n = int(sides[k])
        mr = np.random.default_rng(int(seeds[k]))
        H = shelf_bathymetry(n, n, dx, mr, slr)
        mask = harbour_mask(n, n, mr)
        V = np.zeros((5, n, n))
        V[0] = np.maximum(slr + H, 0.0)
        V[3] = H
        CC, tCC = boundary_series(H, slr, t_series, amp=float(amps[k]), period=float(periods[k]))
        p = make_params(n, n, dx, dx)
        sw = make_switches(order=2, wbc=1, read_files=1, precision=1, eta0=slr)
        out.append(Workload("member%d_%d" % (k, n), p, sw, V, mask, CC, tCC, slr=slr))
    return out
