"""Seeded synthetic workloads for the polar Fourier correlation search.

The reference measures this path on no public dataset; these generators stand
in with the shapes, sizes and value distributions of the workloads the search
is benchmarked on:

* a Gaussian-blob volume (box^3, blob sigma and amplitude uniform, centres
  uniform in a ball);
* references = central sections at uniform-random SO(3) orientations, sampled
  analytically on the polar grid of ``polarft_corrcalc`` (the 3-D Fourier
  transform of a Gaussian blob is known in closed form, so the sections are
  exact);
* particles = a random reference's section, rotated in-plane, shifted, multiplied
  by an astigmatic CTF, phase-flipped (so the particle carries |CTF|, as
  ``prepimg4align`` leaves it) and corrupted by white Gaussian noise at a given
  real-space SNR, delivered as a Cartesian half-plane Fourier transform in the
  ``image%cmat(box/2+1, box)`` layout that ``polarize`` reads.

Random streams: numpy PCG64 with seed = 1000*config + stream, one stream each for
blobs, orientations, in-plane angles, shifts, CTF and noise.  Heavy evaluation
runs in torch on whatever device is given (CPU in tests, the GPU in the bench).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np
import torch

STREAM_BLOBS, STREAM_ORI, STREAM_INPL, STREAM_SHIFT, STREAM_CTF, STREAM_NOISE, STREAM_PICK = range(7)


@dataclass
class Workload:
    name: str
    box: int
    nrots: int
    kfrom: int
    kto: int
    nrefs: int
    nptcls: int
    nblobs: int
    sigma: tuple
    radius: float
    shift_range: float
    smpd: float = 1.3
    kv: float = 300.0
    cs: float = 2.7
    fraca: float = 0.1
    defocus: tuple = (1.0, 3.0)
    astig: tuple = (0.0, 0.1)
    snr: float = 0.1
    shift_grid: tuple = ()        # ((sx, sy), ...) search grid, empty = zero shift only
    seed_base: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def pftsz(self) -> int:
        return self.nrots // 2

    @property
    def K(self) -> int:
        return self.kto - self.kfrom + 1


def shift_grid(half_range: float, step: float):
    n = int(round(half_range / step))
    return tuple((i * step, j * step) for i in range(-n, n + 1) for j in range(-n, n + 1))


def config0(**kw) -> Workload:
    """64^3 box, 50 blobs sigma U[2,4], 100 refs, 1,000 ptcls, shifts U[-3,3], nrots 128, k 2..20."""
    w = Workload("config0_box64_refs100_ptcls1000_nrots128_k2-20", 64, 128, 2, 20, 100, 1000, 50,
                 (2.0, 4.0), 24.0, 3.0, seed_base=0)
    return _override(w, kw)


def config1(**kw) -> Workload:
    """128^3 box, 100 blobs sigma U[2,6], 500 refs, 20,000 ptcls, shifts U[-5,5], nrots 360,
    k 2..40, 9x9 search grid of 0.5 px (+-2 px)."""
    w = Workload("config1_box128_refs500_ptcls20000_shifts81_nrots360_k2-40", 128, 360, 2, 40, 500, 20000,
                 100, (2.0, 6.0), 48.0, 5.0, shift_grid=shift_grid(2.0, 0.5), seed_base=1000)
    return _override(w, kw)


def geometry_c(**kw) -> Workload:
    """box 200 / nrots 600 / k 2..60 geometry of the batching workload."""
    w = Workload("box200_nrots600_k2-60", 200, 600, 2, 60, 100, 1000, 100, (2.0, 6.0), 75.0, 5.0,
                 seed_base=4000)
    return _override(w, kw)


def _override(w: Workload, kw) -> Workload:
    for k, v in kw.items():
        setattr(w, k, v)
    return w


def rng(w: Workload, stream: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(w.seed_base + stream))


def random_rotations(n: int, g: np.random.Generator) -> np.ndarray:
    """Uniform SO(3) rotation matrices from normalised Gaussian quaternions."""
    q = g.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    a, b, c, d = q.T
    R = np.stack([
        np.stack([a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)], -1),
        np.stack([2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)], -1),
        np.stack([2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d], -1),
    ], 1)
    return R


@dataclass
class Blobs:
    centres: np.ndarray   # (nb, 3) px
    sigmas: np.ndarray    # (nb,)
    amps: np.ndarray      # (nb,)


def make_blobs(w: Workload) -> Blobs:
    g = rng(w, STREAM_BLOBS)
    nb = w.nblobs
    d = g.standard_normal((nb, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    r = w.radius * g.uniform(0.0, 1.0, nb) ** (1.0 / 3.0)
    return Blobs(d * r[:, None], g.uniform(w.sigma[0], w.sigma[1], nb), g.uniform(0.5, 1.0, nb))


def polar_tables(w: Workload):
    """polar coordinates of the polarft_corrcalc grid, float32 like the reference
    (ang = TWOPI/nrots, x = sin(a)*k, y = -cos(a)*k); returns x, y of shape (K, P)."""
    N, P = w.nrots, w.pftsz
    twopi = np.float32(2.0) * np.float32(math.acos(-1.0))
    ang = np.float32(twopi / np.float32(N))
    a = (np.arange(P, dtype=np.float32) * ang).astype(np.float32)
    k = np.arange(w.kfrom, w.kto + 1, dtype=np.float32)[:, None]
    return (np.sin(a)[None, :] * k).astype(np.float32), (-np.cos(a)[None, :] * k).astype(np.float32)


def _blob_ft(blobs: Blobs, qx, qy, qz, device, dtype):
    """sum_b amp_b (2 pi sigma_b^2)^(3/2) exp(-2 pi^2 sigma_b^2 |q|^2 - 2 pi i q.c_b); q in cycles/px"""
    cdt = torch.complex128 if dtype == torch.float64 else torch.complex64
    out = torch.zeros(qx.shape, dtype=cdt, device=device)
    q2 = qx * qx + qy * qy + qz * qz
    for b in range(len(blobs.sigmas)):
        s2 = float(blobs.sigmas[b]) ** 2
        scale = float(blobs.amps[b]) * (2.0 * math.pi * s2) ** 1.5
        cx, cy, cz = (float(v) for v in blobs.centres[b])
        mag = scale * torch.exp(-2.0 * math.pi ** 2 * s2 * q2)
        ph = -2.0 * math.pi * (qx * cx + qy * cy + qz * cz)
        out += torch.polar(mag, ph)
    return out


def make_refs(w: Workload, device="cpu", blobs: Blobs | None = None):
    """Reference polar FTs, complex64 tensor (nrefs, K, P), exact central sections."""
    blobs = blobs or make_blobs(w)
    R = random_rotations(w.nrefs, rng(w, STREAM_ORI))
    x, y = polar_tables(w)
    x = torch.as_tensor(x, dtype=torch.float64, device=device) / w.box
    y = torch.as_tensor(y, dtype=torch.float64, device=device) / w.box
    Rt = torch.as_tensor(R, dtype=torch.float64, device=device)
    # section point q = x * u + y * v with u, v the first two rows of R
    qx = x[None] * Rt[:, 0, 0, None, None] + y[None] * Rt[:, 1, 0, None, None]
    qy = x[None] * Rt[:, 0, 1, None, None] + y[None] * Rt[:, 1, 1, None, None]
    qz = x[None] * Rt[:, 0, 2, None, None] + y[None] * Rt[:, 1, 2, None, None]
    return _blob_ft(blobs, qx, qy, qz, device, torch.float64).to(torch.complex64), R


@dataclass
class Particles:
    cmat: torch.Tensor       # complex64 (n, box, box//2+1): cmat[i, kphys, hphys]
    ref: np.ndarray          # true reference index (0-based)
    psi: np.ndarray          # in-plane rotation, degrees
    shift: np.ndarray        # (n, 2) px
    dfx: np.ndarray          # microns
    dfy: np.ndarray
    angast: np.ndarray       # degrees


def ctf_params(w: Workload, n: int):
    g = rng(w, STREAM_CTF)
    df = g.uniform(w.defocus[0], w.defocus[1], n)
    ast = g.uniform(w.astig[0], w.astig[1], n)
    ang = g.uniform(0.0, 180.0, n)
    return (df + ast / 2).astype(np.float32), (df - ast / 2).astype(np.float32), ang.astype(np.float32)


def abs_ctf(w: Workload, s2, ang, dfx, dfy, angast):
    """|CTF| (simple_ctf.f90 conventions: defocus in microns, angast in degrees), torch, broadcasting."""
    kv = w.kv * 1000.0
    wl = 12.26 / math.sqrt(kv + 0.9784 * kv * kv / 1.0e6) / w.smpd
    cs = w.cs * 1.0e7 / w.smpd
    ampc = math.atan(w.fraca / math.sqrt(1.0 - w.fraca ** 2))
    dfxp, dfyp = dfx * 1.0e4 / w.smpd, dfy * 1.0e4 / w.smpd
    angr = angast * math.pi / 180.0
    df = 0.5 * (dfxp + dfyp + torch.cos(2.0 * (ang - angr)) * (dfxp - dfyp))
    chi = math.pi * wl * s2 * (df - 0.5 * wl * wl * s2 * cs) + ampc
    return torch.abs(torch.sin(chi))


def make_particles(w: Workload, R: np.ndarray, device="cpu", blobs: Blobs | None = None, chunk: int = 256,
                   noise: bool = True, ctf: bool = True, first: int = 0, count: int | None = None) -> Particles:
    """Particles [first, first+count) of the workload (the random streams are drawn for all
    w.nptcls particles so any slice is reproducible)."""
    blobs = blobs or make_blobs(w)
    n_all = w.nptcls
    count = n_all - first if count is None else count
    ref = rng(w, STREAM_PICK).integers(0, w.nrefs, n_all)
    psi = rng(w, STREAM_INPL).uniform(0.0, 360.0, n_all)
    shift = rng(w, STREAM_SHIFT).uniform(-w.shift_range, w.shift_range, (n_all, 2))
    dfx, dfy, angast = ctf_params(w, n_all)
    sl = slice(first, first + count)
    box, hh = w.box, w.box // 2 + 1
    h = torch.arange(hh, dtype=torch.float32, device=device)
    kl = torch.arange(box, dtype=torch.float32, device=device)
    kl = torch.where(kl >= box // 2, kl - box, kl)
    H, Kc = torch.meshgrid(h, kl, indexing="xy")   # (box, hh): [kphys, hphys]
    out = torch.empty((count, box, hh), dtype=torch.complex64, device=device)
    Rall = torch.as_tensor(R, dtype=torch.float32, device=device)
    for c0 in range(0, count, chunk):
        c1 = min(count, c0 + chunk)
        idx = np.arange(first + c0, first + c1)
        rr = torch.as_tensor(ref[idx], device=device)
        ps = torch.as_tensor(np.deg2rad(psi[idx]), dtype=torch.float32, device=device)[:, None, None]
        # particle frequency f -> reference frame frequency R(-psi) f
        fx = (torch.cos(ps) * H + torch.sin(ps) * Kc) / box
        fy = (-torch.sin(ps) * H + torch.cos(ps) * Kc) / box
        Rc = Rall[rr]
        qx = fx * Rc[:, 0, 0, None, None] + fy * Rc[:, 1, 0, None, None]
        qy = fx * Rc[:, 0, 1, None, None] + fy * Rc[:, 1, 1, None, None]
        qz = fx * Rc[:, 0, 2, None, None] + fy * Rc[:, 1, 2, None, None]
        F = _blob_ft(blobs, qx, qy, qz, device, torch.float32)
        sx = torch.as_tensor(shift[idx, 0], dtype=torch.float32, device=device)[:, None, None]
        sy = torch.as_tensor(shift[idx, 1], dtype=torch.float32, device=device)[:, None, None]
        F = F * torch.polar(torch.ones_like(H), -2.0 * math.pi * (H * sx + Kc * sy) / box)
        if ctf:
            s2 = (H * H + Kc * Kc) / (box * box)
            ang = torch.atan2(Kc, H)
            tdx = torch.as_tensor(dfx[idx], device=device)[:, None, None]
            tdy = torch.as_tensor(dfy[idx], device=device)[:, None, None]
            tan = torch.as_tensor(angast[idx], device=device)[:, None, None]
            F = F * abs_ctf(w, s2[None], ang[None], tdx, tdy, tan)
        if noise:
            # real-space signal variance from Parseval over the half plane (h>0 counted twice)
            wgt = torch.where(H > 0, 2.0, 1.0)
            p2 = (wgt * (F.real ** 2 + F.imag ** 2)).sum(dim=(1, 2)) / box ** 4
            mean2 = (F[:, 0, 0].real / box ** 2) ** 2
            var = torch.clamp(p2 - mean2, min=1e-30)
            sig_n = torch.sqrt(var / w.snr) * box / math.sqrt(2.0)
            g = np.stack([np.random.Generator(np.random.PCG64([w.seed_base + STREAM_NOISE, int(i)]))
                          .standard_normal((box, hh, 2), dtype=np.float32) for i in idx])
            g = torch.as_tensor(g, device=device)
            F = F + torch.complex(g[..., 0], g[..., 1]) * sig_n[:, None, None]
        out[c0:c1] = F
    return Particles(out, ref[sl], psi[sl], shift[sl], dfx[sl], dfy[sl], angast[sl])
