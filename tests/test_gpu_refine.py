"""GPU tests of the adjoint and the continuous refinement (reference frame):

* torch.autograd.gradcheck of the hand-written d corr / d(shift_x, shift_y, defocus)
  against FP64 finite differences (step 1e-4 px / 1e-4 micron) on 64 particles;
* the batched bound-constrained quasi-Newton refinement recovers perturbed shifts
  and defocus offsets, and takes a fraction of the time of an exhaustive GPU grid.
"""
import math
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup(pkg, nptcls, nrefs=4, noise=False, df_offset=None, seed_base=0):
    w = pkg.synth.config0(nrefs=nrefs, nptcls=nptcls, seed_base=seed_base)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R, noise=noise)
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True)
    pc.set_refs(1, refs.numpy(), True)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    off = np.zeros(nptcls) if df_offset is None else df_offset
    pc.create_polar_absctfmats(pkg.ctfparams_array(nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx + off, dfy=parts.dfy + off, angast=parts.angast))
    return w, pc, parts


def true_pose(w, parts, i):
    """nearest in-plane index and the reference-side shift that undoes the particle's shift"""
    psi = math.radians(parts.psi[i])
    tx, ty = parts.shift[i]
    irot = int(round(parts.psi[i] * w.nrots / 360.0)) % w.nrots + 1
    sh = (-(math.cos(psi) * tx + math.sin(psi) * ty), -(-math.sin(psi) * tx + math.cos(psi) * ty))
    return irot, sh


def test_gradcheck_shift_defocus(pkg):
    import torch
    from simple3_0_b200.autograd import ShiftDefocusCorr
    n = 64
    w, pc, parts = setup(pkg, n, noise=True)
    rng = np.random.default_rng(3)
    iref = parts.ref + 1
    iptcl = np.arange(1, n + 1)
    irot = rng.integers(1, w.nrots + 1, n)
    x = torch.tensor(np.c_[rng.uniform(-2, 2, (n, 2)), rng.uniform(-0.1, 0.1, n)], dtype=torch.float64,
                     requires_grad=True)
    fn = lambda x_: ShiftDefocusCorr.apply(x_, pc, iref, iptcl, irot)
    assert torch.autograd.gradcheck(fn, (x,), eps=1e-4, atol=2e-5, rtol=1e-3)


def test_refine_recovers_shift_and_defocus(pkg):
    n = 32
    rng = np.random.default_rng(5)
    delta = rng.uniform(-0.1, 0.1, n)             # error of the "estimated" defocus
    w, pc, parts = setup(pkg, n, df_offset=delta)
    irot, x0, truth = [], [], []
    for i in range(n):
        r, sh = true_pose(w, parts, i)
        irot.append(r)
        truth.append([sh[0], sh[1], -delta[i]])
        x0.append([sh[0] + rng.uniform(-1.5, 1.5), sh[1] + rng.uniform(-1.5, 1.5), 0.0])
    truth, x0 = np.array(truth), np.array(x0)
    lb, ub = [-6.0, -6.0, -0.2], [6.0, 6.0, 0.2]
    f0, _ = pc.grad_batch(parts.ref + 1, np.arange(1, n + 1), irot, x0[:, 0], x0[:, 1], x0[:, 2])
    x, f, nev, nit, conv = pc.refine_batch(parts.ref + 1, np.arange(1, n + 1), irot, x0, lb, ub, maxits=100)
    assert np.all(f >= f0 - 1e-12)
    dsh = np.hypot(*(x[:, :2] - truth[:, :2]).T)
    ddf = np.abs(x[:, 2] - truth[:, 2])
    print(f"refine: median shift error {np.median(dsh):.3f} px, median defocus error {np.median(ddf):.4f} um, "
          f"median evaluations {np.median(nev):.0f}, converged {conv.mean():.2f}")
    assert np.median(dsh) < 0.25 and np.mean(dsh < 0.5) > 0.8
    assert np.median(ddf) < 0.02


def test_refine_faster_than_exhaustive_grid(pkg):
    """the same problems on an exhaustive GPU grid (0.1 px, 0.02 micron) of the same box
    around the start: the refinement must reach at least the grid's best value in a
    quarter of its time"""
    n = 16
    rng = np.random.default_rng(9)
    delta = rng.uniform(-0.1, 0.1, n)
    w, pc, parts = setup(pkg, n, df_offset=delta)
    irot, x0 = [], []
    for i in range(n):
        r, sh = true_pose(w, parts, i)
        irot.append(r)
        x0.append([sh[0] + rng.uniform(-1, 1), sh[1] + rng.uniform(-1, 1), 0.0])
    x0 = np.array(x0)
    half = np.array([2.0, 2.0, 0.2])
    gx = np.arange(-20, 21) * 0.1
    gd = np.arange(-10, 11) * 0.02
    t0 = time.perf_counter()
    best_grid = np.full(n, -np.inf)
    for i in range(n):
        SX, SY, DD = np.meshgrid(x0[i, 0] + gx, x0[i, 1] + gx, gd, indexing="ij")
        f, _ = pc.grad_batch(np.full(SX.size, parts.ref[i] + 1), np.full(SX.size, i + 1), np.full(SX.size, irot[i]),
                             SX.ravel(), SY.ravel(), DD.ravel())
        best_grid[i] = f.max()
    t_grid = time.perf_counter() - t0
    t0 = time.perf_counter()
    x, f, nev, nit, conv = pc.refine_batch(parts.ref + 1, np.arange(1, n + 1), irot, x0, x0 - half, x0 + half,
                                           maxits=100)
    t_ref = time.perf_counter() - t0
    print(f"exhaustive grid {t_grid:.3f} s ({gx.size ** 2 * gd.size} points/problem), refinement {t_ref:.3f} s "
          f"(median {np.median(nev):.0f} evaluations/problem)")
    assert np.mean(f >= best_grid - 1e-4) > 0.9
    assert t_ref < 0.25 * t_grid
