"""GPU tests of the adjoint and the continuous refinement (reference frame):

* torch.autograd.gradcheck of the hand-written d corr / d(shift_x, shift_y, defocus)
  against FP64 finite differences (step 1e-4 px / 1e-4 micron) on 64 particles.  The
  correlation uses |CTF| (the reference's absctfmats), which has a corner at every CTF
  zero: across a particle's polar samples there are about 1e4 such corners per micron,
  so a +-1e-4 micron central difference often straddles one and no longer measures the
  derivative.  The defocus column is therefore gradchecked on the particles whose
  difference interval contains no corner (found from the oracle's |CTF| and its
  derivative at both ends); every particle's defocus derivative is compared with the
  oracle's analytic one in test_gpu_exact.py::test_grad_batch_defocus.
* the batched bound-constrained quasi-Newton refinement, each problem in its own box,
  recovers perturbed shifts and reaches the maximum of an exhaustive grid over the box,
  in a fraction of the grid's time.  The generator's defocus is not the maximiser of the
  correlation at the nearest discrete rotation (the residual in-plane angle moves it by
  up to ~0.3 micron), so defocus is judged by the grid, not by the generator.
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


def ctf_corner_free(O, w, parts, i, ddf, eps):
    """True when no polar sample's CTF crosses zero for defocus offsets in [ddf-eps, ddf+eps]:
    d|CTF|/d(defocus) keeps its sign at every sample where |CTF| is small"""
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    ends = []
    for s in (-1.0, 1.0):
        cp = O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]) + ddf + s * eps,
                        float(parts.dfy[i]) + ddf + s * eps, float(parts.angast[i]))
        ends.append((O.ctfmat(g, t, cp), O.dctfmat_ddf(g, t, cp)))
    (c0, d0), (c1, d1) = ends
    return not np.any((np.sign(d0) != np.sign(d1)) & (c0 < 0.5) & (c1 < 0.5))


def test_gradcheck_shift_defocus(pkg, O):
    import torch
    from simple3_0_b200.autograd import ShiftDefocusCorr
    n = 64
    w, pc, parts = setup(pkg, n, noise=True)
    rng = np.random.default_rng(3)
    iref = parts.ref + 1
    iptcl = np.arange(1, n + 1)
    irot = rng.integers(1, w.nrots + 1, n)
    x = np.c_[rng.uniform(-2, 2, (n, 2)), rng.uniform(-0.1, 0.1, n)]
    # shifts: all particles, defocus held
    xs = torch.tensor(x[:, :2], dtype=torch.float64, requires_grad=True)
    ddf = torch.tensor(x[:, 2:], dtype=torch.float64)
    fs = lambda xs_: ShiftDefocusCorr.apply(torch.cat([xs_, ddf], 1), pc, iref, iptcl, irot)
    assert torch.autograd.gradcheck(fs, (xs,), eps=1e-4, atol=2e-5, rtol=1e-3)
    # defocus: the particles whose difference interval straddles no |CTF| corner
    sub = np.array([i for i in range(n) if ctf_corner_free(O, w, parts, i, x[i, 2], 1e-4)])
    assert sub.size >= 16
    sh = torch.tensor(x[sub, :2], dtype=torch.float64)
    xd = torch.tensor(x[sub, 2:], dtype=torch.float64, requires_grad=True)
    fd = lambda xd_: ShiftDefocusCorr.apply(torch.cat([sh, xd_], 1), pc, iref[sub], iptcl[sub], irot[sub])
    assert torch.autograd.gradcheck(fd, (xd,), eps=1e-4, atol=2e-5, rtol=1e-3)


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
    # the refined point is the best of a local exhaustive grid (0.05 px, 0.01 micron) around it
    gx = np.arange(-2, 3) * 0.05
    gd = np.arange(-2, 3) * 0.01
    for i in range(n):
        SX, SY, DD = np.meshgrid(x[i, 0] + gx, x[i, 1] + gx, x[i, 2] + gd, indexing="ij")
        keep = (SX >= lb[0]) & (SX <= ub[0]) & (SY >= lb[1]) & (SY <= ub[1]) & (DD >= lb[2]) & (DD <= ub[2])
        fg, _ = pc.grad_batch(np.full(keep.sum(), parts.ref[i] + 1), np.full(keep.sum(), i + 1),
                              np.full(keep.sum(), irot[i]), SX[keep], SY[keep], DD[keep])
        assert f[i] >= fg.max() - 1e-5, (i, f[i], fg.max())


def test_refine_faster_than_exhaustive_grid(pkg):
    """the same problems on an exhaustive GPU grid (0.1 px, 0.02 micron) of the same box
    around the start: the refinement must reach at least the grid's best value in a
    quarter of its time.  The correlation has several maxima in defocus (about 0.09
    micron apart at these shells), so each problem is refined from four defocus starts
    spread over the box, all in the same batch, and keeps its best end point."""
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
    starts = np.array([-0.15, -0.05, 0.05, 0.15])
    ns0 = starts.size
    xs = np.repeat(x0, ns0, axis=0)
    xs[:, 2] += np.tile(starts, n)
    t0 = time.perf_counter()
    xa, fa, neva, nit, conv = pc.refine_batch(np.repeat(parts.ref + 1, ns0), np.repeat(np.arange(1, n + 1), ns0),
                                              np.repeat(irot, ns0), xs, np.repeat(x0 - half, ns0, axis=0),
                                              np.repeat(x0 + half, ns0, axis=0), maxits=100)
    t_ref = time.perf_counter() - t0
    f = fa.reshape(n, ns0).max(1)
    nev = neva.reshape(n, ns0).sum(1)
    print(f"exhaustive grid {t_grid:.3f} s ({gx.size ** 2 * gd.size} points/problem), refinement {t_ref:.3f} s "
          f"(median {np.median(nev):.0f} evaluations/problem)")
    assert np.mean(f >= best_grid - 1e-4) > 0.9
    assert t_ref < 0.25 * t_grid
