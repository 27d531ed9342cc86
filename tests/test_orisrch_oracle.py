"""CPU tests of the oracle's orientation derivatives (the orientation-gradient search's inputs):
euler2dm (simple_ori_light.f90:87-147), the KB derivative dapod (simple_kbinterpol.f90:179-192),
fdf_project_polar / fdf_interp_fcomp (simple_projector.f90:245-267, :338-400) and
gencorr_cont_shift_grad_cc_for_rot_8 (simple_polarft_corrcalc.f90:1788-1847).

Each derivative is checked against central differences of the function it differentiates:
dR/de of euler2m, dapod of apod, the projection's angle derivatives of fproject_polar (on the
samples whose interpolation window does not move between the two evaluations: the window
follows nint(loc) and the Kaiser-Bessel weight at its edge is not zero, so the projection
jumps where a window moves), the correlator's orientation gradient along the derivative
references, and its shift gradient."""
import math

import numpy as np
import pytest

BOX = 32


def volume(O, seed=0):
    rng = np.random.default_rng(seed)
    shape = (BOX, BOX, BOX // 2 + 1)
    half = (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)
    return O.expand_cmat3d(half, BOX)


def geom(O):
    g = O.geom(128, 2, 14, BOX)
    return g, O.tables(g)


def test_euler2dm_is_derivative_of_euler2m(O):
    e = np.array([31.0, 47.0, 113.0])
    dR = O.euler2dm(e)
    h = 1e-4
    for j in range(3):
        d = np.zeros(3)
        d[j] = h
        fd = (O.euler2m(e + d) - O.euler2m(e - d)) / (2 * math.radians(h))
        assert np.max(np.abs(dR[j] - fd)) < 1e-8


def test_dapod_is_derivative_of_apod(O):
    h = 1e-6
    for x in np.linspace(-1.45, 1.45, 29):
        fd = (O.kb_apod(x + h) - O.kb_apod(x - h)) / (2 * h)
        assert abs(O.kb_dapod(x) - fd) < 1e-6 * max(1.0, abs(fd))
    assert O.kb_dapod(1.6) == 0.0 and O.kb_dapod(-1.6) == 0.0


def _windows(O, g, t, eul):
    """nint(loc) of every sample (K, P, 3)"""
    R = O.euler2m(eul)
    N, P = g.nrots, g.pftsz
    pol = t.polar.reshape(g.K, 2 * N)
    v = np.stack([pol[:, :P], pol[:, N:N + P], np.zeros((g.K, P))], -1).astype(np.float64)
    loc = v @ R
    return np.where(loc >= 0, np.floor(loc + 0.5), -np.floor(-loc + 0.5))


@pytest.mark.parametrize("eul", [(31.0, 47.0, 113.0), (200.0, 120.0, 10.0)])
def test_fdf_project_polar(O, eul):
    g, t = geom(O)
    ex = volume(O)
    eul = np.array(eul)
    pft, dpft = O.fdf_project_polar(g, t, ex, BOX, eul)
    # the value is interp_fcomp_norm's
    ref = O.fproject_polar(g, t, ex, BOX, eul)
    assert np.max(np.abs(pft - ref)) < 1e-12 * np.max(np.abs(ref))
    h = 1e-4
    for j in range(3):
        d = np.zeros(3)
        d[j] = h
        fp = O.fproject_polar(g, t, ex, BOX, eul + d)
        fm = O.fproject_polar(g, t, ex, BOX, eul - d)
        fd = (fp - fm) / (2 * math.radians(h))
        stable = np.all((_windows(O, g, t, eul + d) == _windows(O, g, t, eul)) &
                        (_windows(O, g, t, eul - d) == _windows(O, g, t, eul)), axis=-1)
        assert stable.mean() > 0.95
        err = np.abs(dpft[j] - fd)[stable]
        assert np.max(err) < 1e-5 * np.max(np.abs(dpft[j]))


def test_cont_shift_grad(O):
    g = O.geom(128, 2, 14, BOX, kstop=12)
    t = O.tables(g)
    ex = volume(O, 1)
    eul = np.array([77.0, 33.0, 250.0])
    ref, dref = O.fdf_project_polar(g, t, ex, BOX, eul)
    ref = ref.astype(np.complex64)
    dref = dref.astype(np.complex64)
    rng = np.random.default_rng(2)
    ptcl = (0.6 * ref + 0.3 * (rng.standard_normal(ref.shape) + 1j * rng.standard_normal(ref.shape))).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(smpd=2.0, dfx=1.6, dfy=1.4, angast=40.0))
    sh = np.array([0.4, -0.7])
    for irot in (1, 20, 129, 200):
        f, gr = O.gencorr_cont_shift_grad(g, t, ref, dref, ptcl, irot, ctf, sh)
        # the value: unweighted correlation normalised over kfrom..kstop
        assert abs(f - O.gencorr_for_rot(g, t, ref, ptcl, irot, ctf, sh, match_filt=True)) < 1e-12
        # orientation gradient: derivative along the derivative references
        ht = 1e-3
        for j in range(3):
            fp, _ = O.gencorr_cont_shift_grad(g, t, (ref + ht * dref[j]).astype(np.complex64), dref, ptcl, irot, ctf, sh)
            fm, _ = O.gencorr_cont_shift_grad(g, t, (ref - ht * dref[j]).astype(np.complex64), dref, ptcl, irot, ctf, sh)
            fd = (fp - fm) / (2 * ht)
            assert abs(gr[j] - fd) < 2e-4 * max(abs(fd), 1e-3)
        # shift gradient
        hs = 1e-5
        for d in range(2):
            e = np.zeros(2)
            e[d] = hs
            fp, _ = O.gencorr_cont_shift_grad(g, t, ref, dref, ptcl, irot, ctf, sh + e)
            fm, _ = O.gencorr_cont_shift_grad(g, t, ref, dref, ptcl, irot, ctf, sh - e)
            assert abs(gr[3 + d] - (fp - fm) / (2 * hs)) < 1e-6
