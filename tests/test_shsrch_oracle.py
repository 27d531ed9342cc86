"""CPU tests of the shift search's optimiser and of the oracle's restatement of the
reference's shift search (oracle/shsrch.py).

* The L-BFGS-B of simple3.0_b200/csrc/lbfgsb3.h (reverse communication, More-Thuente line
  search) reaches the same bounded minima as SciPy's L-BFGS-B -- an implementation of the
  same published algorithm (Byrd, Lu, Nocedal & Zhu; Morales & Nocedal) -- on analytic
  functions with and without active bounds, and on the shift-search cost itself
  (-gencorr_for_rot_8 of the oracle at a fixed rotation).
* The restated search recovers a known particle shift and rotation: a particle made from a
  reference rotated by j samples and shifted by t peaks at irot = j + 1 with cc -> 1, and
  the reported shift, rotated back into the particle frame, is the shift that undoes t.
"""
import math

import numpy as np
import pytest
import scipy.optimize as so


@pytest.fixture(scope="module")
def S(O):
    import shsrch
    return shsrch


def run_lb3(S, fg, x0, lb, ub, ftol=1e-1, gtol=1e-3, maxits=1000):
    """minimise fg with lbfgsb3 through the oracle's shim; returns (x, f, nfgv)"""
    L = S._lib()
    x0, lb, ub = (np.asarray(v, np.float64) for v in (x0, lb, ub))
    h = L.lb3_new(S._dp(x0), S._dp(lb), S._dp(ub), 1e7, 1e-5, ftol, gtol, 0.1, 15)
    try:
        xt = np.zeros(2)
        task = L.lb3_task(h)
        while True:
            if task == S.FG:
                L.lb3_xt(h, S._dp(xt))
                f, g = fg(xt)
                task = L.lb3_evaluated(h, f, S._dp(np.ascontiguousarray(g, np.float64)))
            elif task == S.NEW_X:
                if L.lb3_nfgv(h) > maxits:
                    break
                task = L.lb3_proceed(h)
            else:
                break
        L.lb3_x(h, S._dp(xt))
        return xt.copy(), L.lb3_f(h), L.lb3_nfgv(h)
    finally:
        L.lb3_free(h)


def rosen(x):
    a, b = x
    f = (1 - a) ** 2 + 100 * (b - a * a) ** 2
    return f, np.array([-2 * (1 - a) - 400 * a * (b - a * a), 200 * (b - a * a)])


def quad(x):
    A = np.array([[3.0, 1.0], [1.0, 2.0]])
    c = np.array([-4.0, 5.0])
    return 0.5 * x @ A @ x + c @ x, A @ x + c


@pytest.mark.parametrize("fun,x0,lb,ub", [
    (rosen, [-1.2, 1.0], [-2.0, -2.0], [2.0, 2.0]),
    (rosen, [-1.2, 1.0], [-2.0, -2.0], [0.8, 2.0]),      # minimum on the bound a = 0.8
    (quad, [0.0, 0.0], [-1.0, -1.0], [1.0, 1.0]),        # both bounds active at the minimum
    (quad, [0.5, 0.5], [-10.0, -10.0], [10.0, 10.0]),
])
def test_lbfgsb3_matches_scipy(S, fun, x0, lb, ub):
    for ftol, gtol in ((1e-3, 0.9), (1e-1, 1e-3)):      # SciPy's line-search constants, the reference's
        x, f, _ = run_lb3(S, fun, x0, lb, ub, ftol, gtol)
        r = so.minimize(lambda v: fun(v)[0], x0, jac=lambda v: fun(v)[1], method="L-BFGS-B",
                        bounds=list(zip(lb, ub)), options={"ftol": 1e7 * np.finfo(float).eps, "gtol": 1e-5})
        assert np.max(np.abs(x - r.x)) < 2e-4, (x, r.x)
        assert abs(f - r.fun) < 1e-8 * max(1.0, abs(r.fun))


def test_lbfgsb3_on_the_shift_cost(O, S):
    """-gencorr_for_rot_8 at a fixed rotation: the same converged shift as SciPy's L-BFGS-B"""
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    rng = np.random.default_rng(11)
    ref = (rng.standard_normal((g.K, g.pftsz)) + 1j * rng.standard_normal((g.K, g.pftsz))).astype(np.complex64)
    sh = O.shmat(g, t, 0.8, -0.6)
    ptcl = (ref * sh + 0.3 * (rng.standard_normal(ref.shape) + 1j * rng.standard_normal(ref.shape))).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=2.0, dfy=1.95, angast=20.0))

    def fg(x):
        f, g3 = O.gencorr_grad3(g, t, ref, ptcl, 1, ctf, None, np.asarray(x, np.float64), False)
        return -f, -g3[:2]

    lb, ub = [-3.0, -3.0], [3.0, 3.0]
    for x0 in ([0.0, 0.0], [-1.5, 1.0]):
        x, f, n = run_lb3(S, fg, x0, lb, ub)
        r = so.minimize(lambda v: fg(v)[0], x0, jac=lambda v: fg(v)[1], method="L-BFGS-B",
                        bounds=list(zip(lb, ub)), options={"ftol": 1e7 * np.finfo(float).eps, "gtol": 1e-5})
        assert np.max(np.abs(x - r.x)) < 1e-3
        assert abs(f - r.fun) < 1e-7
        assert n < 60


def test_shift_search_recovers_rotation_and_shift(O, S):
    """a rotated, shifted copy of the reference: minimize (opt_angle) and minimize_exhaustive
    find irot = j + 1, cc ~ 1, and a shift whose phases undo the particle's"""
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    P = g.pftsz
    rng = np.random.default_rng(5)
    ref = (rng.standard_normal((g.K, P)) + 1j * rng.standard_normal((g.K, P))).astype(np.complex64)
    j = 9
    tx, ty = 0.7, -1.1
    # the reference prepared at shift (tx, ty) and rotated by j samples (conjugate wrap at P)
    prep = ref * O.shmat(g, t, tx, ty)
    ext = np.concatenate([prep, np.conj(prep)], axis=1)
    ptcl = np.roll(ext, j, axis=1)[:, :P].astype(np.complex64)
    lims = [[-3.0, 3.0], [-3.0, 3.0]]
    ss = S.ShiftSearch(g, t, ref, ptcl, None, lims, opt_angle=True)
    irot, cxy = ss.minimize()
    assert irot == j + 1
    assert cxy[0] > 0.9999
    # the shift found in the search frame (before the rotation into the reference frame)
    assert np.max(np.abs(ss.x - np.array([tx, ty], np.float32))) < 2e-3
    ex = S.ShiftSearch(g, t, ref, ptcl, None, lims, opt_angle=True)
    irot2, cxy2, better = ex.minimize_exhaustive(0)
    assert irot2 == j + 1 and cxy2[0] > 0.9999
    assert np.max(np.abs(cxy2[1:] - cxy[1:])) < 2e-3
    # the rotation into the reference frame is rotmat2d(get_rot(irot)) applied as matmul(v, R)
    a = ss.angtab[irot - 1] * np.float32(math.pi) / np.float32(180.0)
    c, s = np.cos(a), np.sin(a)
    assert np.allclose(cxy[1:], [ss.x[0] * c - ss.x[1] * s, ss.x[0] * s + ss.x[1] * c], atol=1e-6)


def test_fixed_angle_search_and_coarse_grid(O, S):
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    rng = np.random.default_rng(6)
    ref = (rng.standard_normal((g.K, g.pftsz)) + 1j * rng.standard_normal((g.K, g.pftsz))).astype(np.complex64)
    ptcl = (ref * O.shmat(g, t, -1.4, 0.9)).astype(np.complex64)
    ss = S.ShiftSearch(g, t, ref, ptcl, None, [[-3.0, 3.0], [-3.0, 3.0]], opt_angle=False)
    irot, cxy = ss.minimize(irot=1)
    assert irot == 1 and cxy[0] > 0.9999
    assert np.max(np.abs(ss.x - np.array([-1.4, 0.9], np.float32))) < 2e-3
    # with the coarse grid the search starts at the grid's best, (-1.2, 1.2); whatever the
    # optimiser then does, the answer is never worse than that start
    ss = S.ShiftSearch(g, t, ref, ptcl, None, [[-3.0, 3.0], [-3.0, 3.0]], opt_angle=False, coarse_init=True)
    irot, cxy = ss.minimize(irot=1)
    start = ss.for_rot(np.array([-1.2, 1.2]), 1)[0]
    assert irot == 0 or cxy[0] >= np.float32(start)
    # already at the optimum: nothing better is found
    ss = S.ShiftSearch(g, t, ref, ref, None, [[-3.0, 3.0], [-3.0, 3.0]], opt_angle=False)
    irot, cxy = ss.minimize(irot=1)
    assert irot == 0 and cxy is None


def test_first_step_at_the_step_bound(O, S):
    """L-BFGS-B bounds the first line search's step by 1 (lnsrlb) and the reference asks for
    the strong Wolfe curvature |g'| <= 1e-3 |g'(0)| (simple_pftcc_shsrch_grad.f90:67).  When
    the full first step still descends steeply enough to miss that but not steeply enough
    for the 'stp = stpmax' exit (g' <= ftol g'(0)), the More-Thuente search keeps proposing
    stp = 1 and L-BFGS-B abandons the run after 20 trials at its starting point -- the
    reference's own behaviour, restated.  With SciPy's line-search constants (1e-3, 0.9)
    the same start converges."""
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    rng = np.random.default_rng(6)
    ref = (rng.standard_normal((g.K, g.pftsz)) + 1j * rng.standard_normal((g.K, g.pftsz))).astype(np.complex64)
    ptcl = (ref * O.shmat(g, t, -1.4, 0.9)).astype(np.complex64)

    def fg(x):
        f, g3 = O.gencorr_grad3(g, t, ref, ptcl, 1, None, None, np.asarray(x, np.float64), False)
        return -f, -g3[:2]

    x, f, n = run_lb3(S, fg, [-1.0, 0.5], [-3.0, -3.0], [3.0, 3.0])
    assert np.array_equal(x, [-1.0, 0.5]) and n == 21
    x, f, n = run_lb3(S, fg, [-1.0, 0.5], [-3.0, -3.0], [3.0, 3.0], ftol=1e-3, gtol=0.9)
    assert np.max(np.abs(x - [-1.4, 0.9])) < 1e-3
