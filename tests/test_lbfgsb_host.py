"""Host (CPU) tests of the refinement's optimiser, the batched bound-constrained L-BFGS
of simple3.0_b200/csrc/lbfgsb.h, built here with g++ through tests/lbfgsb_host.cpp:

* a convex quadratic with active bounds reaches its KKT point (found by enumerating the
  active sets);
* the 3-D Rosenbrock function inside a box reaches (1, 1, 1);
* every problem's result is identical whether it runs alone or in a batch;
* on the correlation itself (the oracle's FP64 gencorr and adjoint, config-0 particles),
  refinement from shifts 1 px off, each problem in its own box, reaches the maximum of an
  exhaustive grid over the same box.
"""
import ctypes as C
import itertools
import math
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "simple3.0_b200", "csrc")
EVAL = C.CFUNCTYPE(C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double),
                   C.POINTER(C.c_double))


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("lbfgsb") / "liblbfgsb_host.so")
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, "-o", out,
                    os.path.join(HERE, "lbfgsb_host.cpp")], check=True)
    L = C.CDLL(out)
    _dp, _ip = C.POINTER(C.c_double), C.POINTER(C.c_int)
    L.lbfgsb_run.argtypes = [C.c_int, _dp, _dp, _dp, C.c_int, C.c_double, C.c_double, EVAL, _dp, _dp, _ip, _ip, _ip]
    L.lbfgsb_run.restype = C.c_int
    return L


def run(L, fg, x0, lb, ub, maxits=100, pgtol=1e-5, factr=1e7):
    """minimise fg(i, x) -> (f, g) for every problem i; returns x, f, nevals, niter, converged"""
    x0 = np.ascontiguousarray(x0, np.float64).reshape(-1, 3)
    n = x0.shape[0]
    lb = np.ascontiguousarray(np.broadcast_to(np.asarray(lb, np.float64), (n, 3)))
    ub = np.ascontiguousarray(np.broadcast_to(np.asarray(ub, np.float64), (n, 3)))

    def cb(nb, idx, xt, f, g):
        for b in range(nb):
            fv, gv = fg(idx[b], np.array([xt[3 * b + v] for v in range(3)]))
            f[b] = fv
            for v in range(3):
                g[3 * b + v] = gv[v]
        return 0

    c_cb = EVAL(cb)
    x = np.zeros((n, 3))
    f = np.zeros(n)
    nev, nit, conv = (np.zeros(n, np.int32) for _ in range(3))
    ptr = lambda a, t: a.ctypes.data_as(C.POINTER(t))
    st = L.lbfgsb_run(n, ptr(x0, C.c_double), ptr(lb, C.c_double), ptr(ub, C.c_double), maxits, pgtol, factr, c_cb,
                      ptr(x, C.c_double), ptr(f, C.c_double), ptr(nev, C.c_int), ptr(nit, C.c_int), ptr(conv, C.c_int))
    assert st == 0
    return x, f, nev, nit, conv.astype(bool)


def kkt_quadratic(A, c, lb, ub):
    """minimiser of 0.5 (x-c)^T A (x-c) over the box by enumerating the active sets"""
    best = None
    for act in itertools.product((0, 1, 2), repeat=3):   # 0 free, 1 at lb, 2 at ub
        act = np.array(act)
        x = np.where(act == 1, lb, np.where(act == 2, ub, 0.0))
        F, X = np.flatnonzero(act == 0), np.flatnonzero(act != 0)
        if F.size:
            # stationarity over the free block: A_FF (x_F - c_F) + A_FX (x_X - c_X) = 0
            x[F] = c[F] - np.linalg.solve(A[np.ix_(F, F)], A[np.ix_(F, X)] @ (x[X] - c[X]))
        if np.any(x < lb - 1e-12) or np.any(x > ub + 1e-12):
            continue
        fv = 0.5 * (x - c) @ A @ (x - c)
        if best is None or fv < best[1]:
            best = (x, fv)
    return best


def test_quadratic_with_active_bounds(lib):
    rng = np.random.default_rng(0)
    for trial in range(20):
        M = rng.normal(size=(3, 3))
        A = M @ M.T + 0.5 * np.eye(3)
        c = rng.uniform(-3, 3, 3)
        lb, ub = np.array([-1.0, -2.0, -0.5]), np.array([1.0, 0.5, 2.0])
        xs, fs = kkt_quadratic(A, c, lb, ub)
        fg = lambda i, x: (0.5 * (x - c) @ A @ (x - c), A @ (x - c))
        x, f, nev, nit, conv = run(lib, fg, rng.uniform(lb, ub), lb, ub, pgtol=1e-9, factr=10.0)
        assert np.max(np.abs(x[0] - xs)) < 1e-5, (trial, x[0], xs)
        assert f[0] <= fs + 1e-9


def rosen(i, x):
    f = sum(100.0 * (x[j + 1] - x[j] ** 2) ** 2 + (1 - x[j]) ** 2 for j in range(2))
    g = np.zeros(3)
    for j in range(2):
        g[j] += -400.0 * x[j] * (x[j + 1] - x[j] ** 2) - 2 * (1 - x[j])
        g[j + 1] += 200.0 * (x[j + 1] - x[j] ** 2)
    return f, g


def test_rosenbrock_in_box(lib):
    x, f, nev, nit, conv = run(lib, rosen, [[-1.2, 1.0, 0.5], [0.0, 0.0, 0.0]], [-2, -2, -2], [2, 2, 2],
                               maxits=500, pgtol=1e-8, factr=10.0)
    assert np.max(np.abs(x - 1.0)) < 1e-4
    assert np.all(conv)


def test_batch_independence(lib):
    rng = np.random.default_rng(1)
    x0 = rng.uniform(-1.5, 1.5, (6, 3))
    lb, ub = x0 - 1.0, x0 + 1.0
    xb, fb, nb, ib, cb = run(lib, rosen, x0, lb, ub, maxits=200)
    for i in range(6):
        xa, fa, na, ia, ca = run(lib, rosen, x0[i], lb[i], ub[i], maxits=200)
        assert np.array_equal(xa[0], xb[i]) and fa[0] == fb[i] and na[0] == nb[i]


def test_refine_correlation_reaches_grid_maximum(lib, pkg, O):
    """shift + defocus refinement of config-0 problems against the oracle's FP64 gencorr
    and adjoint; the exhaustive grid (0.1 px, 0.02 micron) of the same box bounds what the
    refinement must reach"""
    n = 4
    w = pkg.synth.config0(nrefs=3, nptcls=n)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R, noise=False)
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    rng = np.random.default_rng(9)
    probs, x0 = [], []
    for i in range(n):
        psi = math.radians(parts.psi[i])
        tx, ty = parts.shift[i]
        irot = int(round(parts.psi[i] * w.nrots / 360.0)) % w.nrots + 1
        sh = (-(math.cos(psi) * tx + math.sin(psi) * ty), -(-math.sin(psi) * tx + math.cos(psi) * ty))
        probs.append((irot, O.polarize(g, t, parts.cmat[i].numpy()), refs[parts.ref[i]].numpy()))
        x0.append([sh[0] + rng.uniform(-1, 1), sh[1] + rng.uniform(-1, 1), 0.0])
    x0 = np.array(x0)
    half = np.array([1.0, 1.0, 0.1])

    def corr_grad(i, x):
        irot, pft, ref = probs[i]
        cp = O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]) + x[2], float(parts.dfy[i]) + x[2],
                        float(parts.angast[i]))
        return O.gencorr_grad3(g, t, ref, pft, irot, O.ctfmat(g, t, cp), O.dctfmat_ddf(g, t, cp), x[:2], False)

    def fg(i, x):
        f, gr = corr_grad(i, x)
        return -f, -np.asarray(gr)

    x, f, nev, nit, conv = run(lib, fg, x0, x0 - half, x0 + half)
    gx = np.arange(-10, 11) * 0.1
    gd = np.arange(-5, 6) * 0.02
    for i in range(n):
        best = max(corr_grad(i, x0[i] + np.array([a, b, d]))[0] for a in gx for b in gx for d in gd)
        assert -f[i] >= best - 1e-4, (i, -f[i], best, x[i], nev[i])
