"""CPU restatement of the reference's in-plane shift search, TEST INFRASTRUCTURE ONLY
(the checker of pftcc_shsrch_batch in tests/).

Follows simple_pftcc_shsrch_grad.f90 routine by routine for one (reference, particle)
problem, with the oracle's FP64 correlations (oracle.gencorrs = gencorrs_cc_2,
oracle.gencorr_grad3 = gencorr_grad_for_rot_8 in the branch match_filt selects):
  grad_shsrch_minimize       :254-338  (minimize)
  minimize_exhaustive        :159-251  (minimize_exhaustive)
  coarse_search              :340-362
  coarse_search_opt_angle    :364-389
  grad_shsrch_optimize_angle :133-138  (the in-plane re-pick at every new iterate)
The optimiser is the library's L-BFGS-B header (simple3.0_b200/csrc/lbfgsb3.h, compiled
into oracle/_build/liblbfgsb3.so) stepped here in reverse communication the way
lbfgsb_minimize drives setulb (simple_opt_lbfgsb.f90:103-129); that optimiser is checked
against SciPy's L-BFGS-B separately (tests/test_shsrch_oracle.py).  Single-precision
quantities of the reference (ospec%x, the correlations of gencorrs, cxy) are rounded to
float32 where the reference holds them in single precision.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

import oracle as O

_HERE = os.path.dirname(os.path.abspath(__file__))
_lb = None

FG, NEW_X, CONVERGED, ABNORMAL = 0, 1, 2, 3


def _lib():
    global _lb
    if _lb is None:
        path = os.path.join(_HERE, "_build", "liblbfgsb3.so")
        if not os.path.exists(path):
            O.build()
        L = C.CDLL(path)
        dp = C.POINTER(C.c_double)
        L.lb3_new.argtypes = [dp, dp, dp, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
        L.lb3_new.restype = C.c_void_p
        for fn in ("lb3_free",):
            getattr(L, fn).argtypes = [C.c_void_p]
        for fn in ("lb3_task", "lb3_nfgv", "lb3_proceed"):
            getattr(L, fn).argtypes = [C.c_void_p]
            getattr(L, fn).restype = C.c_int
        L.lb3_f.argtypes = [C.c_void_p]
        L.lb3_f.restype = C.c_double
        L.lb3_x.argtypes = [C.c_void_p, dp]
        L.lb3_xt.argtypes = [C.c_void_p, dp]
        L.lb3_evaluated.argtypes = [C.c_void_p, C.c_double, dp]
        L.lb3_evaluated.restype = C.c_int
        _lb = L
    return _lb


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def f32(v):
    return float(np.float32(v))


class ShiftSearch:
    """pftcc_shsrch_grad for one (reference, particle): ref, ptcl (K, P), ctf (K, P) or None,
    lims [[x_lo, x_hi], [y_lo, y_hi]] (ospec%limits)"""

    def __init__(self, g, t, ref, ptcl, ctf, lims, maxits=100, opt_angle=True, coarse_init=False, max_evals=5,
                 match_filt=False):
        self.g, self.t, self.ref, self.ptcl, self.ctf = g, t, ref, ptcl, ctf
        self.lims = np.asarray(lims, np.float32)
        self.maxits, self.opt_angle, self.coarse_init, self.max_evals = maxits, opt_angle, coarse_init, max_evals
        self.match_filt = match_filt
        self.nrots = g.nrots
        self.cur = 0
        self.x = np.zeros(2, np.float32)          # ospec%x
        self.nevals = 0
        self.ncycles = 0
        # angtab (:261-273): real(irot-1)*twopi/real(nrots) in radians, then rad2deg, single precision
        pif = np.float32(math.acos(-1.0))
        ang = np.float32(np.float32(2.0) * pif) / np.float32(g.nrots)
        self.angtab = ((np.arange(g.nrots, dtype=np.float32) * ang) / pif * np.float32(180.0)).astype(np.float32)

    # ---- the correlator calls
    def gencorrs(self, sx, sy):
        """gencorrs(ref, ptcl, [sx, sy]) as the single-precision array the reference returns"""
        cc = O.gencorrs(self.g, self.t, self.ref, self.ptcl, self.ctf, np.array([f32(sx), f32(sy)], np.float64))
        return cc.astype(np.float32)

    def for_rot(self, x, irot):
        """(f, grad) = gencorr_grad_for_rot_8 at irot"""
        f, g3 = O.gencorr_grad3(self.g, self.t, self.ref, self.ptcl, irot, self.ctf, None,
                                np.asarray(x, np.float64), self.match_filt)
        return f, g3[:2]

    @staticmethod
    def maxloc(a, mask=None):
        """Fortran maxloc: the first index of the maximum, 1-based"""
        if mask is not None:
            a = np.where(mask, a, -np.inf)
        return int(np.argmax(a)) + 1

    # ---- lbfgsb_minimize (simple_opt_lbfgsb.f90:60-129) with the opt_callback
    def nlopt_minimize(self):
        L = _lib()
        x0 = self.x.astype(np.float64)                 # spec%x_8 = spec%x
        lb = self.lims[:, 0].astype(np.float64)
        ub = self.lims[:, 1].astype(np.float64)
        h = L.lb3_new(_dp(x0), _dp(lb), _dp(ub), 1e7, 1e-5, 1e-1, 1e-3, 0.1, 15)
        try:
            xt = np.zeros(2)
            task = L.lb3_task(h)
            while True:
                if task == FG:
                    L.lb3_xt(h, _dp(xt))
                    f, gr = self.for_rot(xt, self.cur)
                    self.nevals += 1
                    task = L.lb3_evaluated(h, -f, _dp(np.ascontiguousarray(-gr)))
                elif task == NEW_X:
                    if self.opt_angle:                  # grad_shsrch_optimize_angle (:133-138)
                        L.lb3_x(h, _dp(xt))
                        corrs = self.gencorrs(xt[0], xt[1])
                        self.cur = self.maxloc(corrs)
                    if L.lb3_nfgv(h) > self.maxits:
                        break
                    task = L.lb3_proceed(h)
                else:
                    break
            L.lb3_x(h, _dp(xt))
            self.x = xt.astype(np.float32)              # spec%x = real(spec%x_8)
            self.ncycles += 1
            return f32(L.lb3_f(h))                      # lowest_cost = real(self%f)
        finally:
            L.lb3_free(h)

    def rotate(self, irot, v):
        """matmul(v, rotmat2d(get_rot(irot))) in single precision (simple_math.f90:1550-1559)"""
        a = np.float32(self.angtab[irot - 1]) * np.float32(math.pi) / np.float32(180.0)
        c, s = np.cos(a, dtype=np.float32), np.sin(a, dtype=np.float32)
        x, y = np.float32(v[0]), np.float32(v[1])
        return np.array([x * c - y * s, x * s + y * c], np.float32)

    def coarse_points(self):
        lo, hi = self.lims[:, 0].astype(np.float64), self.lims[:, 1].astype(np.float64)
        stepx = float(np.float32(self.lims[0, 1] - self.lims[0, 0])) / 5.0
        stepy = float(np.float32(self.lims[1, 1] - self.lims[1, 0])) / 5.0
        for ix in range(5):
            for iy in range(5):
                yield lo[0] + stepx / 2.0 + ix * stepx, lo[1] + stepy / 2.0 + iy * stepy

    # ---- grad_shsrch_minimize (:254-338)
    def minimize(self, irot=0):
        """returns (irot, cxy[3]) with irot = 0 when nothing better was found"""
        found_better = False
        if self.opt_angle:
            self.x = np.zeros(2, np.float32)
            corrs = self.gencorrs(0.0, 0.0)
            self.cur = self.maxloc(corrs)
            lowest_cost_overall = -float(corrs[self.cur - 1])
            if self.coarse_init:                        # coarse_search_opt_angle (:364-389)
                lowest, init_xy, init_rot = math.inf, (0.0, 0.0), 0
                for x, y in self.coarse_points():
                    c = self.gencorrs(x, y)
                    loc = self.maxloc(c)
                    cost = -float(c[loc - 1])
                    if cost < lowest:
                        lowest, init_xy, init_rot = cost, (x, y), loc
                if init_rot != 0:
                    self.x = np.array(init_xy, np.float32)
                    self.cur = init_rot
            for _ in range(self.max_evals):
                self.nlopt_minimize()
                corrs = self.gencorrs(self.x[0], self.x[1])
                loc = self.maxloc(corrs)
                if loc == self.cur:
                    break
                self.cur = loc
            lowest_cost = -float(corrs[self.cur - 1])
            if lowest_cost < lowest_cost_overall:
                return self.cur, np.concatenate([[np.float32(-lowest_cost)], self.rotate(self.cur, self.x)])
            return 0, None
        self.cur = irot
        self.x = np.zeros(2, np.float32)
        lowest_cost_overall = -self.for_rot(np.zeros(2), irot)[0]
        if self.coarse_init:                            # coarse_search (:340-362)
            lowest, init_xy = math.inf, (0.0, 0.0)
            for x, y in self.coarse_points():
                cost = -self.for_rot(np.array([x, y]), self.cur)[0]
                if cost < lowest:
                    lowest, init_xy = cost, (x, y)
            if lowest < lowest_cost_overall:
                lowest_cost_overall = lowest
                self.x = np.array(init_xy, np.float32)
        lowest_cost = self.nlopt_minimize()
        if lowest_cost < lowest_cost_overall:
            found_better = True
        if found_better:
            return irot, np.concatenate([[np.float32(-lowest_cost)], self.rotate(irot, self.x)])
        return 0, None

    # ---- minimize_exhaustive (:159-251)
    def minimize_exhaustive(self, irot=0, halfrot=None):
        if irot <= 0:
            irot = 1                                    # get_roind(0.)
        mask = None
        if halfrot is not None and halfrot > 0:
            dang = np.abs(self.angtab - self.angtab[irot - 1])
            dang = np.where(dang > 180.0, np.abs(dang - np.float32(360.0)), dang)
            mask = dang <= np.float32(halfrot)
        lims = self.lims
        nstepx = max(1, int(math.floor(np.float32(lims[0, 1] - lims[0, 0]) / np.float32(4.0))))
        nstepy = max(1, int(math.floor(np.float32(lims[1, 1] - lims[1, 0]) / np.float32(4.0))))
        stepx = np.float32(np.float32(lims[0, 1] - lims[0, 0]) / np.float32(2 * nstepx + 1))
        stepy = np.float32(np.float32(lims[1, 1] - lims[1, 0]) / np.float32(2 * nstepy + 1))
        optcc = -math.inf
        coarse = np.zeros(2, np.float32)
        for i in range(-nstepx, nstepx + 1):
            sx = np.float32(i) * stepx
            for j in range(-nstepy, nstepy + 1):
                sy = np.float32(j) * stepy
                c = self.gencorrs(sx, sy)
                loc = self.maxloc(c, mask)
                if float(c[loc - 1]) > optcc:
                    irot, optcc, coarse = loc, float(c[loc - 1]), np.array([sx, sy], np.float32)
        for frac in (np.float32(2.0), np.float32(4.0)):
            shift = coarse.copy()
            for i in (-1, 0, 1):
                sx = coarse[0] + np.float32(i) * stepx / frac
                for j in (-1, 0, 1):
                    if i == 0 and j == 0:
                        continue
                    sy = coarse[1] + np.float32(j) * stepy / frac
                    c = self.gencorrs(sx, sy)
                    loc = self.maxloc(c, mask)
                    if float(c[loc - 1]) > optcc:
                        irot, optcc, shift = loc, float(c[loc - 1]), np.array([sx, sy], np.float32)
            coarse = shift
        self.cur = irot
        self.x = coarse.copy()
        lowest_cost_overall = f32(-self.for_rot(self.x.astype(np.float64), self.cur)[0])
        lowest_cost = self.nlopt_minimize()
        found_better = False
        if lowest_cost < lowest_cost_overall:
            lowest_cost_overall = lowest_cost
            xy = self.x
            found_better = True
        else:
            xy = coarse
        return irot, np.concatenate([[np.float32(-lowest_cost_overall)], self.rotate(irot, xy)]), found_better
