"""Host-side mirror of SIMPLE 3.0's ``polarft_corrcalc`` over libpftcc_b200.so.

The class keeps the reference's procedure names, argument meaning, 1-based
indices and error behaviour (the reference's THROW_HARD stops the program; here
a :class:`PftccError` is raised), so code written against the reference's
operator surface reads the same:

    pftcc = polarft_corrcalc()
    pftcc.new(nrefs, [fromp, top], box=128, nrots=360, kfromto=(2, 40))
    pftcc.set_ref_pft(iref, pft, iseven=True)
    pftcc.set_ptcl_pft(iptcl, pft)
    pftcc.create_polar_absctfmats(ctfparams)
    cc = pftcc.gencorrs(iref, iptcl, shvec)

A polar FT is a complex64 numpy array of shape (K, P) = (kto-kfrom+1, nrots/2),
i.e. the memory layout of the reference's Fortran pft(P, kfrom:kto).  Every
computation runs in the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib

FRAME_REF, FRAME_PTCL = _lib.FRAME_REF, _lib.FRAME_PTCL
PREC_EXACT, PREC_FP32, PREC_BF16X3 = _lib.PREC_EXACT, _lib.PREC_FP32, _lib.PREC_BF16X3
_FRAMES = {"ref": FRAME_REF, "ptcl": FRAME_PTCL, FRAME_REF: FRAME_REF, FRAME_PTCL: FRAME_PTCL}
_PRECS = {"exact": PREC_EXACT, "fp32": PREC_FP32, "bf16x3": PREC_BF16X3,
          PREC_EXACT: PREC_EXACT, PREC_FP32: PREC_FP32, PREC_BF16X3: PREC_BF16X3}


_GRAD_REQ = np.dtype([("iref", "<i4"), ("iptcl", "<i4"), ("irot", "<i4"), ("pad", "<i4"),
                      ("sx", "<f8"), ("sy", "<f8"), ("ddf", "<f8")])
assert _GRAD_REQ.itemsize == C.sizeof(_lib.GradReq)


class PftccError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"pftcc error {status}: {msg}")
        self.status = status


def _f32p(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _cplx(a, shape=None) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.complex64)
    if shape is not None and a.shape != tuple(shape):
        raise PftccError(_lib.ERR_ARG, f"expected a polar FT of shape {tuple(shape)}, got {a.shape}")
    return a


def ctfparams_array(n, smpd=1.3, kv=300.0, cs=2.7, fraca=0.1, dfx=None, dfy=None, angast=None,
                    phshift=0.0, l_phaseplate=False):
    """per-particle CTF parameters (spproj%get_ctfparams) as a ctypes array"""
    arr = (_lib.CtfParams * n)()
    dfx = np.broadcast_to(np.asarray(2.0 if dfx is None else dfx, np.float32), (n,))
    dfy = np.broadcast_to(np.asarray(dfx if dfy is None else dfy, np.float32), (n,))
    ang = np.broadcast_to(np.asarray(0.0 if angast is None else angast, np.float32), (n,))
    for i in range(n):
        arr[i] = _lib.CtfParams(smpd, kv, cs, fraca, float(dfx[i]), float(dfy[i]), float(ang[i]), phshift,
                                int(l_phaseplate))
    return arr


class polarft_corrcalc:
    """B200 implementation of the polarft_corrcalc operator (simple_polarft_corrcalc.f90:68-198)."""

    def __init__(self):
        self._h = None
        self._L = _lib.load()

    # ---- helpers ------------------------------------------------------------------------
    def _check(self, st: int):
        if st != _lib.OK:
            msg = self._L.pftcc_last_error(self._h).decode() if self._h else self._L.pftcc_strerror(st).decode()
            raise PftccError(st, msg or self._L.pftcc_strerror(st).decode())

    def _geti(self, fn) -> int:
        v = C.c_int()
        self._check(fn(self._h, C.byref(v)))
        return v.value

    @property
    def handle(self):
        return self._h

    # ---- CONSTRUCTOR -----------------------------------------------------------------------
    def new(self, nrefs: int, pfromto, *, box: int, nrots: int, kfromto, kstop: int | None = None,
            ctf: bool = True, match_filt: bool = False, ctf_frame="ref", ptcl_mask=None, eoarr=None,
            device: int = 0):
        """new(nrefs, pfromto, ptcl_mask, eoarr) with the params_glob fields passed explicitly."""
        self.kill()
        cfg = _lib.Config()
        cfg.nrefs = int(nrefs)
        cfg.pfromto[0], cfg.pfromto[1] = int(pfromto[0]), int(pfromto[1])
        cfg.box, cfg.nrots = int(box), int(nrots)
        cfg.kfromto[0], cfg.kfromto[1] = int(kfromto[0]), int(kfromto[1])
        cfg.kstop = int(kfromto[1] if kstop is None else kstop)
        cfg.with_ctf, cfg.match_filt = int(bool(ctf)), int(bool(match_filt))
        cfg.ctf_frame = _FRAMES[ctf_frame]
        cfg.device = int(device)
        span = cfg.pfromto[1] - cfg.pfromto[0] + 1
        mask = None if ptcl_mask is None else np.ascontiguousarray(np.asarray(ptcl_mask, bool).astype(np.int32))
        eo = None if eoarr is None else np.ascontiguousarray(eoarr, np.int32)
        for a in (mask, eo):
            if a is not None and a.size != span:
                raise PftccError(_lib.ERR_ARG, "ptcl_mask/eoarr must cover pfromto")
        h = C.c_void_p()
        st = self._L.pftcc_new(C.byref(cfg), None if mask is None else mask.ctypes.data_as(C.POINTER(C.c_int)),
                               None if eo is None else eo.ctypes.data_as(C.POINTER(C.c_int)), C.byref(h))
        if st != _lib.OK:
            raise PftccError(st, self._L.pftcc_strerror(st).decode())
        self._h = h
        self.cfg = cfg
        self.K = cfg.kfromto[1] - cfg.kfromto[0] + 1
        self.P = cfg.nrots // 2
        return self

    def kill(self):
        if self._h:
            self._L.pftcc_kill(self._h)
            self._h = None

    def __del__(self):
        try:
            self.kill()
        except Exception:
            pass

    def exists(self) -> bool:
        return self._h is not None

    # ---- SETTERS ----------------------------------------------------------------------------
    def reallocate_ptcls(self, nptcls: int, pinds):
        p = np.ascontiguousarray(pinds, np.int32)
        self._check(self._L.pftcc_reallocate_ptcls(self._h, int(nptcls), p.ctypes.data_as(C.POINTER(C.c_int))))

    def set_ref_pft(self, iref: int, pft, iseven: bool):
        a = _cplx(pft, (self.K, self.P))
        self._check(self._L.pftcc_set_ref_pft(self._h, int(iref), _f32p(a.view(np.float32)), int(bool(iseven))))

    def set_refs(self, first_iref: int, pfts, iseven: bool):
        a = _cplx(pfts)
        self._check(self._L.pftcc_set_refs(self._h, int(first_iref), a.shape[0], _f32p(a.view(np.float32)),
                                           int(bool(iseven))))

    def set_ptcl_pft(self, iptcl: int, pft):
        a = _cplx(pft, (self.K, self.P))
        self._check(self._L.pftcc_set_ptcl_pft(self._h, int(iptcl), _f32p(a.view(np.float32))))

    def set_ptcls(self, first_slot: int, pfts):
        a = _cplx(pfts)
        self._check(self._L.pftcc_set_ptcls(self._h, int(first_slot), a.shape[0], _f32p(a.view(np.float32))))

    def set_ref_fcomp(self, iref: int, irot: int, k: int, comp: complex, iseven: bool):
        a = np.asarray([comp], np.complex64)
        self._check(self._L.pftcc_set_ref_fcomp(self._h, int(iref), int(irot), int(k), _f32p(a.view(np.float32)),
                                                int(bool(iseven))))

    def cp_even2odd_ref(self, iref: int):
        self._check(self._L.pftcc_cp_even2odd_ref(self._h, int(iref)))

    def cp_even_ref2ptcl(self, iref: int, iptcl: int):
        self._check(self._L.pftcc_cp_even_ref2ptcl(self._h, int(iref), int(iptcl)))

    def swap_ptclsevenodd(self):
        self._check(self._L.pftcc_swap_ptclsevenodd(self._h))

    def set_eo(self, iptcl: int, is_even: bool):
        self._check(self._L.pftcc_set_eo(self._h, int(iptcl), int(bool(is_even))))

    def set_eos(self, eoarr):
        e = np.ascontiguousarray(eoarr, np.int32)
        self._check(self._L.pftcc_set_eos(self._h, e.ctypes.data_as(C.POINTER(C.c_int))))

    def zero_refs_beyond_kstop(self):
        self._check(self._L.pftcc_zero_refs_beyond_kstop(self._h))

    # ---- CTF / memoisers -------------------------------------------------------------------
    def create_polar_absctfmats(self, ctfparams):
        """ctfparams: ctypes array of CtfParams, one per held particle slot (see ctfparams_array)"""
        self._check(self._L.pftcc_create_polar_absctfmats(self._h, ctfparams))

    def memoize_ffts(self):
        self._check(self._L.pftcc_memoize_ffts(self._h))

    # ---- polarizer (simple_polarizer.f90) ----------------------------------------------------
    def polarize_ptcls(self, first_slot: int, cmats, griddev: bool = False):
        """cmats: complex64 (n, box, box//2+1) = image%cmat(box/2+1, box) per image"""
        a = np.ascontiguousarray(cmats, np.complex64)
        self._check(self._L.pftcc_polarize_ptcls(self._h, int(first_slot), a.shape[0], _f32p(a.view(np.float32)),
                                                 int(bool(griddev))))

    def polarize_ptcls_dev(self, first_slot: int, n: int, dev_ptr: int, griddev: bool = False):
        self._check(self._L.pftcc_polarize_ptcls_dev(self._h, int(first_slot), int(n), C.c_void_p(dev_ptr),
                                                     int(bool(griddev))))

    def polarize_refs(self, first_iref: int, cmats, iseven: bool, griddev: bool = False):
        a = np.ascontiguousarray(cmats, np.complex64)
        self._check(self._L.pftcc_polarize_refs(self._h, int(first_iref), a.shape[0], _f32p(a.view(np.float32)),
                                                int(bool(iseven)), int(bool(griddev))))

    # ---- PROJECTOR (simple_projector.f90) ---------------------------------------------------
    def set_volume_ft(self, cmat_half, factor: float = 1.0):
        """expand_cmat: cmat_half complex64 (box, box, box//2+1) = image%cmat(h, k, m) in [m][k][h]
        order (the Fortran array's memory order)"""
        a = np.ascontiguousarray(cmat_half, np.complex64)
        box = a.shape[0]
        if a.shape != (box, box, box // 2 + 1):
            raise ValueError("set_volume_ft: expected (box, box, box//2+1)")
        self._check(self._L.pftcc_set_volume_ft(self._h, _f32p(a.view(np.float32)), int(box), float(factor)))

    def fproject_polar(self, first_iref: int, euls, iseven: bool = True, mask=None, griddev: bool = False):
        """fproject_polar for len(euls) orientations (Spider Euler triplets, degrees) into
        references first_iref.. (1-based); mask: K booleans for shells kfrom..kto or None"""
        e = np.ascontiguousarray(euls, np.float32).reshape(-1, 3)
        m = None
        if mask is not None:
            m = np.ascontiguousarray(np.asarray(mask, bool).astype(np.int32))
            if m.shape != (self.cfg.kfromto[1] - self.cfg.kfromto[0] + 1,):
                raise ValueError("fproject_polar: mask needs one entry per shell kfrom..kto")
        self._check(self._L.pftcc_fproject_polar(self._h, int(first_iref), e.shape[0], _f32p(e.reshape(-1)),
                                                 None if m is None else m.ctypes.data_as(C.POINTER(C.c_int)),
                                                 int(bool(iseven)), int(bool(griddev))))

    def prep_ptcls(self, first_slot: int, imgs, xy=None, ctfflag=None, ctfparams=None, msk: float | None = None,
                   inner: float = 0.0, width: float = 0.0, focusmsk: float = 0.0, griddev: bool = False):
        """prepimg4align + polarize for images (n, box_in, box_in) [y][x] into slots first_slot..:
        xy (n, 2) the particles' shifts, ctfflag (n,) of _lib.CTFFLAG_*, ctfparams a ctypes array
        (ctfparams_array) needed where a flag is CTFFLAG_YES, msk the mask radius (pixels); inner
        (with width) the inner mask, focusmsk the focus mask, griddev 'yes' (pftcc_prep_opts)"""
        a = np.ascontiguousarray(imgs, np.float32)
        n, box_in = a.shape[0], a.shape[1]
        v = np.zeros((n, 2), np.float32) if xy is None else np.ascontiguousarray(xy, np.float32).reshape(n, 2)
        f = np.zeros(n, np.int32) if ctfflag is None else np.ascontiguousarray(ctfflag, np.int32).reshape(n)
        m = float(self.cfg.box / 2 - 4 if msk is None else msk)
        if inner or width or focusmsk or griddev:
            o = _lib.PrepOpts(m, float(inner), float(width), float(focusmsk), int(bool(griddev)))
            self._check(self._L.pftcc_prep_ptcls_opts(self._h, int(first_slot), n, _f32p(a), int(box_in), _f32p(v),
                                                      f.ctypes.data_as(C.POINTER(C.c_int)), ctfparams, C.byref(o)))
            return
        self._check(self._L.pftcc_prep_ptcls(self._h, int(first_slot), n, _f32p(a), int(box_in), _f32p(v),
                                             f.ctypes.data_as(C.POINTER(C.c_int)), ctfparams, m))

    def fdf_project_polar(self, first_iref: int, euls, iseven: bool = True):
        """projector%fdf_project_polar for n orientations (n, 3) in degrees: the sections into
        references first_iref.. and their Euler-angle derivatives into the derivative references"""
        e = np.ascontiguousarray(np.atleast_2d(euls), np.float64)
        self._check(self._L.pftcc_fdf_project_polar(self._h, int(first_iref), e.shape[0],
                                                    e.ctypes.data_as(C.POINTER(C.c_double)), int(bool(iseven))))

    def get_dref_pft(self, iref: int, iseven: bool = True) -> np.ndarray:
        """(3, K, P) derivatives of reference iref with respect to e1, e2, e3 (per radian)"""
        K = self.cfg.kfromto[1] - self.cfg.kfromto[0] + 1
        out = np.zeros((3, K, self.cfg.nrots // 2), np.complex64)
        self._check(self._L.pftcc_get_dref_pft(self._h, int(iref), int(bool(iseven)), _f32p(out.view(np.float32))))
        return out

    # ---- CALCULATORS -----------------------------------------------------------------------
    def gencorrs(self, iref: int, iptcl: int, shvec=None) -> np.ndarray:
        cc = np.zeros(self.cfg.nrots, np.float32)
        sh = None if shvec is None else np.ascontiguousarray(shvec, np.float32)
        self._check(self._L.pftcc_gencorrs(self._h, int(iref), int(iptcl), None if sh is None else _f32p(sh), _f32p(cc)))
        return cc

    def gencorrs_noalloc(self, iref, iptcl, shifts, cc_dev_ptr: int):
        """gencorrs for many pairs into a caller's device buffer (npairs * nrots floats) without
        any allocation by the library (fixed device scratch; see include/pftcc_b200.h)"""
        ir = np.ascontiguousarray(iref, np.int32)
        ip = np.ascontiguousarray(iptcl, np.int32)
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
        self._check(self._L.pftcc_gencorrs_noalloc(self._h, ir.size, ir.ctypes.data_as(C.POINTER(C.c_int)),
                                                   ip.ctypes.data_as(C.POINTER(C.c_int)),
                                                   None if sh is None else _f32p(sh), C.c_void_p(cc_dev_ptr)))

    def genfrc(self, iref: int, iptcl: int, irot: int, shvec=None) -> np.ndarray:
        """per-shell correlations k = kfrom..kstop at irot (genfrc, or calc_frc with shvec)"""
        frc = np.zeros(self.cfg.kstop - self.cfg.kfromto[0] + 1, np.float32)
        sh = None if shvec is None else np.ascontiguousarray(shvec, np.float32)
        self._check(self._L.pftcc_genfrc(self._h, int(iref), int(iptcl), int(irot), None if sh is None else _f32p(sh),
                                         _f32p(frc)))
        return frc

    def specscore(self, iref: int, iptcl: int, irot: int, shvec=None) -> float:
        """max(0, median shell correlation) at irot (specscore_1, or specscore_2 with shvec)"""
        out = C.c_float()
        sh = None if shvec is None else np.ascontiguousarray(shvec, np.float32)
        self._check(self._L.pftcc_specscore(self._h, int(iref), int(iptcl), int(irot),
                                            None if sh is None else _f32p(sh), C.byref(out)))
        return out.value

    def specscore_batch(self, iref, iptcl, irot, shifts=None, want_frc: bool = False):
        """specscores of many (iref, iptcl, irot) requests in one launch; with want_frc also
        their shell correlations (n, kstop-kfrom+1)"""
        ir, ip, ro = (np.ascontiguousarray(np.atleast_1d(v), np.int32) for v in (iref, iptcl, irot))
        n = ir.size
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(n, 2)
        scores = np.zeros(n, np.float32)
        frcs = np.zeros((n, self.cfg.kstop - self.cfg.kfromto[0] + 1), np.float32) if want_frc else None
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self._check(self._L.pftcc_specscore_batch(self._h, n, ptr(ir), ptr(ip), ptr(ro),
                                                  None if sh is None else _f32p(sh), _f32p(scores),
                                                  None if frcs is None else _f32p(frcs)))
        return (scores, frcs) if want_frc else scores

    # ---- remaining procedures ------------------------------------------------------------------
    def cp_refs(self, other: "polarft_corrcalc"):
        """both reference sets copied from another object of the same shape"""
        self._check(self._L.pftcc_cp_refs(self._h, other._h))

    def set_ptcl_fcomp(self, iptcl: int, irot: int, k: int, comp: complex):
        a = np.asarray([comp], np.complex64)
        self._check(self._L.pftcc_set_ptcl_fcomp(self._h, int(iptcl), int(irot), int(k), _f32p(a.view(np.float32))))

    def calc_ptcl_pspec(self, iptcl: int) -> np.ndarray:
        out = np.zeros(self.K, np.float32)
        self._check(self._L.pftcc_calc_ptcl_pspec(self._h, int(iptcl), _f32p(out)))
        return out

    def assign_pinds(self) -> np.ndarray:
        out = np.zeros(self.cfg.pfromto[1] - self.cfg.pfromto[0] + 1, np.int32)
        self._check(self._L.pftcc_assign_pinds(self._h, out.ctypes.data_as(C.POINTER(C.c_int))))
        return out

    def calc_roinv_corrmat(self) -> np.ndarray:
        n = self.get_nptcls()
        out = np.zeros((n, n), np.float32)
        self._check(self._L.pftcc_calc_roinv_corrmat(self._h, _f32p(out)))
        return out

    # ---- the matched-filter mode (new(..., match_filt=True)) ----------------------------------
    def set_pssnr(self, on: bool = True):
        """params_glob%l_pssnr within the matched-filter mode (pftcc_set_pssnr)"""
        self._check(self._L.pftcc_set_pssnr(self._h, int(bool(on))))

    def set_ref_optlp(self, iref: int, optlp):
        """ref_optlp(kfrom:kstop, iref) = optlp (the reference's matched filter)"""
        a = np.ascontiguousarray(optlp, np.float32)
        self._check(self._L.pftcc_set_ref_optlp(self._h, int(iref), _f32p(a)))

    def prep_matchfilt(self, iptcl: int, iref: int, irot: int):
        self._check(self._L.pftcc_prep_matchfilt(self._h, int(iptcl), int(iref), int(irot)))

    def prep_matchfilt_batch(self, iptcl, iref, irot):
        ip, ir, ro = (np.ascontiguousarray(np.atleast_1d(v), np.int32) for v in (iptcl, iref, irot))
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self._check(self._L.pftcc_prep_matchfilt_batch(self._h, ip.size, ptr(ip), ptr(ir), ptr(ro)))

    # ---- the Euclidean objective (params_glob%cc_objfun = OBJFUN_EUCLID) ---------------------
    def set_objfun(self, objfun: int):
        """cc_objfun: _lib.OBJFUN_CC or _lib.OBJFUN_EUCLID; gencorrs, gencorr_for_rot(_8),
        gencorr_grad(_only)_for_rot_8 and the exact batched searches follow it"""
        self._check(self._L.pftcc_set_objfun(self._h, int(objfun)))

    def assign_sigma2_noise(self, sigma2, fromp: int | None = None):
        """sigma2_noise(kfrom:kto, fromp:top) as an array (top - fromp + 1, K); fromp defaults
        to pfromto(1).  The values are copied."""
        a = np.ascontiguousarray(sigma2, np.float32)
        K = self.cfg.kfromto[1] - self.cfg.kfromto[0] + 1
        if a.ndim != 2 or a.shape[1] != K:
            raise PftccError(_lib.ERR_ARG, f"sigma2 must be (nptcls, {K}), got {a.shape}")
        lo = self.cfg.pfromto[0] if fromp is None else int(fromp)
        self._check(self._L.pftcc_assign_sigma2_noise(self._h, lo, lo + a.shape[0] - 1, _f32p(a)))

    def gencorrs_euclid(self, iref: int, iptcl: int, shvec=None) -> np.ndarray:
        out = np.zeros(self.cfg.nrots, np.float32)
        sh = None if shvec is None else np.ascontiguousarray(shvec, np.float32)
        self._check(self._L.pftcc_gencorrs_euclid(self._h, int(iref), int(iptcl), None if sh is None else _f32p(sh),
                                                  _f32p(out)))
        return out

    def gencorr_euclid_for_rot(self, iref: int, iptcl: int, shvec, irot: int) -> float:
        out = C.c_float()
        sh = np.ascontiguousarray(shvec, np.float32)
        self._check(self._L.pftcc_gencorr_euclid_for_rot(self._h, int(iref), int(iptcl), _f32p(sh), int(irot),
                                                         C.byref(out)))
        return out.value

    def gencorr_euclid_for_rot_8(self, iref: int, iptcl: int, shvec, irot: int) -> float:
        out = C.c_double()
        sh = np.ascontiguousarray(shvec, np.float64)
        self._check(self._L.pftcc_gencorr_euclid_for_rot_8(self._h, int(iref), int(iptcl),
                                                           sh.ctypes.data_as(C.POINTER(C.c_double)), int(irot),
                                                           C.byref(out)))
        return out.value

    def gencorr_euclid_grad_for_rot_8(self, iref: int, iptcl: int, shvec, irot: int):
        f = C.c_double()
        g = np.zeros(2, np.float64)
        sh = np.ascontiguousarray(shvec, np.float64)
        self._check(self._L.pftcc_gencorr_euclid_grad_for_rot_8(self._h, int(iref), int(iptcl),
                                                                sh.ctypes.data_as(C.POINTER(C.c_double)), int(irot),
                                                                C.byref(f), g.ctypes.data_as(C.POINTER(C.c_double))))
        return f.value, g

    def gencorr_euclid_grad_only_for_rot_8(self, iref: int, iptcl: int, shvec, irot: int):
        g = np.zeros(2, np.float64)
        sh = np.ascontiguousarray(shvec, np.float64)
        self._check(self._L.pftcc_gencorr_euclid_grad_only_for_rot_8(self._h, int(iref), int(iptcl),
                                                                     sh.ctypes.data_as(C.POINTER(C.c_double)),
                                                                     int(irot), g.ctypes.data_as(C.POINTER(C.c_double))))
        return g

    def gencorr_sigma_contrib(self, iref: int, iptcl: int, shvec, irot: int):
        """(sigma_contrib, ptcl_sumsq, ref_sumsq), each over the shells kfrom..kto"""
        K = self.cfg.kfromto[1] - self.cfg.kfromto[0] + 1
        sc, ps, rs = (np.zeros(K, np.float32) for _ in range(3))
        sh = np.ascontiguousarray(shvec, np.float32)
        self._check(self._L.pftcc_gencorr_sigma_contrib(self._h, int(iref), int(iptcl), _f32p(sh), int(irot),
                                                        _f32p(sc), _f32p(ps), _f32p(rs)))
        return sc, ps, rs

    def sigma_contrib_batch(self, iref, iptcl, irot, shifts):
        """sigma_contrib for many requests: (n, K) arrays (sigma_contrib, ptcl_sumsq, ref_sumsq)"""
        ir, ip, ro = (np.ascontiguousarray(np.atleast_1d(v), np.int32) for v in (iref, iptcl, irot))
        n = ir.size
        K = self.cfg.kfromto[1] - self.cfg.kfromto[0] + 1
        sh = np.ascontiguousarray(shifts, np.float32).reshape(n, 2)
        sc, ps, rs = (np.zeros((n, K), np.float32) for _ in range(3))
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self._check(self._L.pftcc_sigma_contrib_batch(self._h, n, ptr(ir), ptr(ip), ptr(ro), _f32p(sh), _f32p(sc),
                                                      _f32p(ps), _f32p(rs)))
        return sc, ps, rs

    def gencorr_for_rot(self, iref: int, iptcl: int, shvec, irot: int) -> float:
        out = C.c_float()
        sh = np.ascontiguousarray(shvec, np.float32)
        self._check(self._L.pftcc_gencorr_for_rot(self._h, int(iref), int(iptcl), _f32p(sh), int(irot), C.byref(out)))
        return out.value

    def gencorr_for_rot_8(self, iref: int, iptcl: int, shvec, irot: int) -> float:
        out = C.c_double()
        sh = np.ascontiguousarray(shvec, np.float64)
        self._check(self._L.pftcc_gencorr_for_rot_8(self._h, int(iref), int(iptcl),
                                                    sh.ctypes.data_as(C.POINTER(C.c_double)), int(irot), C.byref(out)))
        return out.value

    def gencorr_grad_for_rot_8(self, iref: int, iptcl: int, shvec, irot: int):
        f = C.c_double()
        g = np.zeros(2, np.float64)
        sh = np.ascontiguousarray(shvec, np.float64)
        self._check(self._L.pftcc_gencorr_grad_for_rot_8(self._h, int(iref), int(iptcl),
                                                         sh.ctypes.data_as(C.POINTER(C.c_double)), int(irot),
                                                         C.byref(f), g.ctypes.data_as(C.POINTER(C.c_double))))
        return f.value, g

    def gencorr_grad_only_for_rot_8(self, iref: int, iptcl: int, shvec, irot: int):
        g = np.zeros(2, np.float64)
        sh = np.ascontiguousarray(shvec, np.float64)
        self._check(self._L.pftcc_gencorr_grad_only_for_rot_8(self._h, int(iref), int(iptcl),
                                                              sh.ctypes.data_as(C.POINTER(C.c_double)), int(irot),
                                                              g.ctypes.data_as(C.POINTER(C.c_double))))
        return g

    # ---- batched entry points ----------------------------------------------------------------
    def corr_all(self, shifts=None) -> np.ndarray:
        """cc[slot, iref-1, ishift, irot-1] for every held particle, reference and shift"""
        n = self.get_nptcls()
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
        ns = 0 if sh is None else sh.shape[0]
        out = np.zeros((n, self.cfg.nrefs, max(1, ns), self.cfg.nrots), np.float32)
        self._check(self._L.pftcc_corr_all(self._h, ns, None if sh is None else _f32p(sh), _f32p(out)))
        return out

    def corr_all_prec(self, shifts=None, precision="fp32") -> np.ndarray:
        """all correlations through the m-domain path (particle frame), same layout as corr_all"""
        n = self.get_nptcls()
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
        ns = 0 if sh is None else sh.shape[0]
        out = np.zeros((n, self.cfg.nrefs, max(1, ns), self.cfg.nrots), np.float32)
        self._check(self._L.pftcc_corr_all_prec(self._h, ns, None if sh is None else _f32p(sh), _PRECS[precision],
                                                _f32p(out)))
        return out

    def search_best(self, shifts=None, precision="exact", ntop: int = 0) -> np.ndarray:
        """structured array (iref, irot, ishift, corr) per held particle slot"""
        n = self.get_nptcls()
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
        ns = 0 if sh is None else sh.shape[0]
        out = (_lib.Best * n)()
        self._check(self._L.pftcc_search_best(self._h, ns, None if sh is None else _f32p(sh), _PRECS[precision],
                                              int(ntop), out))
        dt = np.dtype([("iref", np.int32), ("irot", np.int32), ("ishift", np.int32), ("corr", np.float32)])
        return np.frombuffer(out, dtype=dt).copy()

    def search_groups(self, groups, shifts=None, precision="bf16x3", ntop: int = 8) -> np.ndarray:
        """pftcc_search_groups: groups is a sequence of (ref_first, nref, slot_first, nslot), 1-based;
        each group's particle slots are searched against its references only.  Structured array
        (iref, irot, ishift, corr) per held particle slot (iref 0 outside every group)."""
        n = self.get_nptcls()
        g = np.ascontiguousarray(np.asarray(groups, np.int32).reshape(-1, 4))
        cols = [np.ascontiguousarray(g[:, i]) for i in range(4)]
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
        ns = 0 if sh is None else sh.shape[0]
        out = (_lib.Best * n)()
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self._check(self._L.pftcc_search_groups(self._h, g.shape[0], ip(cols[0]), ip(cols[1]), ip(cols[2]), ip(cols[3]),
                                                ns, None if sh is None else _f32p(sh), _PRECS[precision], int(ntop), out))
        dt = np.dtype([("iref", np.int32), ("irot", np.int32), ("ishift", np.int32), ("corr", np.float32)])
        return np.frombuffer(out, dtype=dt).copy()

    def search_groups_dev(self, groups, shifts, precision, ntop: int, out_dev_ptr: int):
        """pftcc_search_groups_dev: the grouped search into device memory (nptcls 16-byte records at
        out_dev_ptr), enqueued on the handle's stream without synchronising; capturable in a CUDA
        graph after one uncaptured call with the same arguments"""
        g = np.ascontiguousarray(np.asarray(groups, np.int32).reshape(-1, 4))
        self._keep = [np.ascontiguousarray(g[:, i]) for i in range(4)]
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
        ns = 0 if sh is None else sh.shape[0]
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        k = self._keep
        self._check(self._L.pftcc_search_groups_dev(self._h, g.shape[0], ip(k[0]), ip(k[1]), ip(k[2]), ip(k[3]), ns,
                                                    None if sh is None else _f32p(sh), _PRECS[precision], int(ntop),
                                                    C.c_void_p(out_dev_ptr)))

    def search_check(self):
        """raise if a bounded wait of the searches since the last check gave up"""
        self._check(self._L.pftcc_search_check(self._h))

    def search_snhc(self, order, prev_corr, nrefs_bound: int, seed: int, cls_pops=None, precision="exact"):
        """stochastic neighbourhood hill climbing (srch_snhc + shcloc) for every held particle:
        order (nptcls, nrefs) 1-based visiting orders, prev_corr (nptcls,); returns a structured
        array (iref, irot, found_better, nrefs_eval, corr) per particle slot"""
        n = self.get_nptcls()
        o = np.ascontiguousarray(order, np.int32).reshape(n, self.cfg.nrefs)
        pv = np.ascontiguousarray(prev_corr, np.float32).reshape(n)
        pops = None if cls_pops is None else np.ascontiguousarray(cls_pops, np.int32).reshape(self.cfg.nrefs)
        out = (_lib.SnhcOut * n)()
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
        self._check(self._L.pftcc_search_snhc(self._h, ip(o), _f32p(pv), None if pops is None else ip(pops),
                                              int(nrefs_bound), int(seed) & ((1 << 64) - 1), _PRECS[precision], out))
        dt = np.dtype([("iref", np.int32), ("irot", np.int32), ("found_better", np.int32), ("nrefs_eval", np.int32),
                       ("corr", np.float32), ("pad", np.int32, 3)])
        return np.frombuffer(out, dtype=dt).copy()

    def search_best_dev(self, shifts, precision, ntop: int, out_dev_ptr: int):
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
        ns = 0 if sh is None else sh.shape[0]
        self._check(self._L.pftcc_search_best_dev(self._h, ns, None if sh is None else _f32p(sh), _PRECS[precision],
                                                  int(ntop), C.c_void_p(out_dev_ptr)))

    def grad_batch(self, iref, iptcl, irot, sx, sy, ddf):
        """f and grad3 = d f / d(shift_x, shift_y, defocus) for arrays of requests"""
        iref, iptcl, irot, sx, sy, ddf = np.broadcast_arrays(*(np.asarray(v) for v in (iref, iptcl, irot, sx, sy, ddf)))
        n = iref.size
        # pftcc_grad_req records built as a numpy structured array (40 bytes each)
        req = np.zeros(n, dtype=_GRAD_REQ)
        req["iref"], req["iptcl"], req["irot"] = iref.ravel(), iptcl.ravel(), irot.ravel()
        req["sx"], req["sy"], req["ddf"] = sx.ravel(), sy.ravel(), ddf.ravel()
        f = np.zeros(n, np.float64)
        g = np.zeros((n, 3), np.float64)
        self._check(self._L.pftcc_grad_batch(self._h, n, req.ctypes.data_as(C.POINTER(_lib.GradReq)),
                                             f.ctypes.data_as(C.POINTER(C.c_double)),
                                             g.ctypes.data_as(C.POINTER(C.c_double))))
        return f, g

    def cont_shift_grad_batch(self, iref, iptcl, irot, sx, sy):
        """f and grad5 = d f / d(e1, e2, e3, shift_x, shift_y) (gencorr_cont_shift_grad_cc_for_rot_8)
        for arrays of requests, from the references and derivative references of fdf_project_polar"""
        iref, iptcl, irot, sx, sy = np.broadcast_arrays(*(np.asarray(v) for v in (iref, iptcl, irot, sx, sy)))
        n = iref.size
        req = np.zeros(n, dtype=_GRAD_REQ)
        req["iref"], req["iptcl"], req["irot"] = iref.ravel(), iptcl.ravel(), irot.ravel()
        req["sx"], req["sy"] = sx.ravel(), sy.ravel()
        f = np.zeros(n, np.float64)
        g = np.zeros((n, 5), np.float64)
        self._check(self._L.pftcc_cont_shift_grad_batch(self._h, n, req.ctypes.data_as(C.POINTER(_lib.GradReq)),
                                                        f.ctypes.data_as(C.POINTER(C.c_double)),
                                                        g.ctypes.data_as(C.POINTER(C.c_double))))
        return f, g

    def orisrch_batch(self, iptcl, e, angerr_deg, maxhwshift, maxits: int = 100, pgtol: float = 1e-5,
                      factr: float = 1e7):
        """pftcc_orisrch_grad%minimize for arrays of particles (n,) from Euler angles e (n, 3) in
        degrees: list of dicts with e, shift (rotated into the reference frame), corr, corr_init,
        found_better, nevals, niter, converged"""
        ip = np.atleast_1d(np.asarray(iptcl, np.int64))
        ee = np.asarray(e, np.float64).reshape(-1, 3)
        n = ip.size
        ang = np.broadcast_to(np.asarray(angerr_deg, np.float64), (n,))
        msh = np.broadcast_to(np.asarray(maxhwshift, np.float64), (n,))
        req = (_lib.OrisrchReq * n)()
        for i in range(n):
            req[i].iptcl = int(ip[i])
            for v in range(3):
                req[i].e[v] = float(ee[i, v])
            req[i].angerr_deg, req[i].maxhwshift = float(ang[i]), float(msh[i])
        out = (_lib.OrisrchOut * n)()
        self._check(self._L.pftcc_orisrch_batch(self._h, n, req, int(maxits), float(pgtol), float(factr), out))
        return [dict(e=np.array(o.e[:]), shift=np.array(o.shift[:]), corr=o.corr, corr_init=o.corr_init,
                     found_better=bool(o.found_better), nevals=o.nevals, niter=o.niter, converged=bool(o.converged))
                for o in out]

    def gencorr_cont_shift_grad_cc_for_rot_8(self, iref: int, iptcl: int, shvec, irot: int):
        f = C.c_double()
        g = np.zeros(5, np.float64)
        sh = np.ascontiguousarray(shvec, np.float64)
        self._check(self._L.pftcc_gencorr_cont_shift_grad_cc_for_rot_8(
            self._h, int(iref), int(iptcl), sh.ctypes.data_as(C.POINTER(C.c_double)), int(irot), C.byref(f),
            g.ctypes.data_as(C.POINTER(C.c_double))))
        return f.value, g

    def gencorr_cont_grad_cc_for_rot_8(self, iref: int, iptcl: int, shvec, irot: int):
        cc = C.c_double()
        g = np.zeros(3, np.float64)
        sh = np.ascontiguousarray(shvec, np.float64)
        self._check(self._L.pftcc_gencorr_cont_grad_cc_for_rot_8(
            self._h, int(iref), int(iptcl), sh.ctypes.data_as(C.POINTER(C.c_double)), int(irot), C.byref(cc),
            g.ctypes.data_as(C.POINTER(C.c_double))))
        return cc.value, g

    def refine_batch(self, iref, iptcl, irot, x0, lb, ub, maxits: int = 100, pgtol: float = 1e-5,
                     factr: float = 1e7):
        """maximise corr over (shift_x, shift_y, defocus offset) per problem in its box [lb, ub]
        (each (3,) for all problems or (n, 3) per problem);
        returns (x (n,3), corr (n,), nevals (n,), niter (n,), converged (n,))"""
        iref, iptcl, irot = (np.atleast_1d(np.asarray(v)) for v in (iref, iptcl, irot))
        x0 = np.asarray(x0, np.float64).reshape(-1, 3)
        n = x0.shape[0]
        req = (_lib.RefineReq * n)()
        for i in range(n):
            req[i].iref, req[i].iptcl, req[i].irot = int(iref.flat[i % iref.size]), int(iptcl.flat[i % iptcl.size]), \
                int(irot.flat[i % irot.size])
            for v in range(3):
                req[i].x0[v] = float(x0[i, v])
        out = (_lib.RefineOut * n)()
        lb = np.ascontiguousarray(np.broadcast_to(np.asarray(lb, np.float64), (n, 3)))
        ub = np.ascontiguousarray(np.broadcast_to(np.asarray(ub, np.float64), (n, 3)))
        self._check(self._L.pftcc_refine_batch(self._h, n, req, lb.ctypes.data_as(C.POINTER(C.c_double)),
                                               ub.ctypes.data_as(C.POINTER(C.c_double)), int(maxits), float(pgtol),
                                               float(factr), out))
        x = np.array([[o.x[v] for v in range(3)] for o in out])
        return (x, np.array([o.f for o in out]), np.array([o.nevals for o in out]),
                np.array([o.niter for o in out]), np.array([o.converged for o in out], bool))

    def shsrch_batch(self, iref, iptcl, lims, mode: str = "minimize", irot=0, opt_angle: bool = True,
                     coarse_init: bool = False, maxits: int = 100, max_evals: int = 5, halfrot: float = 0.0):
        """pftcc_shsrch_grad (minimize / minimize_exhaustive) for many (reference, particle)
        problems; lims (2, 2) for all problems or (n, 2, 2) per problem.  Returns a structured
        array (irot, found_better, nevals, ncycles, corr, shift[2]) per problem"""
        iref, iptcl, irot = (np.atleast_1d(np.asarray(v)) for v in (iref, iptcl, irot))
        n = max(iref.size, iptcl.size)
        lims = np.broadcast_to(np.asarray(lims, np.float32), (n, 2, 2))
        req = (_lib.ShsrchReq * n)()
        for i in range(n):
            req[i].iref, req[i].iptcl = int(iref.flat[i % iref.size]), int(iptcl.flat[i % iptcl.size])
            req[i].irot = int(irot.flat[i % irot.size])
            for a in range(2):
                for b in range(2):
                    req[i].lims[a][b] = float(lims[i, a, b])
        opts = _lib.ShsrchOpts(int(bool(opt_angle)), int(bool(coarse_init)), int(maxits), int(max_evals),
                               float(halfrot), 0)
        out = (_lib.ShsrchOut * n)()
        m = {"minimize": _lib.SHSRCH_MINIMIZE, "exhaustive": _lib.SHSRCH_EXHAUSTIVE}[mode]
        self._check(self._L.pftcc_shsrch_batch(self._h, m, C.byref(opts), n, req, out))
        dt = np.dtype([("irot", np.int32), ("found_better", np.int32), ("nevals", np.int32), ("ncycles", np.int32),
                       ("corr", np.float32), ("shift", np.float32, 2), ("pad", np.float32)])
        return np.frombuffer(out, dtype=dt).copy()

    # ---- GETTERS ----------------------------------------------------------------------------
    def get_nrots(self) -> int:
        return self._geti(self._L.pftcc_get_nrots)

    def get_pftsz(self) -> int:
        return self._geti(self._L.pftcc_get_pftsz)

    def get_box(self) -> int:
        return self._geti(self._L.pftcc_get_box)

    def get_nrefs(self) -> int:
        return self._geti(self._L.pftcc_get_nrefs)

    def get_nptcls(self) -> int:
        return self._geti(self._L.pftcc_get_nptcls)

    def get_pdim(self):
        p = np.zeros(3, np.int32)
        self._check(self._L.pftcc_get_pdim(self._h, p.ctypes.data_as(C.POINTER(C.c_int))))
        return [int(v) for v in p]

    def get_rot(self, roind: int) -> float:
        v = C.c_float()
        self._check(self._L.pftcc_get_rot(self._h, int(roind), C.byref(v)))
        return v.value

    def get_roind(self, rot: float) -> int:
        v = C.c_int()
        self._check(self._L.pftcc_get_roind(self._h, float(rot), C.byref(v)))
        return v.value

    def get_coord(self, rot: int, k: int):
        xy = np.zeros(2, np.float32)
        self._check(self._L.pftcc_get_coord(self._h, int(rot), int(k), _f32p(xy)))
        return xy

    def ptcl_iseven(self, iptcl: int) -> bool:
        v = C.c_int()
        self._check(self._L.pftcc_ptcl_iseven(self._h, int(iptcl), C.byref(v)))
        return bool(v.value)

    def get_ref_pft(self, iref: int, iseven: bool) -> np.ndarray:
        out = np.zeros((self.K, self.P), np.complex64)
        self._check(self._L.pftcc_get_ref_pft(self._h, int(iref), int(bool(iseven)), _f32p(out.view(np.float32))))
        return out

    def get_ptcl_pft(self, iptcl: int) -> np.ndarray:
        out = np.zeros((self.K, self.P), np.complex64)
        self._check(self._L.pftcc_get_ptcl_pft(self._h, int(iptcl), _f32p(out.view(np.float32))))
        return out

    def get_sqsum_ptcl(self, iptcl: int) -> float:
        v = C.c_float()
        self._check(self._L.pftcc_get_sqsum_ptcl(self._h, int(iptcl), C.byref(v)))
        return v.value

    def kernel_launches(self) -> int:
        return int(self._L.pftcc_kernel_launches(self._h))

    def synchronize(self):
        self._check(self._L.pftcc_synchronize(self._h))

    def set_tuning(self, w_rows: int = 0, w_cols: int = 0, s1_stages: int = 0):
        """wave and tile sizes of the m-domain search (0 = automatic; pftcc_set_tuning)"""
        self._check(self._L.pftcc_set_tuning(self._h, C.byref(_lib.Tuning(int(w_rows), int(w_cols), int(s1_stages), 0))))

    def get_tuning(self) -> dict:
        t = _lib.Tuning()
        self._check(self._L.pftcc_get_tuning(self._h, C.byref(t)))
        return {"w_rows": t.w_rows, "w_cols": t.w_cols, "s1_stages": t.s1_stages, "from_wisdom": bool(t.from_wisdom)}

    def autotune(self, shifts=None, precision="bf16x3", ntop: int = 8, wisdom: str | None = None) -> dict:
        """the autotuner (pftcc_autotune): the fastest wave / tile sizes for this search on the held
        data, read from or appended to the wisdom file"""
        sh = None if shifts is None else np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
        ns = 0 if sh is None else sh.shape[0]
        t = _lib.Tuning()
        self._check(self._L.pftcc_autotune(self._h, ns, None if sh is None else _f32p(sh), _PRECS[precision],
                                           int(ntop), None if wisdom is None else os.fsencode(wisdom), C.byref(t)))
        return {"w_rows": t.w_rows, "w_cols": t.w_cols, "s1_stages": t.s1_stages, "from_wisdom": bool(t.from_wisdom)}

    def set_wait_limit(self, polls: int):
        """polls of a tensor-core pipeline wait before the call gives up with PFTCC_ERR_TIMEOUT
        (0 = the default)"""
        self._check(self._L.pftcc_set_wait_limit(self._h, int(polls)))

    def set_stream(self, stream_handle: int | None):
        """run on a caller's cudaStream_t (e.g. torch.cuda.current_stream().cuda_stream)"""
        self._check(self._L.pftcc_set_stream(self._h, None if not stream_handle else C.c_void_p(stream_handle)))

    def prof_enable(self, on: bool = True):
        self._check(self._L.pftcc_prof_enable(self._h, int(bool(on))))

    def prof_reset(self):
        self._check(self._L.pftcc_prof_reset(self._h))

    def prof_read(self) -> dict:
        """{kernel class: (total ms, launches)} from the CUDA events around each launch"""
        out = {}
        for i, name in enumerate(_lib.KERNEL_CLASSES):
            ms, n = C.c_double(), C.c_longlong()
            self._check(self._L.pftcc_prof_read(self._h, i, C.byref(ms), C.byref(n)))
            out[name] = (ms.value, n.value)
        return out
