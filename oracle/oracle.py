"""numpy front-end of the CPU oracle (oracle/pftcc_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by ``__graft_entry__.smoke()`` as
the parity checker and by ``bench.py`` for its cpu_baseline / reference arm.
The product library never imports this module.  Array conventions follow the
reference's Fortran storage (see pftcc_oracle.h): a polar FT is a complex64
array of shape (K, P), i.e. ``pft[k - kfrom, n]``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (gcc, OpenMP) and return the .so path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class Geom(C.Structure):
    _fields_ = [("nrots", C.c_int), ("pftsz", C.c_int), ("kfrom", C.c_int),
                ("kto", C.c_int), ("kstop", C.c_int), ("box", C.c_int)]

    @property
    def K(self) -> int:
        return self.kto - self.kfrom + 1

    @property
    def Ks(self) -> int:
        return self.kstop - self.kfrom + 1


class Ctf(C.Structure):
    _fields_ = [("smpd", C.c_float), ("kv", C.c_float), ("cs", C.c_float), ("fraca", C.c_float),
                ("dfx", C.c_float), ("dfy", C.c_float), ("angast", C.c_float),
                ("phshift", C.c_float), ("l_phaseplate", C.c_int)]


def geom(nrots: int, kfrom: int, kto: int, box: int, kstop: int | None = None) -> Geom:
    return Geom(nrots, nrots // 2, kfrom, kto, kto if kstop is None else kstop, box)


def _P(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        fp, dp, ip = C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int)
        G = C.POINTER(Geom)
        L.orc_tables.argtypes = [G, fp, dp, dp]
        L.orc_ctfmat.argtypes = [G, fp, C.POINTER(Ctf), dp]
        L.orc_dctfmat_ddf.argtypes = [G, fp, C.POINTER(Ctf), dp]
        L.orc_shmat.argtypes = [G, dp, dp, C.c_double, C.c_double, dp]
        L.orc_gencorrs.argtypes = [G, fp, fp, dp, dp, dp, dp, dp]
        L.orc_gencorrs_ptclframe.argtypes = [G, fp, fp, dp, dp, dp, dp, dp]
        L.orc_gencorr_for_rot.argtypes = [G, fp, fp, dp, dp, C.c_int, C.c_int, dp, dp]
        L.orc_gencorr_for_rot.restype = C.c_double
        L.orc_gencorr_grad3.argtypes = [G, fp, fp, dp, dp, dp, C.c_int, C.c_int, dp, dp, dp, dp]
        L.orc_genfrc.argtypes = [G, fp, fp, dp, dp, C.c_int, dp, dp, dp]
        L.orc_specscore.argtypes = [G, fp, fp, dp, dp, C.c_int, dp, dp]
        L.orc_specscore.restype = C.c_double
        L.orc_snhc_select.argtypes = [C.c_int, C.c_int, fp, ip, ip, C.c_int, C.c_double, C.c_ulonglong, C.c_int, ip]
        L.orc_snhc_select.restype = C.c_double
        L.orc_snhc_uniform.argtypes = [C.c_ulonglong, C.c_int, C.c_int]
        L.orc_snhc_uniform.restype = C.c_double
        L.orc_polarize.argtypes = [G, fp, fp, C.c_int, dp]
        L.orc_euler2m.argtypes = [dp, dp]
        L.orc_expand_cmat3d.argtypes = [C.c_int, fp, C.c_double, fp]
        L.orc_fproject_polar.argtypes = [G, fp, C.c_int, fp, dp, ip, C.c_int, dp]
        L.orc_pxls_p_shell.argtypes = [C.c_int, C.c_int, dp]
        L.orc_gencorrs_euclid.argtypes = [G, fp, fp, dp, dp, dp, dp, dp, dp, dp]
        L.orc_gencorrs_euclid_ptclframe.argtypes = [G, fp, fp, dp, dp, dp, dp, dp, dp, dp]
        L.orc_gencorr_euclid_grad_for_rot.argtypes = [G, fp, fp, dp, dp, C.c_int, dp, dp, dp, dp, dp, dp]
        L.orc_sigma_contrib.argtypes = [G, fp, fp, dp, dp, C.c_int, dp, dp, dp, dp, dp]
        L.orc_shellnorm_factors.argtypes = [G, fp, fp, dp]
        L.orc_shellnorm_factors_mode.argtypes = [G, fp, fp, C.c_int, dp]
        L.orc_prep_matchfilt_pssnr.argtypes = [G, dp, fp, fp]
        L.orc_savgol7.argtypes = [C.c_int, dp]
        L.orc_prep_matchfilt.argtypes = [G, fp, dp, fp, C.c_int, fp]
        L.orc_prepimg4align.argtypes = [C.c_int, C.c_int, fp, C.c_double, C.c_double, C.c_double, C.POINTER(Ctf), dp]
        L.orc_prepimg4align_opts.argtypes = [C.c_int, C.c_int, fp, C.c_double, C.c_double, C.c_double, C.c_double,
                                             C.c_int, C.c_double, C.c_double, C.POINTER(Ctf), dp]
        L.orc_euler2dm.argtypes = [dp, dp]
        L.orc_kb_dapod.argtypes = [C.c_double]
        L.orc_kb_dapod.restype = C.c_double
        L.orc_fdf_project_polar.argtypes = [G, fp, C.c_int, fp, dp, dp, dp]
        L.orc_gencorr_cont_shift_grad.argtypes = [G, fp, fp, fp, dp, dp, C.c_int, dp, dp, dp, dp]
        L.orc_kb_apod.argtypes = [C.c_double]
        L.orc_kb_apod.restype = C.c_double
        L.orc_fftpath_new.argtypes = [G]
        L.orc_fftpath_new.restype = C.c_void_p
        L.orc_fftpath_free.argtypes = [C.c_void_p]
        L.orc_fftpath_memo_size.argtypes = [G]
        L.orc_fftpath_memo_size.restype = C.c_long
        L.orc_fftpath_memoize.argtypes = [C.c_void_p, fp, fp]
        L.orc_fftpath_gencorrs.argtypes = [C.c_void_p, fp, fp, C.c_float, fp, fp, dp, dp, fp]
        L.orc_cpu_search.argtypes = [G, C.c_int, fp, C.c_int, fp, fp, C.c_int, fp, ip, ip, ip, fp, C.c_int]
        L.orc_fftpath_allcorrs.argtypes = [G, C.c_int, fp, fp, fp, C.c_int, fp, fp, C.c_int]
        L.orc_fftpath_allcorrs.restype = C.c_int
        L.orc_cpu_search.restype = C.c_int
        L.orc_cfft.argtypes = [C.c_int, dp, dp, C.c_int]
        _lib = L
    return _lib


def _c64(x) -> np.ndarray:
    """complex64 (K, P) -> contiguous float32 view of interleaved (re, im)"""
    return np.ascontiguousarray(x, dtype=np.complex64).view(np.float32)


def _c128_out(shape) -> np.ndarray:
    return np.zeros(shape, dtype=np.complex128)


@dataclass
class Tables:
    polar: np.ndarray        # float32 (K, 2N)
    argtransf: np.ndarray    # float64 (K, N)
    argtransf1: np.ndarray   # float64 (N,)


def tables(g: Geom) -> Tables:
    polar = np.zeros((g.K, 2 * g.nrots), np.float32)
    at = np.zeros((g.K, g.nrots), np.float64)
    at1 = np.zeros(g.nrots, np.float64)
    lib().orc_tables(C.byref(g), _P(polar, C.c_float), _P(at, C.c_double), _P(at1, C.c_double))
    return Tables(polar, at, at1)


def make_ctf(smpd=1.3, kv=300.0, cs=2.7, fraca=0.1, dfx=2.0, dfy=2.0, angast=0.0, phshift=0.0, phaseplate=False) -> Ctf:
    return Ctf(smpd, kv, cs, fraca, dfx, dfy, angast, phshift, int(phaseplate))


def ctfmat(g: Geom, t: Tables, c: Ctf) -> np.ndarray:
    out = np.zeros((g.K, g.pftsz), np.float64)
    lib().orc_ctfmat(C.byref(g), _P(t.polar, C.c_float), C.byref(c), _P(out, C.c_double))
    return out


def dctfmat_ddf(g: Geom, t: Tables, c: Ctf) -> np.ndarray:
    out = np.zeros((g.K, g.pftsz), np.float64)
    lib().orc_dctfmat_ddf(C.byref(g), _P(t.polar, C.c_float), C.byref(c), _P(out, C.c_double))
    return out


def shmat(g: Geom, t: Tables, sx: float, sy: float) -> np.ndarray:
    out = _c128_out((g.K, g.pftsz))
    lib().orc_shmat(C.byref(g), _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double), sx, sy,
                    out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return out


def _shv(shvec):
    return None if shvec is None else np.asarray(shvec, np.float64)


def _ctf_arg(ctf):
    return None if ctf is None else np.ascontiguousarray(ctf, np.float64)


def gencorrs(g: Geom, t: Tables, ref, ptcl, ctf=None, shvec=None) -> np.ndarray:
    """gencorrs_cc_1 (shvec None) / gencorrs_cc_2, FP64, reference frame"""
    cc = np.zeros(g.nrots, np.float64)
    lib().orc_gencorrs(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float), _P(_ctf_arg(ctf), C.c_double),
                       _P(_shv(shvec), C.c_double), _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double),
                       _P(cc, C.c_double))
    return cc


def gencorrs_ptclframe(g: Geom, t: Tables, ref, ptcl, ctf=None, shvec=None) -> np.ndarray:
    cc = np.zeros(g.nrots, np.float64)
    lib().orc_gencorrs_ptclframe(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float),
                                 _P(_ctf_arg(ctf), C.c_double), _P(_shv(shvec), C.c_double),
                                 _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double), _P(cc, C.c_double))
    return cc


def gencorr_for_rot(g: Geom, t: Tables, ref, ptcl, irot: int, ctf=None, shvec=None, match_filt=False) -> float:
    return lib().orc_gencorr_for_rot(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float),
                                     _P(_ctf_arg(ctf), C.c_double), _P(_shv(shvec), C.c_double), int(irot),
                                     int(bool(match_filt)), _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double))


def gencorr_grad3(g: Geom, t: Tables, ref, ptcl, irot: int, ctf=None, dctf=None, shvec=None, match_filt=False):
    """(f, grad3) with grad3 = d f / d(shift_x, shift_y, defocus[micron]), reference frame"""
    f = np.zeros(1, np.float64)
    g3 = np.zeros(3, np.float64)
    lib().orc_gencorr_grad3(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float),
                            _P(_ctf_arg(ctf), C.c_double), _P(_ctf_arg(dctf), C.c_double), _P(_shv(shvec), C.c_double),
                            int(irot), int(bool(match_filt)), _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double),
                            _P(f, C.c_double), _P(g3, C.c_double))
    return float(f[0]), g3


def pxls_p_shell(g: Geom) -> np.ndarray:
    """pixels per shell k = kfrom..kto (setup_pxls_p_shell)"""
    out = np.zeros(g.K, np.float64)
    lib().orc_pxls_p_shell(g.kfrom, g.kto, _P(out, C.c_double))
    return out


def gencorrs_euclid(g: Geom, t: Tables, ref, ptcl, sigma2, ctf=None, shvec=None) -> np.ndarray:
    """gencorrs_euclid_1 (shvec None) / gencorrs_euclid_2; sigma2[K] is the particle's
    sigma2_noise(kfrom:kto, iptcl)"""
    out = np.zeros(g.nrots, np.float64)
    sig = np.ascontiguousarray(sigma2, np.float64)
    lib().orc_gencorrs_euclid(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float),
                              _P(_ctf_arg(ctf), C.c_double), _P(_shv(shvec), C.c_double),
                              _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double), _P(sig, C.c_double),
                              _P(pxls_p_shell(g), C.c_double), _P(out, C.c_double))
    return out


def gencorrs_euclid_ptclframe(g: Geom, t: Tables, ref, ptcl, sigma2, ctf=None, shvec=None) -> np.ndarray:
    """the Euclidean objective in the particle CTF frame (the m-domain search's), every rotation"""
    out = np.zeros(g.nrots, np.float64)
    sig = np.ascontiguousarray(sigma2, np.float64)
    lib().orc_gencorrs_euclid_ptclframe(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float),
                                        _P(_ctf_arg(ctf), C.c_double), _P(_shv(shvec), C.c_double),
                                        _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double),
                                        _P(sig, C.c_double), _P(pxls_p_shell(g), C.c_double), _P(out, C.c_double))
    return out


def gencorr_euclid_grad_for_rot(g: Geom, t: Tables, ref, ptcl, irot: int, sigma2, ctf=None, shvec=(0.0, 0.0)):
    """(f, grad[2]) of gencorr_euclid_grad_for_rot_8; f alone is gencorr_euclid_for_rot_8"""
    f = np.zeros(1, np.float64)
    gr = np.zeros(2, np.float64)
    sig = np.ascontiguousarray(sigma2, np.float64)
    lib().orc_gencorr_euclid_grad_for_rot(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float),
                                          _P(_ctf_arg(ctf), C.c_double), _P(_shv(shvec), C.c_double), int(irot),
                                          _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double),
                                          _P(sig, C.c_double), _P(pxls_p_shell(g), C.c_double),
                                          _P(f, C.c_double), _P(gr, C.c_double))
    return float(f[0]), gr


def sigma_contrib(g: Geom, t: Tables, ref, ptcl, irot: int, ctf=None, shvec=(0.0, 0.0)):
    """(sigma_contrib, ptcl_sumsq, ref_sumsq), each [K] over kfrom..kto (gencorr_sigma_contrib)"""
    sc, ps, rs = (np.zeros(g.K, np.float64) for _ in range(3))
    lib().orc_sigma_contrib(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float),
                            _P(_ctf_arg(ctf), C.c_double), _P(_shv(shvec), C.c_double), int(irot),
                            _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double), _P(sc, C.c_double),
                            _P(ps, C.c_double), _P(rs, C.c_double))
    return sc, ps, rs


def genfrc(g: Geom, t: Tables, ref, ptcl, irot: int, ctf=None, shvec=None) -> np.ndarray:
    """shell FRCs k = kfrom..kstop at one rotation (genfrc / calc_frc), FP64"""
    frc = np.zeros(g.kstop - g.kfrom + 1, np.float64)
    lib().orc_genfrc(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float), _P(_ctf_arg(ctf), C.c_double),
                     _P(_shv(shvec), C.c_double), int(irot), _P(t.argtransf, C.c_double),
                     _P(t.argtransf1, C.c_double), _P(frc, C.c_double))
    return frc


def specscore(g: Geom, t: Tables, ref, ptcl, irot: int, ctf=None, shvec=None) -> float:
    """specscore_1 (shvec None) / specscore_2: max(0, median shell FRC), FP64"""
    return lib().orc_specscore(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(ptcl), C.c_float),
                               _P(_ctf_arg(ctf), C.c_double), _P(_shv(shvec), C.c_double), int(irot),
                               _P(t.argtransf, C.c_double), _P(t.argtransf1, C.c_double))


def snhc_select(corrs, order, prev_corr: float, nrefs_bound: int, seed: int, iptcl: int, pops=None):
    """srch_snhc + shcloc over corrs[nrefs, nrots] for one particle: (iref, irot, found_better,
    nrefs_eval, corr), iref/irot 1-based"""
    c = np.ascontiguousarray(corrs, np.float32)
    o = np.ascontiguousarray(order, np.int32)
    pp = None if pops is None else np.ascontiguousarray(pops, np.int32)
    out = np.zeros(4, np.int32)
    v = lib().orc_snhc_select(c.shape[1], c.shape[0], _P(c, C.c_float), _P(o, C.c_int), _P(pp, C.c_int),
                              int(nrefs_bound), float(prev_corr), int(seed), int(iptcl), _P(out, C.c_int))
    return int(out[0]), int(out[1]), int(out[2]), int(out[3]), float(v)


def snhc_uniform(seed: int, iptcl: int, isample: int) -> float:
    return lib().orc_snhc_uniform(int(seed), int(iptcl), int(isample))


def polarize(g: Geom, t: Tables, cmat, griddev=False) -> np.ndarray:
    """cmat: complex64 (box, box//2+1) half-plane FT (image%cmat transposed to C order)"""
    out = _c128_out((g.K, g.pftsz))
    lib().orc_polarize(C.byref(g), _P(t.polar, C.c_float), _P(_c64(cmat), C.c_float), int(bool(griddev)),
                       out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return out


def euler2m(eul) -> np.ndarray:
    """rotation matrix of a Spider Euler triplet in degrees (euler2m, simple_ori.f90:1275)"""
    e = np.ascontiguousarray(eul, np.float64)
    R = np.zeros(9, np.float64)
    lib().orc_euler2m(_P(e, C.c_double), _P(R, C.c_double))
    return R.reshape(3, 3)


def expand_cmat3d(cmat_half, box: int, factor: float = 1.0) -> np.ndarray:
    """cmat_half: complex64 (box, box, box//2+1) = image%cmat(h, k, m) in [m][k][h] order;
    returns the expanded cube complex64 (S, S, S), S = box + 5, index [m + E][k + E][h + E]"""
    S = box + 5
    out = np.zeros((S, S, S), np.complex64)
    lib().orc_expand_cmat3d(int(box), _P(_c64(cmat_half), C.c_float), C.c_double(factor),
                            out.view(np.float32).ctypes.data_as(C.POINTER(C.c_float)))
    return out


def fproject_polar(g: Geom, t: Tables, cmat_exp, box: int, eul, mask=None, griddev=False) -> np.ndarray:
    """polar FT (K, P) of the central section at Euler angles eul (degrees) from the expanded cube"""
    out = _c128_out((g.K, g.pftsz))
    e = np.ascontiguousarray(eul, np.float64)
    m = None if mask is None else np.ascontiguousarray(mask, np.int32)
    lib().orc_fproject_polar(C.byref(g), _P(t.polar, C.c_float), int(box), _P(_c64(cmat_exp), C.c_float),
                             _P(e, C.c_double), _P(m, C.c_int), int(bool(griddev)),
                             out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return out


def shellnorm_factors(g: Geom, ref, optlp=None, pssnr: bool = False) -> np.ndarray:
    """per-shell factors k <= kstop of shellnorm_and_filter_ref (l_match_filt; l_pssnr with pssnr)"""
    out = np.zeros(g.Ks, np.float64)
    o = None if optlp is None else np.ascontiguousarray(optlp, np.float32)
    lib().orc_shellnorm_factors_mode(C.byref(g), _P(_c64(ref), C.c_float), _P(o, C.c_float), int(bool(pssnr)),
                                     _P(out, C.c_double))
    return out


def prep_matchfilt_pssnr(g: Geom, ptcl, ctf=None, optlp=None) -> np.ndarray:
    """the particle after prep_matchfilt's l_pssnr branch"""
    out = np.ascontiguousarray(ptcl, np.complex64).copy()
    o = None if optlp is None else np.ascontiguousarray(optlp, np.float32)
    lib().orc_prep_matchfilt_pssnr(C.byref(g), _P(_ctf_arg(ctf), C.c_double), _P(o, C.c_float),
                                   out.view(np.float32).ctypes.data_as(C.POINTER(C.c_float)))
    return out


def savgol7(y) -> np.ndarray:
    a = np.array(y, np.float64)
    lib().orc_savgol7(a.size, _P(a, C.c_double))
    return a


def prep_matchfilt(g: Geom, ref, ptcl, irot: int, ctf=None, optlp=None) -> np.ndarray:
    """the particle after prep_matchfilt against ref at irot (l_match_filt branch)"""
    out = np.ascontiguousarray(ptcl, np.complex64).copy()
    o = None if optlp is None else np.ascontiguousarray(optlp, np.float32)
    lib().orc_prep_matchfilt(C.byref(g), _P(_c64(ref), C.c_float), _P(_ctf_arg(ctf), C.c_double), _P(o, C.c_float),
                             int(irot), out.view(np.float32).ctypes.data_as(C.POINTER(C.c_float)))
    return out


def prepimg4align(img, boxmatch: int, msk: float, x: float = 0.0, y: float = 0.0, ctf: "Ctf | None" = None):
    """prepimg4align of one particle image img (box, box) [y][x]: its FT (boxmatch, boxmatch/2+1)
    [k][h] as polarize takes it; ctf None for ctfflag no / flip, a Ctf for the phase flip"""
    a = np.ascontiguousarray(img, np.float32)
    box = a.shape[0]
    out = _c128_out((boxmatch, boxmatch // 2 + 1))
    lib().orc_prepimg4align(int(box), int(boxmatch), _P(a, C.c_float), float(msk), float(x), float(y),
                            None if ctf is None else C.byref(ctf),
                            out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return out


def prepimg4align_opts(img, boxmatch: int, msk: float, inner: float = 0.0, width: float = 0.0, focusmsk: float = 0.0,
                       griddev: bool = False, x: float = 0.0, y: float = 0.0, ctf: "Ctf | None" = None):
    """prepimg4align with the inner / focus mask and griddev modes (see pftcc_oracle.h)"""
    a = np.ascontiguousarray(img, np.float32)
    box = a.shape[0]
    out = _c128_out((boxmatch, boxmatch // 2 + 1))
    lib().orc_prepimg4align_opts(int(box), int(boxmatch), _P(a, C.c_float), float(msk), float(inner), float(width),
                                 float(focusmsk), int(bool(griddev)), float(x), float(y),
                                 None if ctf is None else C.byref(ctf),
                                 out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return out


def euler2dm(eul) -> np.ndarray:
    """(3, 3, 3): dR/de_j (per radian) of euler2m for j = 1..3"""
    out = np.zeros(27, np.float64)
    lib().orc_euler2dm(_P(np.asarray(eul, np.float64), C.c_double), _P(out, C.c_double))
    return out.reshape(3, 3, 3)


def kb_dapod(x: float) -> float:
    return lib().orc_kb_dapod(float(x))


def fdf_project_polar(g: Geom, t: Tables, cmat_exp, box: int, eul):
    """(pft [K, P], dpft [3, K, P]) of fdf_project_polar"""
    pft = _c128_out((g.K, g.pftsz))
    dpft = _c128_out((3, g.K, g.pftsz))
    lib().orc_fdf_project_polar(C.byref(g), _P(t.polar, C.c_float), int(box), _P(_c64(cmat_exp), C.c_float),
                                _P(np.asarray(eul, np.float64), C.c_double),
                                pft.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                                dpft.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)))
    return pft, dpft


def gencorr_cont_shift_grad(g: Geom, t: Tables, ref, dref, ptcl, irot: int, ctf=None, shvec=(0.0, 0.0)):
    """(f, grad[5]) of gencorr_cont_shift_grad_cc_for_rot_8; dref (3, K, P)"""
    f = np.zeros(1, np.float64)
    gr = np.zeros(5, np.float64)
    lib().orc_gencorr_cont_shift_grad(C.byref(g), _P(_c64(ref), C.c_float), _P(_c64(dref), C.c_float),
                                      _P(_c64(ptcl), C.c_float), _P(_ctf_arg(ctf), C.c_double),
                                      _P(_shv(shvec), C.c_double), int(irot), _P(t.argtransf, C.c_double),
                                      _P(t.argtransf1, C.c_double), _P(f, C.c_double), _P(gr, C.c_double))
    return float(f[0]), gr


def kb_apod(x: float) -> float:
    return lib().orc_kb_apod(float(x))


def cfft(x, sign=-1) -> np.ndarray:
    x = np.ascontiguousarray(x, np.complex128)
    out = np.zeros_like(x)
    lib().orc_cfft(len(x), x.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)),
                   out.view(np.float64).ctypes.data_as(C.POINTER(C.c_double)), int(sign))
    return out


class FFTPath:
    """FP32 FFT path in the reference's loop structure (the timed CPU baseline)."""

    def __init__(self, g: Geom):
        self.g = g
        self.t = tables(g)
        self.h = lib().orc_fftpath_new(C.byref(g))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_fftpath_free(self.h)
            self.h = None

    def memoize(self, ptcl) -> np.ndarray:
        memo = np.zeros(lib().orc_fftpath_memo_size(C.byref(self.g)), np.float32)
        lib().orc_fftpath_memoize(self.h, _P(_c64(ptcl), C.c_float), _P(memo, C.c_float))
        return memo

    def gencorrs(self, ref, ptcl, ctf=None, shvec=None) -> np.ndarray:
        memo = self.memoize(ptcl)
        Ks = self.g.Ks
        sqp = np.float32(np.sum(np.abs(np.asarray(ptcl, np.complex64)[:Ks]) ** 2, dtype=np.float32))
        cc = np.zeros(self.g.nrots, np.float32)
        ctf32 = None if ctf is None else np.ascontiguousarray(ctf, np.float32)
        sh = np.asarray(shvec if shvec is not None else (0.0, 0.0), np.float32)
        lib().orc_fftpath_gencorrs(self.h, _P(_c64(ref), C.c_float), _P(memo, C.c_float), float(sqp),
                                   _P(ctf32, C.c_float), _P(sh, C.c_float), _P(self.t.argtransf, C.c_double),
                                   _P(self.t.argtransf1, C.c_double), _P(cc, C.c_float))
        return cc


def cpu_search(g: Geom, refs, ptcls, ctfmats, shifts, nthreads: int = 0):
    """Exhaustive FP32 FFT-path search over refs x shifts for each particle.
    Returns (best_ref 0-based, best_irot 1-based, best_shift_idx, best_cc, threads_used)."""
    refs = np.ascontiguousarray(refs, np.complex64)
    ptcls = np.ascontiguousarray(ptcls, np.complex64)
    nr, npt = refs.shape[0], ptcls.shape[0]
    ctf32 = None if ctfmats is None else np.ascontiguousarray(ctfmats, np.float32)
    sh = np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
    br = np.zeros(npt, np.int32)
    bro = np.zeros(npt, np.int32)
    bs = np.zeros(npt, np.int32)
    bcc = np.zeros(npt, np.float32)
    used = lib().orc_cpu_search(C.byref(g), nr, _P(refs.view(np.float32), C.c_float), npt,
                                _P(ptcls.view(np.float32), C.c_float), _P(ctf32, C.c_float), sh.shape[0],
                                _P(sh, C.c_float), _P(br, C.c_int), _P(bro, C.c_int), _P(bs, C.c_int),
                                _P(bcc, C.c_float), int(nthreads))
    return br, bro, bs, bcc, used


def fftpath_allcorrs(g: Geom, refs, ptcl, ctf, shifts, nthreads: int = 0):
    """Every correlation of one particle (K, P) against refs (nrefs, K, P) x shifts (ns, 2)
    through the reference's FP32 FFT loop (gencorrs_cc_2 per pair, calc_corrs_over_k
    :1132-1162), OpenMP over the pairs: float32 (nrefs, ns, nrots) and the threads used."""
    refs = np.ascontiguousarray(refs, np.complex64)
    sh = np.ascontiguousarray(shifts, np.float32).reshape(-1, 2)
    out = np.zeros((refs.shape[0], sh.shape[0], g.nrots), np.float32)
    ctf32 = None if ctf is None else np.ascontiguousarray(ctf, np.float32)
    used = lib().orc_fftpath_allcorrs(C.byref(g), refs.shape[0], _P(refs.view(np.float32), C.c_float),
                                      _P(_c64(ptcl), C.c_float), _P(ctf32, C.c_float), sh.shape[0],
                                      _P(sh, C.c_float), _P(out, C.c_float), int(nthreads))
    return out, used


def _ext(x):
    """a half-circle polar FT x(..., P) extended over the full circle: x(n + P) = conj x(n)"""
    return np.concatenate([x, np.conj(x)], axis=-1)


def iter_allcorrs64(g: Geom, t: Tables, refs, ptcls, ctfs, shifts, frame: str = "ref", ref_chunk: int = 8):
    """Every correlation of particles (np, K, P) against refs (nrefs, K, P) x shifts (ns, 2)
    in FP64, yielded per block of references as (r0, r1, cc[np, r1 - r0, ns, nrots]).

    The same sums as the direct oracle (gencorrs_cc_2 :1502-1534 with calc_corr_for_rot_8
    :1218-1243 in the reference frame; gencorrs_ptclframe for the particle frame), each
    circular correlation over the full circle evaluated through length-nrots FP64 FFTs:
    with x~ the conjugate-symmetric extension (x~(n + P) = conj x(n)),
        sum_{n<P} Re A(n) conj Q~(n + rot) = 1/(2N) Re sum_m F[A~](m) conj F[Q~](m) w^{-m rot}.
    Reference frame: A = ref * ctf_p * shmat_s (gen_shmat_8 de Moivre phases, FP64), the
    reference square sum over all K shells (:1531) or kfrom..kstop without shifts (:984).
    Particle frame: A = ref * shmat_s against ctf_p~ Q~, normaliser
    sum_k sum_n |ref(n)|^2 ctf_p~(n + rot)^2 times the particle square sum."""
    import scipy.fft as sf
    N, P, K, Ks = g.nrots, g.pftsz, g.K, g.Ks
    refs = np.asarray(refs, np.complex64).astype(np.complex128)
    Q = np.asarray(ptcls, np.complex64).astype(np.complex128)[:, :Ks]
    npt, nr = Q.shape[0], refs.shape[0]
    ctf = None if ctfs is None else np.asarray(ctfs, np.float64)
    has_shift = shifts is not None
    sh = np.stack([shmat(g, t, float(x), float(y)) for x, y in np.asarray(shifts, np.float64).reshape(-1, 2)]) \
        if has_shift else np.ones((1, K, P), np.complex128)
    ns = sh.shape[0]
    sqp = np.sum(Q.real ** 2 + Q.imag ** 2, axis=(1, 2))
    if frame == "ref":
        FQc = np.conj(sf.fft(_ext(Q), axis=-1, workers=-1))                         # (np, Ks, N)
        ksq = K if has_shift else Ks
        for r0 in range(0, nr, ref_chunk):
            r1 = min(nr, r0 + ref_chunk)
            R = refs[r0:r1]
            A = R[None, :, None] * sh[None, None]                                   # (1, rc, ns, K, P)
            if ctf is not None:
                A = A * ctf[:, None, None]                                          # (np, rc, ns, K, P)
            A = np.broadcast_to(A, (npt,) + A.shape[1:])
            sqr = np.sum(A[..., :ksq, :].real ** 2 + A[..., :ksq, :].imag ** 2, axis=(-2, -1))
            FA = sf.fft(_ext(A[..., :Ks, :]), axis=-1, workers=-1)                  # (np, rc, ns, Ks, N)
            X = np.einsum("prskm,pkm->prsm", FA, FQc, optimize=True)
            num = sf.fft(X, axis=-1, workers=-1).real / (2.0 * N)
            yield r0, r1, num / np.sqrt(sqr * sqp[:, None, None])[..., None]
    elif frame == "ptcl":
        Qc = Q if ctf is None else Q * ctf[:, :Ks]
        FQc = np.conj(sf.fft(_ext(Qc), axis=-1, workers=-1))                        # (np, Ks, N)
        R2 = refs[:, :Ks].real ** 2 + refs[:, :Ks].imag ** 2                        # (nr, Ks, P)
        C2 = np.ones((npt, Ks, P)) if ctf is None else ctf[:, :Ks] ** 2
        FR2 = sf.fft(np.concatenate([R2, R2], axis=-1), axis=-1, workers=-1)        # (nr, Ks, N)
        FC2c = np.conj(sf.fft(np.concatenate([C2, C2], axis=-1), axis=-1, workers=-1))
        Bm = np.ascontiguousarray(FQc.transpose(2, 1, 0))                           # (N, Ks, np)
        for r0 in range(0, nr, ref_chunk):
            r1 = min(nr, r0 + ref_chunk)
            rc = r1 - r0
            A = refs[r0:r1, None, :Ks] * sh[None, :, :Ks]                           # (rc, ns, Ks, P)
            FA = sf.fft(_ext(A), axis=-1, workers=-1)                               # (rc, ns, Ks, N)
            Am = np.ascontiguousarray(FA.reshape(rc * ns, Ks, N).transpose(2, 0, 1))  # (N, rc*ns, Ks)
            X = np.matmul(Am, Bm)                                                   # (N, rc*ns, np)
            X = X.transpose(2, 1, 0).reshape(npt, rc, ns, N)
            num = sf.fft(X, axis=-1, workers=-1).real / (2.0 * N)
            Y = np.einsum("rkm,pkm->prm", FR2[r0:r1], FC2c, optimize=True)          # (np, rc, N)
            den = sf.fft(Y, axis=-1, workers=-1).real / (2.0 * N)
            yield r0, r1, num / np.sqrt(den[:, :, None, :] * sqp[:, None, None, None])
    else:
        raise ValueError("frame must be 'ref' or 'ptcl'")


def allcorrs64(g: Geom, t: Tables, refs, ptcls, ctfs, shifts, frame: str = "ref", ref_chunk: int = 8) -> np.ndarray:
    """all of iter_allcorrs64 in one array (np, nrefs, ns, nrots), for small cases"""
    nr = np.asarray(refs).shape[0]
    out = None
    for r0, r1, cc in iter_allcorrs64(g, t, refs, ptcls, ctfs, shifts, frame, ref_chunk):
        if out is None:
            out = np.zeros((cc.shape[0], nr) + cc.shape[2:], np.float64)
        out[:, r0:r1] = cc
    return out
