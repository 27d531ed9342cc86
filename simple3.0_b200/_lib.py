"""ctypes binding of libpftcc_b200.so (include/pftcc_b200.h).

There is no fallback: if the shared library is missing or no sm_100 device is
present the calls raise.  This mirrors what a Fortran ISO_C_BINDING interface
module would bind."""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

SHSRCH_MINIMIZE, SHSRCH_EXHAUSTIVE = 0, 1
OK, ERR_ARG, ERR_INDEX, ERR_STATE, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_NODEV, ERR_UNSUPPORTED = range(9)
FRAME_REF, FRAME_PTCL = 0, 1
PREC_EXACT, PREC_FP32, PREC_BF16X3 = 0, 1, 2
OBJFUN_CC, OBJFUN_EUCLID = 0, 1
CTFFLAG_NO, CTFFLAG_YES, CTFFLAG_FLIP = 0, 1, 2


class Config(C.Structure):
    _fields_ = [("nrefs", C.c_int), ("pfromto", C.c_int * 2), ("box", C.c_int), ("nrots", C.c_int),
                ("kfromto", C.c_int * 2), ("kstop", C.c_int), ("with_ctf", C.c_int), ("match_filt", C.c_int),
                ("ctf_frame", C.c_int), ("device", C.c_int)]


class CtfParams(C.Structure):
    _fields_ = [("smpd", C.c_float), ("kv", C.c_float), ("cs", C.c_float), ("fraca", C.c_float),
                ("dfx", C.c_float), ("dfy", C.c_float), ("angast", C.c_float), ("phshift", C.c_float),
                ("l_phaseplate", C.c_int)]


class Best(C.Structure):
    _fields_ = [("iref", C.c_int), ("irot", C.c_int), ("ishift", C.c_int), ("corr", C.c_float)]


class GradReq(C.Structure):
    _fields_ = [("iref", C.c_int), ("iptcl", C.c_int), ("irot", C.c_int), ("pad", C.c_int),
                ("sx", C.c_double), ("sy", C.c_double), ("ddf", C.c_double)]


class OrisrchReq(C.Structure):
    _fields_ = [("iptcl", C.c_int), ("pad", C.c_int), ("e", C.c_double * 3), ("angerr_deg", C.c_double),
                ("maxhwshift", C.c_double)]


class OrisrchOut(C.Structure):
    _fields_ = [("e", C.c_double * 3), ("shift", C.c_double * 2), ("corr", C.c_double), ("corr_init", C.c_double),
                ("found_better", C.c_int), ("nevals", C.c_int), ("niter", C.c_int), ("converged", C.c_int),
                ("pad", C.c_int)]


class RefineReq(C.Structure):
    _fields_ = [("iref", C.c_int), ("iptcl", C.c_int), ("irot", C.c_int), ("pad", C.c_int),
                ("x0", C.c_double * 3)]


class RefineOut(C.Structure):
    _fields_ = [("x", C.c_double * 3), ("f", C.c_double), ("nevals", C.c_int), ("niter", C.c_int),
                ("converged", C.c_int), ("pad", C.c_int)]


class PrepOpts(C.Structure):
    _fields_ = [("msk", C.c_float), ("inner", C.c_float), ("width", C.c_float), ("focusmsk", C.c_float),
                ("griddev", C.c_int)]


class Tuning(C.Structure):
    _fields_ = [("w_rows", C.c_int), ("w_cols", C.c_int), ("s1_stages", C.c_int), ("from_wisdom", C.c_int)]


class ShsrchOpts(C.Structure):
    _fields_ = [("opt_angle", C.c_int), ("coarse_init", C.c_int), ("maxits", C.c_int), ("max_evals", C.c_int),
                ("halfrot", C.c_float), ("pad", C.c_int)]


class ShsrchReq(C.Structure):
    _fields_ = [("iref", C.c_int), ("iptcl", C.c_int), ("irot", C.c_int), ("pad", C.c_int),
                ("lims", (C.c_float * 2) * 2)]


class ShsrchOut(C.Structure):
    _fields_ = [("irot", C.c_int), ("found_better", C.c_int), ("nevals", C.c_int), ("ncycles", C.c_int),
                ("corr", C.c_float), ("shift", C.c_float * 2), ("pad", C.c_float)]


class SnhcOut(C.Structure):
    _fields_ = [("iref", C.c_int), ("irot", C.c_int), ("found_better", C.c_int), ("nrefs_eval", C.c_int),
                ("corr", C.c_float), ("pad", C.c_int * 3)]


# every exported entry point with its argument types (restype is int unless noted)
_h = C.c_void_p
_fp, _dp, _ip, _vp = C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_void_p
SIGNATURES = {
    "pftcc_new": [C.POINTER(Config), _ip, _ip, C.POINTER(_h)],
    "pftcc_kill": [_h],
    "pftcc_reallocate_ptcls": [_h, C.c_int, _ip],
    "pftcc_set_ref_pft": [_h, C.c_int, _fp, C.c_int],
    "pftcc_set_ptcl_pft": [_h, C.c_int, _fp],
    "pftcc_set_ref_fcomp": [_h, C.c_int, C.c_int, C.c_int, _fp, C.c_int],
    "pftcc_cp_even2odd_ref": [_h, C.c_int],
    "pftcc_cp_even_ref2ptcl": [_h, C.c_int, C.c_int],
    "pftcc_swap_ptclsevenodd": [_h],
    "pftcc_set_eo": [_h, C.c_int, C.c_int],
    "pftcc_set_eos": [_h, _ip],
    "pftcc_zero_refs_beyond_kstop": [_h],
    "pftcc_set_refs": [_h, C.c_int, C.c_int, _fp, C.c_int],
    "pftcc_set_ptcls": [_h, C.c_int, C.c_int, _fp],
    "pftcc_create_polar_absctfmats": [_h, C.POINTER(CtfParams)],
    "pftcc_polarize_ptcls": [_h, C.c_int, C.c_int, _fp, C.c_int],
    "pftcc_polarize_ptcls_dev": [_h, C.c_int, C.c_int, _vp, C.c_int],
    "pftcc_polarize_refs": [_h, C.c_int, C.c_int, _fp, C.c_int, C.c_int],
    "pftcc_set_volume_ft": [_h, _fp, C.c_int, C.c_float],
    "pftcc_fproject_polar": [_h, C.c_int, C.c_int, _fp, C.POINTER(C.c_int), C.c_int, C.c_int],
    "pftcc_memoize_ffts": [_h],
    "pftcc_gencorrs": [_h, C.c_int, C.c_int, _fp, _fp],
    "pftcc_gencorr_for_rot": [_h, C.c_int, C.c_int, _fp, C.c_int, _fp],
    "pftcc_gencorr_for_rot_8": [_h, C.c_int, C.c_int, _dp, C.c_int, _dp],
    "pftcc_gencorr_grad_for_rot_8": [_h, C.c_int, C.c_int, _dp, C.c_int, _dp, _dp],
    "pftcc_gencorr_grad_only_for_rot_8": [_h, C.c_int, C.c_int, _dp, C.c_int, _dp],
    "pftcc_genfrc": [_h, C.c_int, C.c_int, C.c_int, _fp, _fp],
    "pftcc_specscore": [_h, C.c_int, C.c_int, C.c_int, _fp, _fp],
    "pftcc_specscore_batch": [_h, C.c_int, _ip, _ip, _ip, _fp, _fp, _fp],
    "pftcc_prep_ptcls": [_h, C.c_int, C.c_int, _fp, C.c_int, _fp, _ip, C.POINTER(CtfParams), C.c_float],
    "pftcc_prep_ptcls_dev": [_h, C.c_int, C.c_int, C.c_void_p, C.c_int, _fp, _ip, C.POINTER(CtfParams), C.c_float],
    "pftcc_prep_ptcls_opts": [_h, C.c_int, C.c_int, _fp, C.c_int, _fp, _ip, C.POINTER(CtfParams), C.POINTER(PrepOpts)],
    "pftcc_prep_ptcls_opts_dev": [_h, C.c_int, C.c_int, C.c_void_p, C.c_int, _fp, _ip, C.POINTER(CtfParams),
                                  C.POINTER(PrepOpts)],
    "pftcc_fdf_project_polar": [_h, C.c_int, C.c_int, _dp, C.c_int],
    "pftcc_get_dref_pft": [_h, C.c_int, C.c_int, _fp],
    "pftcc_gencorr_cont_shift_grad_cc_for_rot_8": [_h, C.c_int, C.c_int, _dp, C.c_int, _dp, _dp],
    "pftcc_gencorr_cont_grad_cc_for_rot_8": [_h, C.c_int, C.c_int, _dp, C.c_int, _dp, _dp],
    "pftcc_cont_shift_grad_batch": [_h, C.c_int, C.POINTER(GradReq), _dp, _dp],
    "pftcc_orisrch_batch": [_h, C.c_int, C.POINTER(OrisrchReq), C.c_int, C.c_double, C.c_double,
                            C.POINTER(OrisrchOut)],
    "pftcc_cp_refs": [_h, _h],
    "pftcc_set_ptcl_fcomp": [_h, C.c_int, C.c_int, C.c_int, _fp],
    "pftcc_calc_ptcl_pspec": [_h, C.c_int, _fp],
    "pftcc_assign_pinds": [_h, _ip],
    "pftcc_calc_roinv_corrmat": [_h, _fp],
    "pftcc_set_ref_optlp": [_h, C.c_int, _fp],
    "pftcc_set_pssnr": [_h, C.c_int],
    "pftcc_prep_matchfilt": [_h, C.c_int, C.c_int, C.c_int],
    "pftcc_prep_matchfilt_batch": [_h, C.c_int, _ip, _ip, _ip],
    "pftcc_set_objfun": [_h, C.c_int],
    "pftcc_assign_sigma2_noise": [_h, C.c_int, C.c_int, _fp],
    "pftcc_gencorrs_euclid": [_h, C.c_int, C.c_int, _fp, _fp],
    "pftcc_gencorr_euclid_for_rot": [_h, C.c_int, C.c_int, _fp, C.c_int, _fp],
    "pftcc_gencorr_euclid_for_rot_8": [_h, C.c_int, C.c_int, _dp, C.c_int, _dp],
    "pftcc_gencorr_euclid_grad_for_rot_8": [_h, C.c_int, C.c_int, _dp, C.c_int, _dp, _dp],
    "pftcc_gencorr_euclid_grad_only_for_rot_8": [_h, C.c_int, C.c_int, _dp, C.c_int, _dp],
    "pftcc_gencorr_sigma_contrib": [_h, C.c_int, C.c_int, _fp, C.c_int, _fp, _fp, _fp],
    "pftcc_sigma_contrib_batch": [_h, C.c_int, _ip, _ip, _ip, _fp, _fp, _fp, _fp],
    "pftcc_corr_all": [_h, C.c_int, _fp, _fp],
    "pftcc_corr_all_prec": [_h, C.c_int, _fp, C.c_int, _fp],
    "pftcc_search_best": [_h, C.c_int, _fp, C.c_int, C.c_int, C.POINTER(Best)],
    "pftcc_search_best_dev": [_h, C.c_int, _fp, C.c_int, C.c_int, _vp],
    "pftcc_search_groups": [_h, C.c_int, _ip, _ip, _ip, _ip, C.c_int, _fp, C.c_int, C.c_int, C.POINTER(Best)],
    "pftcc_search_groups_dev": [_h, C.c_int, _ip, _ip, _ip, _ip, C.c_int, _fp, C.c_int, C.c_int, _vp],
    "pftcc_search_check": [_h],
    "pftcc_grad_batch": [_h, C.c_int, C.POINTER(GradReq), _dp, _dp],
    "pftcc_refine_batch": [_h, C.c_int, C.POINTER(RefineReq), _dp, _dp, C.c_int, C.c_double, C.c_double,
                           C.POINTER(RefineOut)],
    "pftcc_gencorrs_noalloc": [_h, C.c_int, _ip, _ip, _fp, _vp],
    "pftcc_set_tuning": [_h, C.POINTER(Tuning)],
    "pftcc_get_tuning": [_h, C.POINTER(Tuning)],
    "pftcc_autotune": [_h, C.c_int, _fp, C.c_int, C.c_int, C.c_char_p, C.POINTER(Tuning)],
    "pftcc_shsrch_batch": [_h, C.c_int, C.POINTER(ShsrchOpts), C.c_int, C.POINTER(ShsrchReq), C.POINTER(ShsrchOut)],
    "pftcc_search_snhc": [_h, _ip, _fp, _ip, C.c_int, C.c_ulonglong, C.c_int, C.POINTER(SnhcOut)],
    "pftcc_get_nrots": [_h, _ip],
    "pftcc_get_pftsz": [_h, _ip],
    "pftcc_get_pdim": [_h, _ip],
    "pftcc_get_box": [_h, _ip],
    "pftcc_get_nrefs": [_h, _ip],
    "pftcc_get_nptcls": [_h, _ip],
    "pftcc_get_rot": [_h, C.c_int, _fp],
    "pftcc_get_roind": [_h, C.c_float, _ip],
    "pftcc_get_coord": [_h, C.c_int, C.c_int, _fp],
    "pftcc_ptcl_iseven": [_h, C.c_int, _ip],
    "pftcc_get_ref_pft": [_h, C.c_int, C.c_int, _fp],
    "pftcc_get_ptcl_pft": [_h, C.c_int, _fp],
    "pftcc_get_sqsum_ptcl": [_h, C.c_int, _fp],
    "pftcc_exists": [_h, _ip],
    "pftcc_strerror": ([C.c_int], C.c_char_p),
    "pftcc_last_error": ([_h], C.c_char_p),
    "pftcc_kernel_launches": ([_h], C.c_longlong),
    "pftcc_synchronize": [_h],
    "pftcc_set_stream": [_h, _vp],
    "pftcc_set_wait_limit": [_h, C.c_longlong],
    "pftcc_prof_enable": [_h, C.c_int],
    "pftcc_prof_read": [_h, C.c_int, _dp, C.POINTER(C.c_longlong)],
    "pftcc_prof_reset": [_h],
}

# kernel classes of the per-kernel timing (PFTCC_K_*)
KERNEL_CLASSES = ["polarize", "ctfmat", "spec_ptcl", "spec_ref", "pack", "stage1", "norm", "stage2", "exact",
                  "other"]

_LIB = None


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load libpftcc_b200.so (building it with nvcc first if it is absent)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = lib_path()
    if not os.path.exists(path):
        if not build_if_missing:
            raise RuntimeError(f"{path} is missing: run __graft_entry__.build()")
        _build.build()
    L = C.CDLL(path)
    for name, sig in SIGNATURES.items():
        fn = getattr(L, name)
        if isinstance(sig, tuple):
            fn.argtypes, fn.restype = sig
        else:
            fn.argtypes, fn.restype = sig, C.c_int
    _LIB = L
    return L
