/*
 * pftcc_b200.h -- C ABI of the B200 polar Fourier correlation search.
 *
 * Each entry point replaces one type-bound procedure of SIMPLE 3.0's
 * polarft_corrcalc (src/main/simple_polarft_corrcalc.f90, cited below by line)
 * so that a Fortran shim type with the same procedure names can forward to it
 * through ISO_C_BINDING.  Conventions:
 *   - every function returns an int status (PFTCC_OK = 0); the shim maps a
 *     non-zero status to THROW_HARD, which is what the reference does on error;
 *   - indices are 1-based as in the reference: iref in 1..nrefs, iptcl a GLOBAL
 *     particle index in pfromto(1)..pfromto(2) mapped through pinds, irot in
 *     1..nrots with irot = 1 the zero rotation;
 *   - a polar FT is nrots/2 x (kto-kfrom+1) complex single precision, Fortran
 *     column-major pft(pftsz, kfrom:kto), passed as interleaved (re, im) floats;
 *   - all buffers are host memory unless the name ends in _dev; the library
 *     copies what it is given and never keeps a caller pointer;
 *   - calls on one handle are serialised by the caller (the reference's setters
 *     are likewise called outside the OpenMP search loops); the per-pair
 *     correlation calls are thread safe (an internal lock orders them).
 */
#ifndef PFTCC_B200_H
#define PFTCC_B200_H
#ifdef __cplusplus
extern "C" {
#endif

enum {
    PFTCC_OK = 0,
    PFTCC_ERR_ARG = 1,          /* bad dimensions, sizes or flags            */
    PFTCC_ERR_INDEX = 2,        /* iref / iptcl / irot out of range          */
    PFTCC_ERR_STATE = 3,        /* call out of order (e.g. no CTF matrices)  */
    PFTCC_ERR_CUDA = 4,         /* CUDA runtime or launch error              */
    PFTCC_ERR_OOM = 5,          /* device allocation failed                  */
    PFTCC_ERR_TIMEOUT = 6,      /* a bounded device wait ran out             */
    PFTCC_ERR_NODEV = 7,        /* no usable sm_100 device                   */
    PFTCC_ERR_UNSUPPORTED = 8   /* a reference mode this build does not serve */
};

enum { PFTCC_FRAME_REF = 0,     /* |CTF| applied to the reference at the reference's own
                                   polar index, exactly as prep_ref4corr :982 / :1527     */
       PFTCC_FRAME_PTCL = 1 };  /* |CTF| at the particle's polar index n+rot with the
                                   rotation-dependent normaliser sum |ref|^2 CTF^2(n+rot);
                                   equal to FRAME_REF for an isotropic CTF               */
/* params_glob%cc_objfun (simple_defs.f90:61): the objective gencorrs / gencorr_for_rot(_8) /
 * gencorr_grad_for_rot_8 / the batched searches evaluate */
enum { PFTCC_OBJFUN_CC = 0, PFTCC_OBJFUN_EUCLID = 1 };

enum { PFTCC_PREC_EXACT = 0,    /* FP32 direct sums per (ref, ptcl, shift), FRAME_REF/PTCL  */
       PFTCC_PREC_FP32 = 1,     /* m-domain contraction on CUDA cores (FP32), FRAME_PTCL    */
       PFTCC_PREC_BF16X3 = 2 }; /* m-domain contraction on tcgen05, BF16 hi+lo split with
                                   three products and FP32 accumulation, FRAME_PTCL         */

typedef struct pftcc_handle pftcc_handle;

/* new() arguments plus the params_glob fields polarft_corrcalc reads implicitly
 * (boxmatch :235, ring2 -> nrots :251-252, kfromto/kstop :256-258, ctf :355-356,
 * l_match_filt :254; l_pssnr through pftcc_set_pssnr).  Not served: clsfrcs = 'yes'
 * (l_clsfrcs :415, which filters with the column ref_optlp(:, iptcl) of the particle's global
 * index, :976-980): ref_optlp is allocated with nrefs columns (:255), so that mode reads past the
 * array for every iptcl > nrefs and has no defined result to reproduce; the matched filter is
 * always ref_optlp(:, iref). */
typedef struct {
    int nrefs;            /* new(nrefs, ...)                                    */
    int pfromto[2];       /* new(..., pfromto, ...), global particle index range */
    int box;              /* params_glob%boxmatch, even                         */
    int nrots;            /* 2*magic_pftsz(ring2), even                         */
    int kfromto[2];       /* params_glob%kfromto                                */
    int kstop;            /* params_glob%kstop, kfromto(1) <= kstop <= kfromto(2) */
    int with_ctf;         /* params_glob%ctf /= 'no'                            */
    int match_filt;       /* params_glob%l_match_filt: branch of gencorr_*_for_rot_8 */
    int ctf_frame;        /* PFTCC_FRAME_REF (reference semantics) or PFTCC_FRAME_PTCL */
    int device;           /* CUDA device ordinal                                */
} pftcc_config;

/* spproj%get_ctfparams (simple_polarft_corrcalc.f90:948) for one particle */
typedef struct {
    float smpd, kv, cs, fraca;  /* A/pixel, kV, mm, amplitude contrast         */
    float dfx, dfy, angast;     /* microns, microns, degrees                   */
    float phshift;              /* radians (phase plate)                       */
    int l_phaseplate;
} pftcc_ctfparams;

/* one search result per particle: 16 bytes */
typedef struct { int iref; int irot; int ishift; float corr; } pftcc_best;

/* one request of the adjoint: f and d f / d(shift_x, shift_y, defocus) */
typedef struct { int iref, iptcl, irot, pad; double sx, sy, ddf; } pftcc_grad_req;

/* ---- construction / destruction ------------------------------------------------ */
/* new :209-422.  ptcl_mask (length pfromto(2)-pfromto(1)+1, nullable) selects the
 * particles held (:245-249, :276-288); eoarr (same length, nullable) the even/odd
 * assignment (:289-306; -1 everywhere = all even). */
int pftcc_new(const pftcc_config *cfg, const int *ptcl_mask, const int *eoarr, pftcc_handle **out);
/* kill :2234-2279 */
int pftcc_kill(pftcc_handle *h);
/* reallocate_ptcls :509-555 (pinds = global indices of the nptcls particles) */
int pftcc_reallocate_ptcls(pftcc_handle *h, int nptcls, const int *pinds);

/* ---- setters -------------------------------------------------------------------- */
int pftcc_set_ref_pft(pftcc_handle *h, int iref, const float *pft, int iseven);           /* :426-436 */
int pftcc_set_ptcl_pft(pftcc_handle *h, int iptcl, const float *pft);                     /* :438-445 */
int pftcc_set_ref_fcomp(pftcc_handle *h, int iref, int irot, int k, const float *comp, int iseven); /* :447-457 */
int pftcc_cp_even2odd_ref(pftcc_handle *h, int iref);                                     /* :485-489 */
int pftcc_cp_even_ref2ptcl(pftcc_handle *h, int iref, int iptcl);                         /* :497-502 */
int pftcc_swap_ptclsevenodd(pftcc_handle *h);                                             /* :504-507 */
int pftcc_set_eo(pftcc_handle *h, int iptcl, int is_even);                                /* :557-562 */
int pftcc_set_eos(pftcc_handle *h, const int *eoarr);                                     /* :564-579 */
int pftcc_zero_refs_beyond_kstop(pftcc_handle *h);                                        /* :747-754 */
/* bulk setters (no reference counterpart; what a batched shim uses): refs [n][K][P] */
int pftcc_set_refs(pftcc_handle *h, int first_iref, int n, const float *pfts, int iseven);
int pftcc_set_ptcls(pftcc_handle *h, int first_slot, int n, const float *pfts);

/* ---- CTF ------------------------------------------------------------------------ */
/* create_polar_absctfmats :906-959 given the per-particle parameters (params[i]
 * belongs to the particle in slot i, i.e. global index pinds^-1(i)) */
int pftcc_create_polar_absctfmats(pftcc_handle *h, const pftcc_ctfparams *params);

/* ---- polarizer ------------------------------------------------------------------ */
/* init_polarizer + polarize (simple_polarizer.f90:41-151) for n particles in slots
 * first_slot.. from half-plane FTs cmat(box/2+1, box) (Fortran order, complex
 * interleaved); griddev as params_glob%griddev == 'yes' */
int pftcc_polarize_ptcls(pftcc_handle *h, int first_slot, int n, const float *cmats, int griddev);
int pftcc_polarize_ptcls_dev(pftcc_handle *h, int first_slot, int n, const void *cmats_dev, int griddev);
int pftcc_polarize_refs(pftcc_handle *h, int first_iref, int n, const float *cmats, int iseven, int griddev);

/* ---- particle ingestion --------------------------------------------------------------- */
/* spproj%get_ctfparams(...)%ctfflag (simple_defs.f90:55) */
enum { PFTCC_CTFFLAG_NO = 0, PFTCC_CTFFLAG_YES = 1, PFTCC_CTFFLAG_FLIP = 2 };
/* prepimg4align (simple_strategy2D3D_common.f90:316-366) followed by polarize
 * (build_pftcc_batch_particles :353-376) for n particle images of side box_in (even,
 * >= boxmatch = cfg.box), imgs [n][box_in][box_in] real, rmat(x, y) order: noise normalisation
 * against the background outside the disc of radius msk, FFT, shift by -(x, y) = -xy[2 i..],
 * the CTF phase flip for ctfflag[i] == PFTCC_CTFFLAG_YES (ctf[i]; ctf may be NULL when no flag
 * is YES), inverse FFT, clip to boxmatch, soft mask of radius msk,
 * FFT and the factor boxmatch^2 / box_in^2, then the polar gridding into slots
 * first_slot..first_slot+n-1 (griddev 'no'); the _dev form takes the images in device memory */
int pftcc_prep_ptcls(pftcc_handle *h, int first_slot, int n, const float *imgs, int box_in, const float *xy,
                     const int *ctfflag, const pftcc_ctfparams *ctf, float msk);
int pftcc_prep_ptcls_dev(pftcc_handle *h, int first_slot, int n, const void *imgs_dev, int box_in, const float *xy,
                         const int *ctfflag, const pftcc_ctfparams *ctf, float msk);
/* the same with prepimg4align's other mask modes (:349-362): msk as above (the noise
 * normalisation's disc, build_glob%lmsk); inner > 0 (params_glob%l_innermsk) masks with the
 * inner cosine edge too, mask(msk, 'soft', inner, width), width <= 0 meaning the default 10;
 * else focusmsk > 0 (params_glob%l_focusmsk) takes mask(focusmsk, 'soft') for the final mask;
 * griddev = 1 (params_glob%griddev 'yes') divides the masked image by the gridding's instrument
 * function (div_by_instrfun, simple_polarizer.f90:111-116) and grids with un-normalised
 * weights (init_polarizer :87) */
typedef struct { float msk, inner, width, focusmsk; int griddev; } pftcc_prep_opts;
int pftcc_prep_ptcls_opts(pftcc_handle *h, int first_slot, int n, const float *imgs, int box_in, const float *xy,
                          const int *ctfflag, const pftcc_ctfparams *ctf, const pftcc_prep_opts *opts);
int pftcc_prep_ptcls_opts_dev(pftcc_handle *h, int first_slot, int n, const void *imgs_dev, int box_in, const float *xy,
                              const int *ctfflag, const pftcc_ctfparams *ctf, const pftcc_prep_opts *opts);

/* ---- polar projection of a volume -------------------------------------------------- */
/* projector%expand_cmat (simple_projector.f90:66-132): the volume's half FT
 * image%cmat(box/2+1, box, box) (Fortran order, complex interleaved; even box with
 * kfromto(2) <= box/2) expanded on the device by cyclic addressing and Friedel symmetry,
 * times factor (1 unless norm4proj) */
int pftcc_set_volume_ft(pftcc_handle *h, const float *cmat_half, int box, float factor);
/* projector%fproject_polar (simple_projector.f90:218-239) for n orientations at once:
 * references first_iref..first_iref+n-1 of the even (iseven != 0) or odd set from Spider
 * Euler triplets euls[3 n] in degrees (ori%get_mat = euler2m, simple_ori.f90:1275), the
 * 3x3x3 Kaiser-Bessel interpolation of interp_fcomp (:269-307; griddev != 0 skips the
 * normalisation by the weights' sum); mask: K ints for shells kfrom..kto (0 = set to zero)
 * or NULL for all */
int pftcc_fproject_polar(pftcc_handle *h, int first_iref, int n, const float *euls, const int *mask, int iseven,
                         int griddev);
/* projector%fdf_project_polar (simple_projector.f90:245-267, fdf_interp_fcomp :338-400) for n
 * orientations: the normalised sections into references first_iref.. of set iseven
 * (set_ref_fcomp :447-457) and their derivatives with respect to the Euler angles e1, e2, e3
 * (per radian; euler2dm, simple_ori_light.f90:87-147) into the derivative references
 * (set_dref_fcomp :459-469); euls[3 n] in degrees, double as the reference's real(dp) */
int pftcc_fdf_project_polar(pftcc_handle *h, int first_iref, int n, const double *euls, int iseven);
/* the derivative references of iref: dpft [3][K][P] complex (d/de1, d/de2, d/de3) */
int pftcc_get_dref_pft(pftcc_handle *h, int iref, int iseven, float *dpft);

/* ---- memoisers ------------------------------------------------------------------ */
/* memoize_ffts :848-861: prepares the particle-side angular spectra of the
 * m-domain search (no-op for the exact path, which needs none) */
int pftcc_memoize_ffts(pftcc_handle *h);

/* ---- correlators ---------------------------------------------------------------- */
/* gencorrs_1 / gencorrs_2 (:1594-1617 -> :1486-1534); shvec nullable -> gencorrs_cc_1 */
int pftcc_gencorrs(pftcc_handle *h, int iref, int iptcl, const float *shvec, float *cc);
/* gencorr_for_rot :1619-1630 and gencorr_for_rot_8 :1632-1643 */
int pftcc_gencorr_for_rot(pftcc_handle *h, int iref, int iptcl, const float *shvec, int irot, float *cc);
int pftcc_gencorr_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot, double *cc);
/* gencorr_grad_for_rot_8 :1849-1861 and gencorr_grad_only_for_rot_8 :1927-1939 */
int pftcc_gencorr_grad_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                 double *f, double *grad);
int pftcc_gencorr_grad_only_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                      double *grad);

/* ---- remaining procedures of the object ----------------------------------------------- */
/* cp_refs (:491-495): both reference sets copied from src (same nrefs, shells and angles) */
int pftcc_cp_refs(pftcc_handle *h, const pftcc_handle *src);
/* set_ptcl_fcomp (:471-476): one component pfts_ptcls(irot, k, pinds(iptcl)) = comp[2]
 * (irot 1..nrots/2, k kfrom..kto); the square sum is not refreshed, as in the reference */
int pftcc_set_ptcl_fcomp(pftcc_handle *h, int iptcl, int irot, int k, const float *comp);
/* calc_ptcl_pspec (:897-904): pspec[kto - kfrom + 1], the mean power of each shell */
int pftcc_calc_ptcl_pspec(pftcc_handle *h, int iptcl, float *pspec);
/* assign_pinds (:706-710): pinds[pfromto(2) - pfromto(1) + 1], each index's slot (1-based, 0 = not held) */
int pftcc_assign_pinds(const pftcc_handle *h, int *pinds);
/* calc_roinv_corrmat (:2207-2231), particles and references the same set (nptcls == nrefs):
 * corrmat[nptcls][nptcls], the best in-plane correlation of reference i with particle pfrom + j
 * for i < j (gencorrs maxloc), symmetrised, 1 on the diagonal */
int pftcc_calc_roinv_corrmat(pftcc_handle *h, float *corrmat);

/* ---- the matched-filter mode (pftcc_config.match_filt = params_glob%l_match_filt) ---------- */
/* params_glob%l_pssnr (implies l_match_filt, simple_parameters.f90:1364-1365): the shell
 * factors of shellnorm_and_filter_ref(_8) become sqrt(ssnr k) / sqrt(power) (:763-770,
 * :789-796) with ssnr = ref_optlp(k, iref), and prep_matchfilt rescales the particle's shells
 * by sqrt(k) / sqrt(power) and sqrt(1 + ssnr |CTF|^2) per sample (:999-1019).
 * PFTCC_ERR_STATE on a handle created without match_filt. */
int pftcc_set_pssnr(pftcc_handle *h, int on);
/* With match_filt the correlators apply shellnorm_and_filter_ref(_8) (:756-807) to the reference:
 * shell k <= kstop scaled by ref_optlp(k, iref) / sqrt(mean power of the raw shell) (gencorrs_cc_1/_2,
 * gencorrs_euclid_1, gencorr_cc_for_rot(_8), gencorr_cc_grad_for_rot_8, the continuous-gradient
 * correlators' reference, genfrc / calc_frc, the batched searches).  set_ref_optlp (:587-592):
 * ref_optlp(kfrom:kstop, iref) = optlp[kstop - kfrom + 1] (1 until set). */
int pftcc_set_ref_optlp(pftcc_handle *h, int iref, const float *optlp);
/* prep_matchfilt (:987-1095), l_match_filt branch: particle iptcl re-weighted in place against
 * reference iref (its eo set, times |CTF|) at rotation irot by the shell-normalised, Savitzky-Golay
 * smoothed Wiener-like filter; iref 0 or match_filt off: nothing to do.  The batch holds each
 * particle at most once. */
int pftcc_prep_matchfilt(pftcc_handle *h, int iptcl, int iref, int irot);
int pftcc_prep_matchfilt_batch(pftcc_handle *h, int n, const int *iptcl, const int *iref, const int *irot);

/* ---- the orientation gradient (reference frame only) -------------------------------- */
/* gencorr_cont_shift_grad_cc_for_rot_8 (:1788-1847): f and grad[5] = d f / d(e1, e2, e3, sx, sy)
 * at rotation irot from the references and derivative references of fdf_project_polar; the
 * orientation part correlates the derivative references with particle iptcl */
int pftcc_gencorr_cont_shift_grad_cc_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                               double *f, double *grad);
/* gencorr_cont_grad_cc_for_rot_8 (:1735-1786): cc and dcc[3] = d cc / d(e1, e2, e3) */
int pftcc_gencorr_cont_grad_cc_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                         double *cc, double *dcc);
/* n requests in one launch (req[i].ddf unused): f[n], grad5[n][5] */
int pftcc_cont_shift_grad_batch(pftcc_handle *h, int n, const pftcc_grad_req *req, double *f, double *grad5);
/* pftcc_orisrch_grad%minimize (simple_pftcc_orisrch_grad.f90:60-122) for n particles at once on the
 * volume of pftcc_set_volume_ft: variables (e1, e2, e3) in degrees within e +- angerr_deg and a
 * shift within +- maxhwshift, started at (e, 0, 0); cost -corr of
 * gencorr_cont_shift_grad_cc_for_rot_8 at irot = 1 on the sections of fdf_project_polar at the
 * trial angles, its gradient as that routine gives it (angle components per radian);
 * bound-constrained L-BFGS (pgtol, factr as pftcc_refine_batch).  out: the angles and the shift
 * rotated by rotmat2d(e3) when the cost fell below its start (found_better), else the input
 * angles and a zero shift; corr and the starting corr_init.  One volume per call: odd and even
 * particles whose volumes differ are searched in two calls. */
typedef struct { int iptcl, pad; double e[3]; double angerr_deg, maxhwshift; } pftcc_orisrch_req;
typedef struct { double e[3], shift[2], corr, corr_init; int found_better, nevals, niter, converged, pad; } pftcc_orisrch_out;
int pftcc_orisrch_batch(pftcc_handle *h, int n, const pftcc_orisrch_req *req, int maxits, double pgtol, double factr,
                        pftcc_orisrch_out *out);

/* ---- the Euclidean objective (reference frame only) -------------------------------- */
/* params_glob%cc_objfun: PFTCC_OBJFUN_EUCLID makes pftcc_gencorrs, pftcc_gencorr_for_rot(_8),
 * pftcc_gencorr_grad(_only)_for_rot_8 and the PFTCC_PREC_EXACT batched searches evaluate the
 * Euclidean objective, as gencorrs_1/_2 (:1594-1617), gencorr_for_rot(_8) (:1619-1643) and
 * gencorr_grad(_only)_for_rot_8 (:1849-1939) dispatch on it (reference frame).  On a
 * particle-frame handle the FP32 / BF16X3 batched searches evaluate it instead, with the CTF at
 * the particle's polar index: -1/2 sum_k w_k sum_n |ref shmat ctf~(n+rot) - ptcl~(n+rot)|^2,
 * w_k = pxls(k) / (P sigma2(k)) (the exact and per-pair calls refuse it there) */
int pftcc_set_objfun(pftcc_handle *h, int objfun);
/* assign_sigma2_noise (:581-585): sigma2_noise(kfrom:kto, fromp:top), column-major, i.e.
 * [top - fromp + 1][kto - kfrom + 1].  The values are copied: assign again after changing them.
 * Every held particle needs a column before a Euclidean evaluation. */
int pftcc_assign_sigma2_noise(pftcc_handle *h, int fromp, int top, const float *sigma2);
/* gencorrs_euclid_1 (:1536-1557, shvec NULL) / gencorrs_euclid_2 (:1559-1592), euclids[nrots] */
int pftcc_gencorrs_euclid(pftcc_handle *h, int iref, int iptcl, const float *shvec, float *euclids);
/* gencorr_euclid_for_rot (:2002-2024) / _8 (:2026-2048) */
int pftcc_gencorr_euclid_for_rot(pftcc_handle *h, int iref, int iptcl, const float *shvec, int irot, float *f);
int pftcc_gencorr_euclid_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot, double *f);
/* gencorr_euclid_grad_for_rot_8 (:2071-2109) / gencorr_euclid_grad_only_for_rot_8 (:2111-2148) */
int pftcc_gencorr_euclid_grad_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                        double *f, double *grad);
int pftcc_gencorr_euclid_grad_only_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                             double *grad);
/* gencorr_sigma_contrib (:2150-2188): sigma_contrib[K] (and, when not NULL, ptcl_sumsq[K],
 * ref_sumsq[K]) over every shell kfrom..kto; needs no sigma2 */
int pftcc_gencorr_sigma_contrib(pftcc_handle *h, int iref, int iptcl, const float *shvec, int irot,
                                float *sigma_contrib, float *ptcl_sumsq, float *ref_sumsq);
/* gencorr_sigma_contrib for n requests in one launch: sigma_contrib [n][K] (ptcl_sumsq,
 * ref_sumsq likewise, or NULL), shifts [n][2] (the loop of euclid_sigma2%calc_sigma2 :107-120) */
int pftcc_sigma_contrib_batch(pftcc_handle *h, int n, const int *iref, const int *iptcl, const int *irot,
                              const float *shifts, float *sigma_contrib, float *ptcl_sumsq, float *ref_sumsq);

/* ---- batched entry points (no single reference counterpart) ---------------------- */
/* genfrc (:1417-1441) / calc_frc (:1443-1484): the per-shell correlation at irot,
 * frc[k - kfrom] for k = kfrom..kstop, each shell normalised by
 * sqrt(sum|ptcl_k|^2 * sum|ref_k|^2) and 0 where that is below 1e-12; the reference
 * is prepared in the reference frame (ref * ctf, times the shift phases when shvec is
 * given).  specscore_1/_2 (:2190-2205): max(0, median of those values), the median
 * of median_nocopy (simple_math.f90:2111-2130).  The batch serves n (iref, iptcl, irot)
 * requests in one launch; shifts is [n][2] or NULL, frcs [n][kstop-kfrom+1] or NULL. */
int pftcc_genfrc(pftcc_handle *h, int iref, int iptcl, int irot, const float *shvec, float *frc);
int pftcc_specscore(pftcc_handle *h, int iref, int iptcl, int irot, const float *shvec, float *score);
int pftcc_specscore_batch(pftcc_handle *h, int n, const int *iref, const int *iptcl, const int *irot,
                          const float *shifts, float *scores, float *frcs);

/* all correlations: cc[slot][iref-1][ishift][irot-1] for every held particle,
 * reference and shift (the loop strategy2D_greedy :42 runs over gencorrs) */
int pftcc_corr_all(pftcc_handle *h, int nshifts, const float *shifts, float *cc);
/* all correlations through the m-domain path in the given precision (PFTCC_PREC_FP32 or
 * PFTCC_PREC_BF16X3; PFTCC_PREC_EXACT = pftcc_corr_all), particle frame, same layout
 * as pftcc_corr_all: the full array the precision report measures */
int pftcc_corr_all_prec(pftcc_handle *h, int nshifts, const float *shifts, int precision, float *cc);
/* best (ref, rot, shift) per particle over all references and a shift grid, the
 * greedy strategies' maxloc (simple_strategy2D_greedy.f90:42-43) fused with the
 * coarse shift grid of minimize_exhaustive (simple_pftcc_shsrch_grad.f90:182-199).
 * ntop > 0 re-scores the ntop best (ref, shift) candidates per particle with the
 * exact FP32 path in cfg.ctf_frame. */
int pftcc_search_best(pftcc_handle *h, int nshifts, const float *shifts, int precision, int ntop,
                      pftcc_best *out);
int pftcc_search_best_dev(pftcc_handle *h, int nshifts, const float *shifts, int precision, int ntop,
                          void *out_dev);
/* The search of a queue of independent chunks held in one handle: group q searches the particle
 * slots slot_first[q]..slot_first[q]+nslot[q]-1 (1-based, disjoint between groups) against the
 * references ref_first[q]..ref_first[q]+nref[q]-1 (1-based) over the shift list, as
 * pftcc_search_best would for that chunk alone (the strategies' matcher loop over its particle
 * batches, simple_strategy2D_matcher.f90:220-297, each batch against its own references); iref
 * in out is the handle's reference index.  m-domain precisions only (PFTCC_PREC_FP32 or
 * PFTCC_PREC_BF16X3), the correlation objective.  Every chunk's (references x shifts) x particles
 * block is a wave; the waves share one persistent tcgen05 stage-1 launch over all their work items
 * (a device-resident wave table) and one stage-2 launch over all their particles.  Slots outside
 * every group return iref = 0, ishift = -1, corr = -inf. */
int pftcc_search_groups(pftcc_handle *h, int ngroups, const int *ref_first, const int *nref, const int *slot_first,
                        const int *nslot, int nshifts, const float *shifts, int precision, int ntop, pftcc_best *out);
/* The same into device memory (out_dev: nptcls pftcc_best records), enqueued on the handle's stream
 * with no host synchronisation and no read-back of the bounded waits' error word (check it with
 * pftcc_search_check once the stream has run).  After one call outside stream capture with the
 * same arguments (which sizes the workspace and the staging of its tables), the call may be
 * captured into a CUDA graph on the handle's stream (pftcc_set_stream); the graph replays the
 * groups and shifts given at capture, and a later capture of a call on the same handle replaces
 * them.  Inside a capture a call that would allocate returns PFTCC_ERR_STATE. */
int pftcc_search_groups_dev(pftcc_handle *h, int ngroups, const int *ref_first, const int *nref, const int *slot_first,
                            const int *nslot, int nshifts, const float *shifts, int precision, int ntop, void *out_dev);
/* the bounded waits' error word of every search since the last check (graph replays included):
 * PFTCC_ERR_TIMEOUT when a wait gave up, and the word is cleared; synchronises the handle's
 * stream, so it is called outside stream capture */
int pftcc_search_check(pftcc_handle *h);
/* adjoint: f and grad3 = d f / d(shift_x, shift_y, defocus[micron]) per request, with
 * the particle's CTF evaluated at defocus + ddf; the shift part is
 * gencorr_grad_for_rot_8 (:1863-1925) in the branch cfg.match_filt selects */
int pftcc_grad_batch(pftcc_handle *h, int nreq, const pftcc_grad_req *req, double *f, double *grad3);
/* continuous refinement: for each request i maximise corr over x = (shift_x, shift_y,
 * defocus offset in microns) inside its own box [lb[i], ub[i]] (lb, ub are [n][3], as the
 * reference bounds each particle's search, simple_pftcc_shsrch_grad.f90:44-68) at the
 * fixed (iref, iptcl, irot),
 * starting from x0 -- the role of pftcc_shsrch_grad%minimize with the reference's
 * L-BFGS-B (simple_pftcc_shsrch_grad.f90:254-338, simple_opt_lbfgsb.f90:103-129)
 * extended to the defocus.  All problems advance together; every round's pending
 * function+gradient evaluations go to the GPU in one adjoint launch.  maxits bounds
 * the iterations, pgtol/factr are L-BFGS-B's stopping tolerances (1e-5 / 1e7 in the
 * reference's defaults). */
typedef struct { int iref, iptcl, irot, pad; double x0[3]; } pftcc_refine_req;
typedef struct { double x[3]; double f; int nevals, niter, converged, pad; } pftcc_refine_out;
int pftcc_refine_batch(pftcc_handle *h, int n, const pftcc_refine_req *req, const double *lb, const double *ub,
                       int maxits, double pgtol, double factr, pftcc_refine_out *out);

/* pftcc_shsrch_grad (simple_pftcc_shsrch_grad.f90:44-391) for n (reference, particle)
 * problems at once, each with its own shift box lims = [[x_lo, x_hi], [y_lo, y_hi]]
 * (ospec%limits).  The optimiser is L-BFGS-B as the reference specifies it (:67-68: line
 * search ftol 1e-1, gtol 1e-3; factr 1e7, pgtol 1e-5, 15 pairs) on the cost
 * -gencorr_for_rot_8 with the gradient of gencorr_grad_for_rot_8 (:85-131, the branch
 * cfg.match_filt selects); maxits bounds its cost+gradient evaluations per run as
 * simple_opt_lbfgsb.f90:120-122 does.  Every round's pending evaluations of all problems
 * go to the GPU in one launch per kind (the single-rotation adjoint; gencorrs over all
 * rotations with maxloc, in the reference frame).
 *   PFTCC_SHSRCH_MINIMIZE, opt_angle = 1 (grad_shsrch_minimize :262-298): the in-plane
 *     index from gencorrs at zero shift, optionally the 5 x 5 coarse grid
 *     (coarse_search_opt_angle :364-389), then up to max_evals cycles of L-BFGS-B (the
 *     in-plane index re-picked by gencorrs at every new iterate, :139-144) each followed by
 *     a re-pick that ends the cycles when it keeps the index.
 *   PFTCC_SHSRCH_MINIMIZE, opt_angle = 0 (:299-337): the fixed in-plane index req.irot,
 *     optionally the 5 x 5 grid of coarse_search (:340-362), one L-BFGS-B run.
 *   PFTCC_SHSRCH_EXHAUSTIVE (minimize_exhaustive :159-251): the coarse grid of step
 *     (hi - lo) / (2 floor((hi - lo) / 4) + 1) around zero, two 3 x 3 refinements at half and
 *     a quarter of the step, with the rotations limited to within halfrot degrees of req.irot
 *     when halfrot > 0 (req.irot <= 0 means get_roind(0)), then L-BFGS-B from the best.
 * out: irot (0 when minimize found nothing better than its start, as the reference
 * signals), found_better, corr = cxy(1), shift = cxy(2:3) rotated into the reference frame
 * by rotmat2d(get_rot(irot)); nevals counts the optimiser's cost+gradient evaluations and
 * ncycles the L-BFGS-B runs. */
enum { PFTCC_SHSRCH_MINIMIZE = 0, PFTCC_SHSRCH_EXHAUSTIVE = 1 };
typedef struct { int opt_angle, coarse_init, maxits, max_evals; float halfrot; int pad; } pftcc_shsrch_opts;
typedef struct { int iref, iptcl, irot, pad; float lims[2][2]; } pftcc_shsrch_req;
typedef struct { int irot, found_better, nevals, ncycles; float corr, shift[2], pad; } pftcc_shsrch_out;
int pftcc_shsrch_batch(pftcc_handle *h, int mode, const pftcc_shsrch_opts *opts, int n, const pftcc_shsrch_req *req,
                       pftcc_shsrch_out *out);

/* wave and tile sizes of the m-domain search (no counterpart in the reference; FFTW's plans
 * and wisdom file play this role there, simple_polarft_corrcalc.f90:391-408): w_rows x w_cols
 * (reference x shift) rows by particle columns per stage-1 / stage-2 round (multiples of 64 and
 * 128; the stage-1 output of a round takes (nrots/2 + 1) w_rows w_cols x 8 bytes), s1_stages the
 * depth of the tcgen05 kernel's row-tile ring (2..4).  0 keeps the automatic choice.  The sizes
 * change only how the work is cut, never a result. */
typedef struct { int w_rows, w_cols, s1_stages, from_wisdom; } pftcc_tuning;
int pftcc_set_tuning(pftcc_handle *h, const pftcc_tuning *t);
int pftcc_get_tuning(const pftcc_handle *h, pftcc_tuning *t);
/* the autotuner: times the search (precision, ntop, the shift list) on the handle's current
 * references and particles over candidate wave sizes and ring depths (coordinate descent from
 * the automatic choice, each candidate run twice and the second run timed with CUDA events) and
 * keeps the fastest on the handle.  With wisdom (a file path, nullable) a line for this search's
 * shape (device, nrots, shells, rows, columns, precision, frame, ntop) is read first and, when
 * found, used without timing (out->from_wisdom = 1); otherwise the tuned line is appended. */
int pftcc_autotune(pftcc_handle *h, int nshifts, const float *shifts, int precision, int ntop, const char *wisdom,
                   pftcc_tuning *out);

/* stochastic neighbourhood hill climbing over the references for every held particle
 * (strategy2D_snhc srch_snhc, simple_strategy2D_snhc.f90:33-93, with shcloc,
 * simple_rnd.f90:273-295): order is [nptcls][nrefs] (slot order; each row the particle's
 * 1-based reference visiting order, s2D%srch_order), prev_corr [nptcls] the particle's
 * previous best correlation, cls_pops [nrefs] the class populations (0 = empty, skipped
 * after being counted) or NULL, nrefs_bound the visit limit (the reference's
 * max(2, min(nrefs, nint(nrefs * (1 - stoch_bound))))).  Every visited reference is
 * correlated over all rotations without shift (gencorrs); shcloc's uniform pick among the
 * rotations with corr >= prev_corr ends the search (found_better = 1), otherwise the
 * greedy best of the visited references is returned.  The random draw of visit isample
 * of particle iptcl is splitmix64(seed + iptcl * 0x9E3779B97F4A7C15 + isample *
 * 0xD1B54A32D192ED03) -> u in [0,1), selecting the floor(u * count)-th improving
 * rotation in rotation order.  precision: PFTCC_PREC_EXACT (the exact kernel, handle's
 * CTF frame) or the m-domain FP32 / BF16X3 paths (particle frame only).  The correlations
 * of all held particles are kept on the device (nptcls * nrefs * nrots floats, at most
 * 32 GiB). */
typedef struct { int iref, irot, found_better, nrefs_eval; float corr; int pad[3]; } pftcc_snhc_out;
int pftcc_search_snhc(pftcc_handle *h, const int *order, const float *prev_corr, const int *cls_pops, int nrefs_bound,
                      unsigned long long seed, int precision, pftcc_snhc_out *out);

/* gencorrs for npairs (reference, particle, shift) pairs that allocates no memory.  It
 * is for callers that cannot let a library call cudaMalloc: applications that hand all
 * device memory to their own pool at start-up (an allocation behind the pool's back can
 * fail or fragment it) and services that must keep a fixed device footprint.  No
 * counterpart in the reference.  The work descriptors live in a fixed 256 KiB device
 * array that every GPU loading the library holds until exit, so npairs is limited to
 * 6553 (larger batches are rejected with PFTCC_ERR_ARG -- split them).  iref/iptcl are
 * 1-based as in pftcc_gencorrs, shifts is [npairs][2] or NULL (gencorrs_cc_1), cc_dev a
 * device buffer of npairs*nrots floats written as cc_dev[pair*nrots + irot-1].  The
 * first call on a device looks up the array's device address, so make that first call
 * before any stream capture; calls that overlap on the GPU race on the shared array --
 * order them on one stream. */
int pftcc_gencorrs_noalloc(pftcc_handle *h, int npairs, const int *iref, const int *iptcl, const float *shifts,
                           float *cc_dev);

/* ---- getters (:597-710) ----------------------------------------------------------- */
int pftcc_get_nrots(const pftcc_handle *h, int *nrots);
int pftcc_get_pftsz(const pftcc_handle *h, int *pftsz);
int pftcc_get_pdim(const pftcc_handle *h, int pdim[3]);
int pftcc_get_box(const pftcc_handle *h, int *box);
int pftcc_get_nrefs(const pftcc_handle *h, int *nrefs);
int pftcc_get_nptcls(const pftcc_handle *h, int *nptcls);
int pftcc_get_rot(const pftcc_handle *h, int roind, float *rot);
int pftcc_get_roind(const pftcc_handle *h, float rot, int *roind);
int pftcc_get_coord(const pftcc_handle *h, int rot, int k, float xy[2]);
int pftcc_ptcl_iseven(const pftcc_handle *h, int iptcl, int *iseven);
int pftcc_get_ref_pft(pftcc_handle *h, int iref, int iseven, float *pft);
int pftcc_get_ptcl_pft(pftcc_handle *h, int iptcl, float *pft);
int pftcc_get_sqsum_ptcl(pftcc_handle *h, int iptcl, float *sqsum);
int pftcc_exists(const pftcc_handle *h, int *exists);

/* ---- runtime ------------------------------------------------------------------------ */
const char *pftcc_strerror(int status);
/* last error message recorded on the handle (never NULL) */
const char *pftcc_last_error(const pftcc_handle *h);
/* number of kernels this handle has launched so far (for launch accounting) */
long long pftcc_kernel_launches(const pftcc_handle *h);
/* block until all device work of the handle is done */
int pftcc_synchronize(pftcc_handle *h);
/* run the handle's work on a caller's CUDA stream (a cudaStream_t; NULL restores the
 * handle's own stream) -- lets a caller order the library with its own kernels and
 * time it with events on that stream */
int pftcc_set_stream(pftcc_handle *h, void *stream);
/* bounded waits of the tensor-core kernels (no counterpart in the reference): a pipeline
 * wait inside k_umma_stage1 gives up after `polls` polls of its barrier (0 restores the
 * default, about a second), the kernel then drains the copies and MMAs it has issued,
 * frees its tensor memory and returns, and the call reports PFTCC_ERR_TIMEOUT.  A short
 * limit lets a caller (or a test) exercise that path on a normal launch. */
int pftcc_set_wait_limit(pftcc_handle *h, long long polls);
/* per-kernel device timing with CUDA events recorded on the handle's stream around
 * each launch of a kernel class (PFTCC_K_*): enable, then read total milliseconds and
 * launch counts (reading synchronises the stream), reset clears the totals */
enum { PFTCC_K_POLARIZE = 0, PFTCC_K_CTFMAT = 1, PFTCC_K_SPEC_PTCL = 2, PFTCC_K_SPEC_REF = 3, PFTCC_K_PACK = 4,
       PFTCC_K_STAGE1 = 5, PFTCC_K_NORM = 6, PFTCC_K_STAGE2 = 7, PFTCC_K_EXACT = 8, PFTCC_K_OTHER = 9,
       PFTCC_K_COUNT = 10 };
int pftcc_prof_enable(pftcc_handle *h, int on);
int pftcc_prof_read(pftcc_handle *h, int kernel_class, double *total_ms, long long *launches);
int pftcc_prof_reset(pftcc_handle *h);

#ifdef __cplusplus
}
#endif
#endif
