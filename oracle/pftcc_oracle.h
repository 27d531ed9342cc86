/*
 * pftcc_oracle.h -- CPU restatement of SIMPLE 3.0's polar Fourier correlation
 * search (polarft_corrcalc), used ONLY as test infrastructure: the checker in
 * tests/, the smoke() parity check and bench.py's cpu_baseline / reference arm.
 * Nothing in the product library links, loads or calls this code.
 *
 * Parity status: the reference (Fortran 2008 + FFTW3) cannot be compiled in
 * this environment (no Fortran compiler, no FFTW), and the reference ships no
 * golden vectors for this path.  The restatement is therefore pinned by
 * known-answer tests derived from the reference formulas (self-correlation,
 * rotation and shift recovery, FFT path == direct path, finite-difference
 * gradients, KB weights summing to one) -- "parity unpinned" against
 * reference-produced outputs.
 *
 * Array conventions (all follow the reference's Fortran column-major storage,
 * written here 0-based):
 *   pft  [K][P] complex   -> pfts_refs_even(P, kfrom:kto, :)      (simple_polarft_corrcalc.f90:319)
 *   polar[K][2N] float    -> polar(2*nrots, kfrom:kto)            (:258-267)
 *   argtransf[K][N] double-> argtransf(nrots, kfrom:kto)          (:308-317)
 *   ctfmat[K][P]          -> ctfmats(P, kfrom:kto, :)             (:924)
 *   cmat [box][box/2+1]   -> image%cmat(box/2+1, box, 1)          (simple_image.f90:1894-1907)
 * complex values are interleaved (re, im) pairs.
 */
#ifndef PFTCC_ORACLE_H
#define PFTCC_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int nrots;   /* N, number of in-plane rotations = 2*pftsz        */
    int pftsz;   /* P                                                 */
    int kfrom;   /* params_glob%kfromto(1)                            */
    int kto;     /* params_glob%kfromto(2)                            */
    int kstop;   /* params_glob%kstop (<= kto)                        */
    int box;     /* params_glob%boxmatch (even)                       */
} orc_geom;

typedef struct {
    float smpd, kv, cs, fraca;   /* A, kV, mm, amplitude contrast fraction       */
    float dfx, dfy, angast;      /* microns, microns, degrees                    */
    float phshift;               /* radians, used when l_phaseplate != 0         */
    int   l_phaseplate;
} orc_ctf;

/* polar / argtransf tables (simple_polarft_corrcalc.f90:261-317) */
void orc_tables(const orc_geom *g, float *polar, double *argtransf, double *argtransf_shellone);

/* |CTF| on the polar grid for one particle (create_polar_absctfmats :906-959) */
void orc_ctfmat(const orc_geom *g, const float *polar, const orc_ctf *c, double *ctfmat);

/* shift phase matrix, FP64 de Moivre recurrence (gen_shmat_8 :1098-1120); out [K][P] complex */
void orc_shmat(const orc_geom *g, const double *argtransf, const double *argtransf_shellone,
               double sx, double sy, double *shmat);

/* gencorrs, FP64 direct sums (gencorrs_cc_1 :1486-1500 when shvec == NULL,
 * gencorrs_cc_2 :1502-1534 otherwise).  ref/ptcl are FP32 pfts, ctfmat may be NULL. */
void orc_gencorrs(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                  const double *shvec, const double *argtransf, const double *argtransf_shellone,
                  double *cc);

/* gencorr_cc_for_rot_8 (:1690-1733), both branches selected by match_filt; irot is 1-based */
double orc_gencorr_for_rot(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                           const double *shvec, int irot, int match_filt,
                           const double *argtransf, const double *argtransf_shellone);

/* gencorr_cc_grad_for_rot_8 (:1863-1925), both branches; grad[2] = d/d(sx, sy) */
void orc_gencorr_grad_for_rot(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                              const double *shvec, int irot, int match_filt,
                              const double *argtransf, const double *argtransf_shellone,
                              double *f, double *grad);

/* particle-frame objective: the particle's |CTF| is applied at the particle's own polar
 * index (n + rot), with the rotation-dependent normaliser sum |ref|^2 CTF^2(n + rot).
 * Identical to gencorrs_cc_2 when the CTF is isotropic.  Sums run over kfrom..kstop. */
void orc_gencorrs_ptclframe(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                            const double *shvec, const double *argtransf, const double *argtransf_shellone,
                            double *cc);

/* f and d f / d(shift_x, shift_y, defocus) at one rotation, reference frame, both
 * branches of gencorr_cc_grad_for_rot_8 (:1863-1925).  The shift part equals the
 * reference's grad(1:2); the defocus part (no counterpart in the reference) uses
 * dctfmat = d|CTF|/d(defocus) on the grid in 1/micron (NULL -> grad3[2] = 0). */
void orc_gencorr_grad3(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                       const double *dctfmat, const double *shvec, int irot, int match_filt,
                       const double *argtransf, const double *argtransf_shellone,
                       double *f, double *grad3);

/* per-shell correlation coefficient at one rotation, k = kfrom..kstop into frc[Ks]:
 * genfrc (:1417-1441) when shvec == NULL, calc_frc (:1443-1484) otherwise --
 * kcorrs(irot) / sqrt(sum_n |ptcl(n,k)|^2 * sum_n |ref_prep(n,k)|^2), 0 when that
 * denominator is below 1e-12 (no shell normalisation or filter: l_pssnr and
 * l_match_filt off) */
void orc_genfrc(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat, const double *shvec,
                int irot, const double *argtransf, const double *argtransf_shellone, double *frc);
/* specscore_1/_2 (:2190-2205): max(0, median of the shell FRCs), median as
 * median_nocopy (simple_math.f90:2111-2130): the middle order statistic for an odd
 * count, the mean of the two middle ones for an even count */
double orc_specscore(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                     const double *shvec, int irot, const double *argtransf, const double *argtransf_shellone);

/* stochastic neighbourhood hill climbing for one particle (strategy2D_snhc srch_snhc,
 * simple_strategy2D_snhc.f90:33-93) over given per-rotation correlations
 * corrs[nrefs][nrots] (reference iref at row iref-1): references visited in order[]
 * (1-based), counting every visit against nrefs_bound (empty classes, pops[iref-1] == 0,
 * are skipped after being counted); for each, shcloc (simple_rnd.f90:273-295): a uniformly
 * random rotation among those with corr >= prev_corr -- the k-th such rotation in rotation
 * order, k = floor(u * count) with u = orc_snhc_uniform(seed, iptcl, isample) -- ending the
 * search (found_better = 1); otherwise the greedy best rotation, tracked as the global best
 * returned when no reference improves.  The comparison corr - prev_corr < 0 of the
 * reference's single precision is corr < prev_corr with prev_corr rounded to float.
 * out4 = {iref, irot (1-based), found_better, nrefs_eval}; the return value is the chosen
 * correlation. */
double orc_snhc_select(int nrots, int nrefs, const float *corrs, const int *order, const int *pops, int nrefs_bound,
                       double prev_corr, unsigned long long seed, int iptcl, int *out4);
/* the uniform deviate of draw isample for particle iptcl: splitmix64 of a Weyl sequence */
double orc_snhc_uniform(unsigned long long seed, int iptcl, int isample);

/* d|CTF|/d(mean defocus) in 1/micron, with dfx and dfy both moved by the same amount */
void orc_dctfmat_ddf(const orc_geom *g, const float *polar, const orc_ctf *c, double *dctfmat);

/* Kaiser-Bessel gridding (init_polarizer / polarize, simple_polarizer.f90:41-151) */
void orc_polarize(const orc_geom *g, const float *polar, const float *cmat, int griddev, double *pft);
double orc_kb_apod(double x);   /* simple_kbinterpol.f90:130-141 with Whalf=1.5, alpha=sqrt(2) */

/* polar projection of a volume FT (simple_projector.f90: expand_cmat :66-132,
 * fproject_polar :218-239, interp_fcomp :269-307; simple_ori.f90 euler2m :1275) */
void orc_euler2m(const double eul[3], double R[9]);
void orc_expand_cmat3d(int box, const float *cmat_half, double factor, float *cmat_exp);
void orc_fproject_polar(const orc_geom *g, const float *polar, int box, const float *cmat_exp,
                        const double eul[3], const int *mask, int griddev, double *pft);

/* the matched-filter mode (params_glob%l_match_filt): shellnorm_and_filter_ref(_8) (:756-807) scales
 * shell k <= kstop of the raw reference by optlp(k) / sqrt(pw), pw = sum_n |ref(n,k)|^2 / P, or by
 * optlp(k) where pw <= 1e-12; scale[Ks] (optlp = ref_optlp(:, iref), 1 unless set_ref_optlp) */
void orc_shellnorm_factors(const orc_geom *g, const float *ref, const float *optlp, double *scale);
/* the same, pssnr = 1 for the l_pssnr branch: sqrt(ssnr k) / sqrt(pw), ssnr = optlp(k) */
void orc_shellnorm_factors_mode(const orc_geom *g, const float *ref, const float *optlp, int pssnr, double *scale);
/* prep_matchfilt, the l_pssnr branch (:999-1019): the particle ptcl[K][P] rescaled in place */
void orc_prep_matchfilt_pssnr(const orc_geom *g, const double *ctfmat, const float *optlp, float *ptcl);
/* SavitzkyGolay_filter (simple_math.f90:3511-3588): 7-point quartic smoothing (nl = nr = 3, m = 4)
 * of y[n] in place, points left of the first omitted, the last 3 points unchanged */
void orc_savgol7(int n, double *y);
/* prep_matchfilt (:987-1095), the l_match_filt branch (l_pssnr off): the particle ptcl[K][P] is
 * rescaled per shell k <= kstop against reference ref (raw, its set chosen by the caller) times
 * ctfmat (NULL without CTF) at rotation irot (1-based), optlp the reference's ref_optlp column */
void orc_prep_matchfilt(const orc_geom *g, const float *ref, const double *ctfmat, const float *optlp, int irot,
                        float *ptcl);
/* particle ingestion: prepimg4align (simple_strategy2D3D_common.f90:316-366) for one particle
 * with the soft mask of radius msk (no inner or focus mask) and griddev 'no'; img [box][box]
 * real in C order [y][x] (rmat(x, y)); (x, y) the particle's shift; ctf NULL for ctfflag
 * no / flip, else the phase flip of ctfflag yes; out [boxmatch][boxmatch/2+1] complex, i.e.
 * cmat(h, k) with k at its physical index */
void orc_prepimg4align(int box, int boxmatch, const float *img, double msk, double x, double y, const orc_ctf *ctf,
                       double *cmat_out);
/* the same with the other mask modes of prepimg4align (:349-362): inner > 0 the inner cosine
 * edge of width width (<= 0: 10), else focusmsk > 0 the final mask's radius, griddev the
 * division by the gridding's instrument function */
void orc_prepimg4align_opts(int box, int boxmatch, const float *img, double msk, double inner, double width,
                            double focusmsk, int griddev, double x, double y, const orc_ctf *ctf, double *cmat_out);
/* orientation derivatives: euler2dm (simple_ori_light.f90:87-147), dR[j] = dR/de_j per radian,
 * three row-major 3x3 matrices; dapod (simple_kbinterpol.f90:179-192); fdf_project_polar
 * (simple_projector.f90:245-267 with fdf_interp_fcomp :338-400): pft [K][P] and its three
 * angle derivatives dpft [3][K][P], complex */
void orc_euler2dm(const double eul[3], double dR[27]);
double orc_kb_dapod(double x);
void orc_fdf_project_polar(const orc_geom *g, const float *polar, int box, const float *cmat_exp,
                           const double eul[3], double *pft, double *dpft);
/* gencorr_cont_shift_grad_cc_for_rot_8 (:1788-1847): f and grad[5] = d f / d(e1, e2, e3, sx, sy);
 * dref [3][K][P] complex FP32 as pfts_drefs holds it.  gencorr_cont_grad_cc_for_rot_8
 * (:1735-1786) is f and grad[0..2]. */
void orc_gencorr_cont_shift_grad(const orc_geom *g, const float *ref, const float *dref, const float *ptcl,
                                 const double *ctfmat, const double *shvec, int irot, const double *argtransf,
                                 const double *argtransf_shellone, double *f, double *grad5);
/* Euclidean objective (cc_objfun = OBJFUN_EUCLID).  sigma2[K] is the particle's column
 * sigma2_noise(kfrom:kto, iptcl); pxls[K] the pixel counts per shell of setup_pxls_p_shell
 * (:879-893); the reference is prepared in the reference frame as ref * ctf (* shmat). */
void orc_pxls_p_shell(int kfrom, int kto, double *pxls);
/* gencorrs_euclid_1 (:1536-1557, shvec == NULL) / gencorrs_euclid_2 (:1559-1592) */
void orc_gencorrs_euclid(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                         const double *shvec, const double *argtransf, const double *argtransf_shellone,
                         const double *sigma2, const double *pxls, double *euclids);
/* the Euclidean objective in the particle CTF frame (the m-domain search's frame): the CTF at the
 * particle's polar index, euclid(s) = -1/2 sum_{k<=kstop} w_k sum_n |A(n) ctf~(n+s) - ptcl~(n+s)|^2,
 * A = ref * shmat, w_k = pxls(k) / (P sigma2(k)); equal to gencorrs_euclid_2 for an isotropic CTF */
void orc_gencorrs_euclid_ptclframe(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                                   const double *shvec, const double *argtransf, const double *argtransf_shellone,
                                   const double *sigma2, const double *pxls, double *euclids);
/* gencorr_euclid_grad_for_rot_8 (:2071-2109): f = calc_euclid_for_rot_8 (:1308-1334),
 * grad[2] = d f / d(sx, sy); gencorr_euclid_for_rot_8 (:2026-2048) is f alone */
void orc_gencorr_euclid_grad_for_rot(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                                     const double *shvec, int irot, const double *argtransf,
                                     const double *argtransf_shellone, const double *sigma2, const double *pxls,
                                     double *f, double *grad);
/* gencorr_sigma_contrib (:2150-2188) over all shells kfrom..kto: sigma_contrib[K],
 * ptcl_sumsq[K], ref_sumsq[K] */
void orc_sigma_contrib(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                       const double *shvec, int irot, const double *argtransf, const double *argtransf_shellone,
                       double *sigma_contrib, double *ptcl_sumsq, double *ref_sumsq);
/* ---------------------------------------------------------------------------
 * FP32 FFT path, the reference's loop structure (memoize_fft :864-877 and
 * calc_corrs_over_k :1132-1162) on a project-written mixed-radix FFT that stands
 * in for FFTW.  Used as the timed CPU baseline. */
typedef struct orc_fftpath orc_fftpath;
orc_fftpath *orc_fftpath_new(const orc_geom *g);
void orc_fftpath_free(orc_fftpath *p);
/* memoised particle transforms: out buffer of K*(P/2+1)*2 + K*P*2 floats (see orc_fftpath_memo_size) */
long orc_fftpath_memo_size(const orc_geom *g);
void orc_fftpath_memoize(orc_fftpath *p, const float *ptcl, float *memo);
/* gencorrs_cc_2 through the FFT path: ref prepared with ctf (float, nullable) and shift */
void orc_fftpath_gencorrs(orc_fftpath *p, const float *ref, const float *ptcl_memo, float sqsum_ptcl,
                          const float *ctfmat, const float *shvec, const double *argtransf,
                          const double *argtransf_shellone, float *cc);

/* all correlations of one particle ptcl [K][P] (ctfmat [K][P] float, nullable) against
 * refs [nrefs][K][P] x shifts [nshifts][2] through the FP32 FFT path, OpenMP over the
 * (reference, shift) pairs: out [nrefs][nshifts][nrots].  Returns the threads used. */
int orc_fftpath_allcorrs(const orc_geom *g, int nrefs, const float *refs, const float *ptcl, const float *ctfmat,
                         int nshifts, const float *shifts, float *out, int nthreads);

/* exhaustive CPU search (greedy strategy over all refs x shift grid, OpenMP over particles).
 * refs [nrefs][K][P], ptcls [nptcls][K][P], ctfmats [nptcls][K][P] (float, nullable),
 * shifts [nshifts][2].  Output per particle: best ref (0-based), best irot (1-based),
 * best shift index, best cc.  Returns the number of OpenMP threads used. */
int orc_cpu_search(const orc_geom *g, int nrefs, const float *refs, int nptcls, const float *ptcls,
                   const float *ctfmats, int nshifts, const float *shifts,
                   int *best_ref, int *best_rot, int *best_shift, float *best_cc, int nthreads);

/* complex FFT helpers exposed for tests: forward (sign=-1) or backward (+1), unnormalised */
void orc_cfft(int n, const double *in, double *out, int sign);

#ifdef __cplusplus
}
#endif
#endif
