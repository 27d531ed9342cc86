/*
 * pftcc_oracle.c -- CPU restatement of SIMPLE 3.0's polar Fourier correlation
 * search, TEST INFRASTRUCTURE ONLY (the checker for tests/, smoke() and the
 * cpu_baseline / reference arm of bench.py).  See pftcc_oracle.h for the array
 * conventions and the parity status.  Every function cites the reference
 * routine it restates (paths relative to the SIMPLE 3.0 source tree).
 */
#include "pftcc_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define K_OF(g) ((g)->kto - (g)->kfrom + 1)

/* ------------------------------------------------------------------------- */
/* tables: simple_polarft_corrcalc.f90:261-274 (polar, in single precision
 * exactly as the reference: ang = TWOPI/real(nrots), angtab = real(irot-1)*ang,
 * x = sin(angtab)*real(k), y = -cos(angtab)*real(k)) and :311-317 (argtransf in
 * double: real(polar,dp) * DPI/real(box/2,dp)). */
void orc_tables(const orc_geom *g, float *polar, double *argtransf, double *argtransf_shellone)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g);
    const float twopi = 2.0f * acosf(-1.0f);
    const float ang = twopi / (float)N;
    const double A = acos(-1.0) / (double)(g->box / 2);
    for (int ik = 0; ik < K; ++ik) {
        const int k = g->kfrom + ik;
        for (int irot = 0; irot < N; ++irot) {
            const float a = (float)irot * ang;
            polar[ik * 2 * N + irot]     =  sinf(a) * (float)k;
            polar[ik * 2 * N + N + irot] = -cosf(a) * (float)k;
        }
        for (int irot = 0; irot < P; ++irot) {
            argtransf[ik * N + irot]     = (double)polar[ik * 2 * N + irot] * A;       /* x-part */
            argtransf[ik * N + P + irot] = (double)polar[ik * 2 * N + N + irot] * A;   /* y-part */
        }
    }
    for (int irot = 0; irot < P; ++irot) {
        const float a = (float)irot * ang;
        argtransf_shellone[irot]     = (double)sinf(a) * A;
        argtransf_shellone[P + irot] = (double)(-cosf(a)) * A;
    }
}

/* ------------------------------------------------------------------------- */
/* CTF: simple_ctf.f90 constructor :54-70 (wl = kV2wl/smpd, Cs*1e7/smpd,
 * amp_contr_const = atan(fraca/sqrt(1-fraca^2))), init :73-81 (defocus in
 * pixels, angast in radians), evalPhSh :88-98, eval_df :185-189, kV2wl :522-525;
 * polar sampling from create_polar_absctfmats :926-935, |CTF| at :952-954. */
typedef struct { double wl, cs, ampc, dfx, dfy, angast, phshift, dfscale; } ctf_consts;

static ctf_consts ctf_setup(const orc_ctf *c)
{
    ctf_consts k;
    const double kv = c->kv * 1000.0;
    const double wl_A = 12.26 / sqrt(kv + 0.9784 * kv * kv / 1.0e6);
    k.wl = wl_A / c->smpd;
    k.cs = (c->cs * 1.0e7) / c->smpd;
    k.ampc = atan(c->fraca / sqrt(1.0 - (double)c->fraca * c->fraca));
    k.dfscale = 1.0e4 / c->smpd;
    k.dfx = c->dfx * k.dfscale;
    k.dfy = c->dfy * k.dfscale;
    k.angast = c->angast / 180.0 * acos(-1.0);
    k.phshift = c->l_phaseplate ? c->phshift : 0.0;
    return k;
}

static void polar_freq(const orc_geom *g, const float *polar, int ik, int irot, double *spafreqsq, double *ang)
{
    const int N = g->nrots;
    const double x = polar[ik * 2 * N + irot], y = polar[ik * 2 * N + N + irot];
    const double hinv = x / g->box, kinv = y / g->box;
    *spafreqsq = hinv * hinv + kinv * kinv;
    *ang = atan2(y, x);
}

static double ctf_chi(const ctf_consts *k, double s2, double ang)
{
    const double df = 0.5 * (k->dfx + k->dfy + cos(2.0 * (ang - k->angast)) * (k->dfx - k->dfy));
    return acos(-1.0) * k->wl * s2 * (df - 0.5 * k->wl * k->wl * s2 * k->cs) + k->phshift + k->ampc;
}

void orc_ctfmat(const orc_geom *g, const float *polar, const orc_ctf *c, double *ctfmat)
{
    const int P = g->pftsz, K = K_OF(g);
    const ctf_consts k = ctf_setup(c);
    for (int ik = 0; ik < K; ++ik)
        for (int irot = 0; irot < P; ++irot) {
            double s2, ang;
            polar_freq(g, polar, ik, irot, &s2, &ang);
            ctfmat[ik * P + irot] = fabs(sin(ctf_chi(&k, s2, ang)));
        }
}

void orc_dctfmat_ddf(const orc_geom *g, const float *polar, const orc_ctf *c, double *dctfmat)
{
    const int P = g->pftsz, K = K_OF(g);
    const ctf_consts k = ctf_setup(c);
    for (int ik = 0; ik < K; ++ik)
        for (int irot = 0; irot < P; ++irot) {
            double s2, ang;
            polar_freq(g, polar, ik, irot, &s2, &ang);
            const double chi = ctf_chi(&k, s2, ang);
            const double dchi = acos(-1.0) * k.wl * s2 * k.dfscale;  /* d chi / d df[micron] */
            const double s = sin(chi);
            dctfmat[ik * P + irot] = (s >= 0.0 ? 1.0 : -1.0) * cos(chi) * dchi;
        }
}

/* ------------------------------------------------------------------------- */
/* gen_shmat_8, simple_polarft_corrcalc.f90:1098-1120: first shell analytic,
 * later shells by the de Moivre recurrence with the shell-one phase vector. */
void orc_shmat(const orc_geom *g, const double *argtransf, const double *argtransf_shellone,
               double sx, double sy, double *shmat)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g);
    for (int n = 0; n < P; ++n) {
        const double a = argtransf[n] * sx + argtransf[P + n] * sy;
        shmat[2 * n] = cos(a);
        shmat[2 * n + 1] = sin(a);
    }
    for (int n = 0; n < P; ++n) {
        const double a1 = argtransf_shellone[n] * sx + argtransf_shellone[P + n] * sy;
        const double vr = cos(a1), vi = sin(a1);
        for (int ik = 1; ik < K; ++ik) {
            const double pr = shmat[2 * ((ik - 1) * P + n)], pi = shmat[2 * ((ik - 1) * P + n) + 1];
            shmat[2 * (ik * P + n)]     = pr * vr - pi * vi;
            shmat[2 * (ik * P + n) + 1] = pr * vi + pi * vr;
        }
    }
    (void)N;
}

/* prepared reference: pft_ref = ref * ctf * shmat in double (prep_ref4corr :961-985
 * and gencorrs_cc_2 :1516-1530) */
static void prep_ref(const orc_geom *g, const float *ref, const double *ctfmat, const double *shvec,
                     const double *argtransf, const double *argtransf_shellone, double *out)
{
    const int P = g->pftsz, K = K_OF(g);
    double *sh = NULL;
    if (shvec) {
        sh = (double *)malloc(sizeof(double) * 2 * K * P);
        orc_shmat(g, argtransf, argtransf_shellone, shvec[0], shvec[1], sh);
    }
    for (int i = 0; i < K * P; ++i) {
        double re = ref[2 * i], im = ref[2 * i + 1];
        if (ctfmat) { re *= ctfmat[i]; im *= ctfmat[i]; }
        if (sh) {
            const double sr = sh[2 * i], si = sh[2 * i + 1];
            const double tr = re * sr - im * si, ti = re * si + im * sr;
            re = tr; im = ti;
        }
        out[2 * i] = re; out[2 * i + 1] = im;
    }
    free(sh);
}

/* calc_corrk_for_rot_8 (:1364-1390): Re sum_n ref(n) * conj(ptcl~(n + irot - 1)),
 * where ptcl~ is the particle extended over the full circle by ptcl~(j + P) =
 * conj(ptcl(j)).  The reference's four-way case split on irot is exactly this
 * cyclic index with the conjugation rule. */
static double corrk_for_rot(int P, const double *ref_k, const float *ptcl_k, int irot)
{
    const int N = 2 * P, s = irot - 1;
    double acc = 0.0;
    for (int n = 0; n < P; ++n) {
        int j = (n + s) % N;
        double qr, qi;
        if (j < P) { qr = ptcl_k[2 * j]; qi = ptcl_k[2 * j + 1]; }
        else { qr = ptcl_k[2 * (j - P)]; qi = -ptcl_k[2 * (j - P) + 1]; }
        /* Re(a * conj(q)) = ar*qr + ai*qi */
        acc += ref_k[2 * n] * qr + ref_k[2 * n + 1] * qi;
    }
    return acc;
}

static double sqsum_k(int P, const double *x)
{
    double s = 0.0;
    for (int n = 0; n < P; ++n) s += x[2 * n] * x[2 * n] + x[2 * n + 1] * x[2 * n + 1];
    return s;
}

static double sqsum_kf(int P, const float *x)
{
    double s = 0.0;
    for (int n = 0; n < P; ++n) s += (double)x[2 * n] * x[2 * n] + (double)x[2 * n + 1] * x[2 * n + 1];
    return s;
}

/* gencorrs_cc_1 (:1486-1500) / gencorrs_cc_2 (:1502-1534).  Note the reference's
 * asymmetry: cc_1 takes sqsum_ref over kfrom..kstop (prep_ref4corr :984) while
 * cc_2 takes it over all shells kfrom..kto (:1531).  The correlation always runs
 * over kfrom..kstop (:1498, :1532), as does sqsums_ptcls (memoize_sqsum_ptcl :844). */
void orc_gencorrs(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                  const double *shvec, const double *argtransf, const double *argtransf_shellone,
                  double *cc)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    prep_ref(g, ref, ctfmat, shvec, argtransf, argtransf_shellone, pr);
    double sqr = 0.0, sqp = 0.0;
    const int ksq = shvec ? K : Ks;
    for (int ik = 0; ik < ksq; ++ik) sqr += sqsum_k(P, pr + 2 * ik * P);
    for (int ik = 0; ik < Ks; ++ik) sqp += sqsum_kf(P, ptcl + 2 * ik * P);
    const double den = sqrt(sqr * sqp);
    for (int irot = 1; irot <= N; ++irot) {
        double c = 0.0;
        for (int ik = 0; ik < Ks; ++ik) c += corrk_for_rot(P, pr + 2 * ik * P, ptcl + 2 * ik * P, irot);
        cc[irot - 1] = c / den;
    }
    free(pr);
}

void orc_genfrc(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat, const double *shvec,
                int irot, const double *argtransf, const double *argtransf_shellone, double *frc)
{
    const int P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    prep_ref(g, ref, ctfmat, shvec, argtransf, argtransf_shellone, pr);
    for (int ik = 0; ik < Ks; ++ik) {
        const double den = sqrt(sqsum_kf(P, ptcl + 2 * ik * P) * sqsum_k(P, pr + 2 * ik * P));
        frc[ik] = den < 1e-12 ? 0.0 : corrk_for_rot(P, pr + 2 * ik * P, ptcl + 2 * ik * P, irot) / den;
    }
    free(pr);
}

static int cmp_double(const void *a, const void *b)
{
    const double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

double orc_specscore(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                     const double *shvec, int irot, const double *argtransf, const double *argtransf_shellone)
{
    const int Ks = g->kstop - g->kfrom + 1;
    double *frc = (double *)malloc(sizeof(double) * Ks);
    orc_genfrc(g, ref, ptcl, ctfmat, shvec, irot, argtransf, argtransf_shellone, frc);
    qsort(frc, Ks, sizeof(double), cmp_double);
    const double med = (Ks % 2) ? frc[Ks / 2] : 0.5 * (frc[Ks / 2 - 1] + frc[Ks / 2]);
    free(frc);
    return med > 0.0 ? med : 0.0;
}

double orc_snhc_uniform(unsigned long long seed, int iptcl, int isample)
{
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(unsigned)iptcl +
                           0xD1B54A32D192ED03ULL * (unsigned long long)(unsigned)isample;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

double orc_snhc_select(int nrots, int nrefs, const float *corrs, const int *order, const int *pops, int nrefs_bound,
                       double prev_corr, unsigned long long seed, int iptcl, int *out4)
{
    const float pf = (float)prev_corr;
    double cc_glob = -HUGE_VAL;
    int class_glob = 0, inpl_glob = 0, neval = 0, found = 0, best_ref = 0, best_rot = 0;
    double best_corr = 0.0;
    for (int isample = 1; isample <= nrefs; ++isample) {
        const int iref = order[isample - 1];
        ++neval;
        if (neval > nrefs_bound) break;
        if (pops && pops[iref - 1] == 0) continue;
        const float *c = corrs + (size_t)(iref - 1) * nrots;
        /* shcloc: the rotations whose difference to the previous best is not negative */
        int navail = 0;
        for (int r = 0; r < nrots; ++r) navail += !(c[r] < pf);
        int inpl;
        double inpl_corr;
        if (navail == 0) {
            inpl = 0;   /* maxloc: the first maximum */
            for (int r = 1; r < nrots; ++r)
                if (c[r] > c[inpl]) inpl = r;
            inpl_corr = c[inpl];
        } else {
            int k = (int)(orc_snhc_uniform(seed, iptcl, isample) * navail);
            if (k >= navail) k = navail - 1;
            inpl = -1;
            for (int r = 0; r < nrots; ++r)
                if (!(c[r] < pf) && k-- == 0) { inpl = r; break; }
            inpl_corr = c[inpl];
            best_ref = iref; best_rot = inpl + 1; best_corr = inpl_corr;
            found = 1;
        }
        if (inpl_corr > cc_glob) { cc_glob = inpl_corr; class_glob = iref; inpl_glob = inpl + 1; }
        if (found) break;
    }
    if (!found) { best_ref = class_glob; best_rot = inpl_glob; best_corr = class_glob ? cc_glob : 0.0; }
    out4[0] = best_ref; out4[1] = best_rot; out4[2] = found; out4[3] = neval;
    return best_corr;
}

/* gencorr_cc_for_rot_8 (:1690-1733).  match_filt: unweighted sums normalised by
 * sqsum over kfrom..kstop (:1729-1731).  Otherwise the shell-weighted ("jacobian")
 * form sum_k k*corr_k / sqrt(sum_k k|ref_k|^2 * sum_k k|ptcl_k|^2) (:1717-1727). */
double orc_gencorr_for_rot(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                           const double *shvec, int irot, int match_filt,
                           const double *argtransf, const double *argtransf_shellone)
{
    const int P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    const double zero[2] = {0.0, 0.0};
    prep_ref(g, ref, ctfmat, shvec ? shvec : zero, argtransf, argtransf_shellone, pr);
    double corr = 0.0, sqr = 0.0, sqp = 0.0;
    for (int ik = 0; ik < Ks; ++ik) {
        const double w = match_filt ? 1.0 : (double)(g->kfrom + ik);
        sqr += w * sqsum_k(P, pr + 2 * ik * P);
        sqp += w * sqsum_kf(P, ptcl + 2 * ik * P);
        corr += w * corrk_for_rot(P, pr + 2 * ik * P, ptcl + 2 * ik * P, irot);
    }
    free(pr);
    return corr / sqrt(sqr * sqp);
}

/* gencorr_cc_grad_for_rot_8 (:1863-1925) extended with a defocus derivative.
 * d/dsx multiplies the shifted reference by i*argtransf_x (:1896, :1914), d/dsy by
 * i*argtransf_y (:1899, :1918); the denominator is shift invariant.  For the
 * defocus, d pft_ref = ref * dctf * shmat and the quotient rule adds
 * -f/2 * d(sqsum_ref)/sqsum_ref. */
void orc_gencorr_grad3(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                       const double *dctfmat, const double *shvec, int irot, int match_filt,
                       const double *argtransf, const double *argtransf_shellone,
                       double *f, double *grad3)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    double *tmp = (double *)malloc(sizeof(double) * 2 * K * P);
    double *dr = (double *)malloc(sizeof(double) * 2 * K * P);
    const double zero[2] = {0.0, 0.0};
    const double *sv = shvec ? shvec : zero;
    prep_ref(g, ref, ctfmat, sv, argtransf, argtransf_shellone, pr);
    double corr = 0.0, sqr = 0.0, sqp = 0.0, gx = 0.0, gy = 0.0, gdn = 0.0, dsq = 0.0;
    if (dctfmat) prep_ref(g, ref, dctfmat, sv, argtransf, argtransf_shellone, dr);
    for (int ik = 0; ik < Ks; ++ik) {
        const double w = match_filt ? 1.0 : (double)(g->kfrom + ik);
        const double *prk = pr + 2 * ik * P;
        sqr += w * sqsum_k(P, prk);
        sqp += w * sqsum_kf(P, ptcl + 2 * ik * P);
        corr += w * corrk_for_rot(P, prk, ptcl + 2 * ik * P, irot);
        for (int d = 0; d < 2; ++d) {
            double *tk = tmp + 2 * ik * P;
            for (int n = 0; n < P; ++n) {
                const double a = argtransf[ik * N + d * P + n];
                /* (re + i im) * i * a = -im*a + i re*a */
                tk[2 * n] = -prk[2 * n + 1] * a;
                tk[2 * n + 1] = prk[2 * n] * a;
            }
            const double c = w * corrk_for_rot(P, tk, ptcl + 2 * ik * P, irot);
            if (d == 0) gx += c; else gy += c;
        }
        if (dctfmat) {
            const double *drk = dr + 2 * ik * P;
            gdn += w * corrk_for_rot(P, drk, ptcl + 2 * ik * P, irot);
            for (int n = 0; n < P; ++n) dsq += w * 2.0 * (prk[2 * n] * drk[2 * n] + prk[2 * n + 1] * drk[2 * n + 1]);
        }
    }
    const double den = sqrt(sqr * sqp);
    *f = corr / den;
    grad3[0] = gx / den;
    grad3[1] = gy / den;
    grad3[2] = dctfmat ? (gdn / den - 0.5 * (*f) * dsq / sqr) : 0.0;
    free(pr); free(tmp); free(dr);
}

void orc_gencorr_grad_for_rot(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                              const double *shvec, int irot, int match_filt,
                              const double *argtransf, const double *argtransf_shellone,
                              double *f, double *grad)
{
    double g3[3];
    orc_gencorr_grad3(g, ref, ptcl, ctfmat, NULL, shvec, irot, match_filt, argtransf, argtransf_shellone, f, g3);
    grad[0] = g3[0];
    grad[1] = g3[1];
}

/* particle-frame objective (see header): numerator Re sum_n (ref*shmat)(n) *
 * conj(ctf~(n+s) * ptcl~(n+s)) with ctf~(j) = ctf(j mod P), normaliser
 * sum_n |ref(n)|^2 ctf~(n+s)^2 (shift invariant since |shmat| = 1). */
void orc_gencorrs_ptclframe(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                            const double *shvec, const double *argtransf, const double *argtransf_shellone,
                            double *cc)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    prep_ref(g, ref, NULL, shvec, argtransf, argtransf_shellone, pr);
    double sqp = 0.0;
    for (int ik = 0; ik < Ks; ++ik) sqp += sqsum_kf(P, ptcl + 2 * ik * P);
    for (int s = 0; s < N; ++s) {
        double num = 0.0, den = 0.0;
        for (int ik = 0; ik < Ks; ++ik) {
            const double *a = pr + 2 * ik * P;
            const float *q = ptcl + 2 * ik * P;
            for (int n = 0; n < P; ++n) {
                const int j = (n + s) % N;
                const int jp = j % P;
                double qr = q[2 * jp], qi = q[2 * jp + 1];
                if (j >= P) qi = -qi;
                const double c = ctfmat ? ctfmat[ik * P + jp] : 1.0;
                num += c * (a[2 * n] * qr + a[2 * n + 1] * qi);
                const double r2 = (double)ref[2 * (ik * P + n)] * ref[2 * (ik * P + n)]
                                + (double)ref[2 * (ik * P + n) + 1] * ref[2 * (ik * P + n) + 1];
                den += r2 * c * c;
            }
        }
        cc[s] = num / sqrt(den * sqp);
    }
    free(pr);
}

/* ------------------------------------------------------------------------- */
/* Kaiser-Bessel window, simple_kbinterpol.f90: new :92-109 with Whalf = KBWINSZ
 * = 1.5 (simple_defs.f90:131) -> W = 3, beta = 7.4 (the Whalf <= 1.5 branch),
 * apod :130-141, bessi0 :229-252 (Abramowitz & Stegun 9.8.1 / 9.8.2 polynomial
 * approximations of I0). */
static double bessi0(double x)
{
    const double ax = x;
    if (ax < 3.75) {
        double y = x / 3.75;
        y = y * y;
        return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 + y * (0.0360768 + y * 0.0045813)))));
    }
    const double y = 3.75 / ax;
    return (0.39894228 + y * (0.01328592 + y * (0.00225319 + y * (-0.00157565 + y * (0.00916281 +
            y * (-0.02057706 + y * (0.02635537 + y * (-0.01647633 + y * 0.00392377)))))))) * exp(ax) / sqrt(ax);
}

double orc_kb_apod(double x)
{
    const double whalf = 1.5, W = 3.0, beta = 7.4;
    if (fabs(x) > whalf) return 0.0;
    double arg = (2.0 / W) * x;
    arg = 1.0 - arg * arg;
    if (arg < 0.0) arg = 0.0;
    return (1.0 / W) * bessi0(beta * sqrt(arg));
}

/* Fortran nint: round half away from zero */
static int f_nint(double x) { return (int)(x >= 0.0 ? floor(x + 0.5) : -floor(-x + 0.5)); }

/* cyci_1d, simple_math.f90:746-757 */
static int cyci_1d(int lo, int hi, int i)
{
    if (i > hi) return lo + (i - hi) - 1;
    if (i < lo) return hi - (lo - i) + 1;
    return i;
}

/* get_fcomp2D, simple_image.f90:1894-1907: Hermitian half-plane gather */
static void get_fcomp2d(const float *cmat, int box, int h, int k, double *re, double *im)
{
    const int ld = box / 2 + 1;
    int p1, p2;
    double sgn = 1.0;
    if (h >= 0) { p1 = h; p2 = k + (k < 0 ? box : 0); }
    else { p1 = -h; p2 = -k + (-k < 0 ? box : 0); sgn = -1.0; }
    *re = cmat[2 * (p2 * ld + p1)];
    *im = sgn * cmat[2 * (p2 * ld + p1) + 1];
}

/* init_polarizer :41-92 (3x3 window sqwin_2d around nint(loc), weights the outer
 * product of apod(win - loc), normalised by their sum unless griddev, cyclic
 * addresses over the logical limits [-box/2, box/2] x [-box/2, box/2-1]) and
 * polarize :120-151 (pft(i,k) = sum w * F(h,k)); rotations 1..P only. */
void orc_polarize(const orc_geom *g, const float *polar, const float *cmat, int griddev, double *pft)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), box = g->box;
    for (int ik = 0; ik < K; ++ik)
        for (int i = 0; i < P; ++i) {
            const double lx = polar[ik * 2 * N + i], ly = polar[ik * 2 * N + N + i];
            const int wx = f_nint(lx) - 1, wy = f_nint(ly) - 1;
            double w[3][3], wsum = 0.0;
            for (int l = 0; l < 3; ++l)
                for (int m = 0; m < 3; ++m) {
                    w[l][m] = orc_kb_apod((double)(wx + l) - lx) * orc_kb_apod((double)(wy + m) - ly);
                    wsum += w[l][m];
                }
            double accr = 0.0, acci = 0.0;
            for (int l = 0; l < 3; ++l) {
                const int h = cyci_1d(-box / 2, box / 2, wx + l);
                for (int m = 0; m < 3; ++m) {
                    const int kk = cyci_1d(-box / 2, box / 2 - 1, wy + m);
                    double re, im;
                    get_fcomp2d(cmat, box, h, kk, &re, &im);
                    const double ww = griddev ? w[l][m] : w[l][m] / wsum;
                    accr += ww * re;
                    acci += ww * im;
                }
            }
            pft[2 * (ik * P + i)] = accr;
            pft[2 * (ik * P + i) + 1] = acci;
        }
}

/* ------------------------------------------------------------------------- */
/* Polar projection of a volume's Fourier transform (the references of refine3D). */

/* rotmat :1350-1390 (angle in degrees; the z rotation is the negative one) and
 * euler2m :1275-1284 of simple_ori.f90: R = R3(e3) R2(e2) R1(e1), z-y-z (Spider).
 * R row-major, R[3 i + j] = r(i+1, j+1). */
static void rotmat3(double ang_deg, int choice, double r[9])
{
    const double a = ang_deg * 3.14159265358979323846 / 180.0, c = cos(a), s = sin(a);
    for (int i = 0; i < 9; ++i) r[i] = 0.0;
    if (choice == 1) { r[0] = 1.0; r[4] = c; r[5] = -s; r[7] = s; r[8] = c; }
    else if (choice == 2) { r[0] = c; r[2] = -s; r[4] = 1.0; r[6] = s; r[8] = c; }
    else { r[0] = c; r[1] = s; r[3] = -s; r[4] = c; r[8] = 1.0; }
}

static void matmul3(const double a[9], const double b[9], double c[9])
{
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double t = 0.0;
            for (int l = 0; l < 3; ++l) t += a[3 * i + l] * b[3 * l + j];
            c[3 * i + j] = t;
        }
}

void orc_euler2m(const double eul[3], double R[9])
{
    double r1[9], r2[9], r3[9], t[9];
    rotmat3(eul[0], 3, r1);
    rotmat3(eul[1], 2, r2);
    rotmat3(eul[2], 3, r3);
    matmul3(r3, r2, t);
    matmul3(t, r1, R);
}

/* comp_addr_phys / get_fcomp (simple_ftiter.f90:241-265, simple_image.f90) for a
 * volume: the half volume image%cmat(h, k, m), h = 0..B/2, stored here as
 * [m][k][h] complex; negative h read as the conjugate of (-h, -k, -m) */
static void get_fcomp3d(const float *cmat, int box, int h, int k, int m, double *re, double *im)
{
    const int ld = box / 2 + 1;
    double sgn = 1.0;
    if (h < 0) { h = -h; k = -k; m = -m; sgn = -1.0; }
    const int p2 = k + (k < 0 ? box : 0), p3 = m + (m < 0 ? box : 0);
    const size_t e = ((size_t)p3 * box + p2) * ld + h;
    *re = cmat[2 * e];
    *im = sgn * cmat[2 * e + 1];
}

/* expand_cmat (simple_projector.f90:66-132) of a volume of even box B: the cube
 * cmat_exp(h, k, m), h, k, m in [-E, E] with E = B/2 + 2 (maxval(|lims|) + ceiling(KBWINSZ)),
 * each logical address wrapped cyclically into the mode-3 limits [-B/2, B/2] x
 * [-B/2, B/2 - 1] x [-B/2, B/2 - 1] (cyci_1d) and read with Friedel symmetry, times
 * factor. Output [m][k][h] complex, side S = 2E + 1. */
void orc_expand_cmat3d(int box, const float *cmat_half, double factor, float *cmat_exp)
{
    const int E = box / 2 + 2, S = 2 * E + 1;
    for (int m = -E; m <= E; ++m)
        for (int k = -E; k <= E; ++k)
            for (int h = -E; h <= E; ++h) {
                const int hh = cyci_1d(-box / 2, box / 2, h);
                const int kk = cyci_1d(-box / 2, box / 2 - 1, k);
                const int mm = cyci_1d(-box / 2, box / 2 - 1, m);
                double re, im;
                get_fcomp3d(cmat_half, box, hh, kk, mm, &re, &im);
                const size_t e = ((size_t)(m + E) * S + (k + E)) * S + (h + E);
                cmat_exp[2 * e] = (float)(factor * re);
                cmat_exp[2 * e + 1] = (float)(factor * im);
            }
}

/* fproject_polar (simple_projector.f90:218-239) with interp_fcomp_norm / _grid
 * (:269-307): for rotations irot < P and shells kfrom..kto, loc = vec R with
 * vec = (polar(irot, k), polar(irot + nrots, k), 0) (get_coord), the 3x3x3 window
 * around nint(loc), weights the product of apod(win - loc) per axis, normalised by
 * their sum unless griddev; shells with mask[k - kfrom] == 0 are zero. */
void orc_fproject_polar(const orc_geom *g, const float *polar, int box, const float *cmat_exp,
                        const double eul[3], const int *mask, int griddev, double *pft)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g);
    const int E = box / 2 + 2, S = 2 * E + 1;
    double R[9];
    orc_euler2m(eul, R);
    for (int ik = 0; ik < K; ++ik)
        for (int i = 0; i < P; ++i) {
            double accr = 0.0, acci = 0.0;
            if (!mask || mask[ik]) {
                const double vx = polar[ik * 2 * N + i], vy = polar[ik * 2 * N + N + i];
                double loc[3];
                for (int j = 0; j < 3; ++j) loc[j] = vx * R[j] + vy * R[3 + j];
                int w0[3];
                double wa[3][3];
                for (int d = 0; d < 3; ++d) {
                    w0[d] = f_nint(loc[d]) - 1;
                    for (int l = 0; l < 3; ++l) wa[d][l] = orc_kb_apod((double)(w0[d] + l) - loc[d]);
                }
                double wsum = 0.0;
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b)
                        for (int c = 0; c < 3; ++c) {
                            const double w = wa[0][a] * wa[1][b] * wa[2][c];
                            const size_t e = ((size_t)(w0[2] + c + E) * S + (w0[1] + b + E)) * S + (w0[0] + a + E);
                            accr += w * cmat_exp[2 * e];
                            acci += w * cmat_exp[2 * e + 1];
                            wsum += w;
                        }
                if (!griddev) { accr /= wsum; acci /= wsum; }
            }
            pft[2 * (ik * P + i)] = accr;
            pft[2 * (ik * P + i) + 1] = acci;
        }
}

/* ------------------------------------------------------------------------- */
/* Project-written mixed-radix FFT (recursive decimation in time, radices 4, 2,
 * 3, 5 and a plain DFT for any other prime factor).  Stands in for FFTW. */
typedef struct { int n; int nf; int f[32]; double *tw; float *twf; } fftplan;

static void fftplan_init(fftplan *p, int n)
{
    p->n = n; p->nf = 0;
    int m = n;
    const int rad[4] = {4, 2, 3, 5};
    for (int r = 0; r < 4; ++r) while (m % rad[r] == 0) { p->f[p->nf++] = rad[r]; m /= rad[r]; }
    for (int q = 7; m > 1; q += 2) while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
    p->tw = (double *)malloc(sizeof(double) * 2 * n);
    p->twf = (float *)malloc(sizeof(float) * 2 * n);
    for (int j = 0; j < n; ++j) {
        const double a = -2.0 * acos(-1.0) * j / n;
        p->tw[2 * j] = cos(a); p->tw[2 * j + 1] = sin(a);
        p->twf[2 * j] = (float)cos(a); p->twf[2 * j + 1] = (float)sin(a);
    }
}

static void fftplan_free(fftplan *p) { free(p->tw); free(p->twf); }

#define DEFINE_FFT(NAME, T, TW)                                                                   \
static void NAME(const fftplan *p, int lvl, int n, const T *in, int stride, T *out, int sign)     \
{                                                                                                  \
    if (n == 1) { out[0] = in[0]; out[1] = in[1]; return; }                                        \
    const int r = p->f[lvl], m = n / r, step = p->n / n;                                          \
    for (int q = 0; q < r; ++q) NAME(p, lvl + 1, m, in + 2 * q * stride, stride * r, out + 2 * q * m, sign); \
    T tr[64], ti[64];                                                                              \
    for (int k = 0; k < m; ++k) {                                                                  \
        for (int q = 0; q < r; ++q) {                                                              \
            const int ti_ = (q * k * step) % p->n;                                                 \
            const T wr = p->TW[2 * ti_], wi = -sign * p->TW[2 * ti_ + 1];                          \
            const T xr = out[2 * (q * m + k)], xi = out[2 * (q * m + k) + 1];                      \
            tr[q] = xr * wr - xi * wi; ti[q] = xr * wi + xi * wr;                                 \
        }                                                                                          \
        for (int s = 0; s < r; ++s) {                                                              \
            T ar = 0, ai = 0;                                                                      \
            for (int q = 0; q < r; ++q) {                                                          \
                const int e = ((q * s) % r) * (p->n / r);                                          \
                const T wr = p->TW[2 * e], wi = -sign * p->TW[2 * e + 1];                          \
                ar += tr[q] * wr - ti[q] * wi; ai += tr[q] * wi + ti[q] * wr;                     \
            }                                                                                      \
            out[2 * (s * m + k)] = ar; out[2 * (s * m + k) + 1] = ai;                              \
        }                                                                                          \
    }                                                                                              \
}
/* the combine above writes in place over the sub-transforms it has already read
 * for the same k only (all r inputs of column k are consumed before any output of
 * column k is written, and columns do not overlap), so no scratch is needed. */
DEFINE_FFT(fft_rec_d, double, tw)
DEFINE_FFT(fft_rec_f, float, twf)

void orc_cfft(int n, const double *in, double *out, int sign)
{
    fftplan p;
    fftplan_init(&p, n);
    fft_rec_d(&p, 0, n, in, 1, out, sign);
    fftplan_free(&p);
}

/* ------------------------------------------------------------------------- */
/* FP32 FFT path: memoize_fft (:864-877) and calc_corrs_over_k (:1132-1162).
 * r2c(P) of Re(x) keeps P/2+1 outputs; c2c(P) of Im(x)*fft_factors with
 * fft_factors(n) = exp(-i*pi*n/P) (:410-413); the product spectrum interleaves
 * 4*conj(ref_re)*ptcl_re at the odd 1-based slots and 4*conj(ref_im)*ptcl_im at
 * the even ones, then a c2r(N) per shell, accumulated and divided by 2N. */
struct orc_fftpath {
    orc_geom g;
    fftplan pP, pN;
    float *ff;               /* fft_factors, P complex                  */
};

orc_fftpath *orc_fftpath_new(const orc_geom *g)
{
    orc_fftpath *p = (orc_fftpath *)calloc(1, sizeof(orc_fftpath));
    p->g = *g;
    fftplan_init(&p->pP, g->pftsz);
    fftplan_init(&p->pN, g->nrots);
    p->ff = (float *)malloc(sizeof(float) * 2 * g->pftsz);
    const float pif = acosf(-1.0f);
    for (int n = 0; n < g->pftsz; ++n) {
        const float a = -pif * (float)n / (float)g->pftsz;
        p->ff[2 * n] = cosf(a); p->ff[2 * n + 1] = sinf(a);
    }
    return p;
}

void orc_fftpath_free(orc_fftpath *p)
{
    if (!p) return;
    fftplan_free(&p->pP); fftplan_free(&p->pN); free(p->ff); free(p);
}

long orc_fftpath_memo_size(const orc_geom *g)
{
    return (long)K_OF(g) * 2 * 2 * g->pftsz;   /* per shell: re-transform (P cplx slots) + im-transform (P cplx) */
}

/* transforms of one shell: xr_out = fft_P(Re x) (first P/2+1 valid), xi_out = fft_P(Im x * ff) */
static void shell_transforms(const orc_fftpath *p, const float *x, float *work, float *xr_out, float *xi_out)
{
    const int P = p->g.pftsz;
    float *a = work, *b = work + 2 * P;
    for (int n = 0; n < P; ++n) { a[2 * n] = x[2 * n]; a[2 * n + 1] = 0.0f; }
    fft_rec_f(&p->pP, 0, P, a, 1, xr_out, -1);
    for (int n = 0; n < P; ++n) {
        const float im = x[2 * n + 1];
        b[2 * n] = im * p->ff[2 * n]; b[2 * n + 1] = im * p->ff[2 * n + 1];
    }
    fft_rec_f(&p->pP, 0, P, b, 1, xi_out, -1);
}

void orc_fftpath_memoize(orc_fftpath *p, const float *ptcl, float *memo)
{
    const int P = p->g.pftsz, K = K_OF(&p->g);
    float *work = (float *)malloc(sizeof(float) * 4 * P);
    for (int ik = 0; ik < K; ++ik)
        shell_transforms(p, ptcl + 2 * ik * P, work, memo + ik * 4 * P, memo + ik * 4 * P + 2 * P);
    free(work);
}

void orc_fftpath_gencorrs(orc_fftpath *p, const float *ref, const float *ptcl_memo, float sqsum_ptcl,
                          const float *ctfmat, const float *shvec, const double *argtransf,
                          const double *argtransf_shellone, float *cc)
{
    const orc_geom *g = &p->g;
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    float *pr = (float *)malloc(sizeof(float) * 2 * K * P);
    float *work = (float *)malloc(sizeof(float) * (4 * P + 4 * P + 2 * N + 2 * N + 2 * N));
    float *rre = work + 4 * P, *rim = rre + 2 * P, *prod = work + 8 * P, *full = prod + 2 * N, *bt = full + 2 * N;
    float *acc = (float *)calloc(N, sizeof(float));
    /* reference preparation in single precision: pft_ref = (ref*ctf)*cmplx(shmat_8) */
    double *sh8 = NULL;
    if (shvec) {
        sh8 = (double *)malloc(sizeof(double) * 2 * K * P);
        orc_shmat(g, argtransf, argtransf_shellone, (double)shvec[0], (double)shvec[1], sh8);
    }
    float sqr = 0.0f;
    for (int i = 0; i < K * P; ++i) {
        float re = ref[2 * i], im = ref[2 * i + 1];
        if (ctfmat) { re *= ctfmat[i]; im *= ctfmat[i]; }
        if (sh8) {
            const float sr = (float)sh8[2 * i], si = (float)sh8[2 * i + 1];
            const float tr = re * sr - im * si, ti = re * si + im * sr;
            re = tr; im = ti;
        }
        pr[2 * i] = re; pr[2 * i + 1] = im;
        sqr += re * re + im * im;      /* gencorrs_cc_2: sum over all shells */
    }
    for (int ik = 0; ik < Ks; ++ik) {
        shell_transforms(p, pr + 2 * ik * P, work, rre, rim);
        const float *mre = ptcl_memo + ik * 4 * P, *mim = mre + 2 * P;
        /* product spectrum X(m), m = 0..N/2: even m = 2j from the re-transforms,
         * odd m = 2j+1 from the im-transforms */
        for (int m = 0; m <= N / 2; ++m) {
            const int j = m / 2;
            const float *a = (m & 1) ? rim : rre, *b = (m & 1) ? mim : mre;
            const float ar = a[2 * j], ai = -a[2 * j + 1], br = b[2 * j], bi = b[2 * j + 1];
            prod[2 * m] = 4.0f * (ar * br - ai * bi);
            prod[2 * m + 1] = 4.0f * (ar * bi + ai * br);
        }
        /* c2r(N): Hermitian extension, backward transform, real part */
        for (int m = 0; m <= N / 2; ++m) { full[2 * m] = prod[2 * m]; full[2 * m + 1] = prod[2 * m + 1]; }
        full[1] = 0.0f; full[2 * (N / 2) + 1] = 0.0f;
        for (int m = N / 2 + 1; m < N; ++m) { full[2 * m] = prod[2 * (N - m)]; full[2 * m + 1] = -prod[2 * (N - m) + 1]; }
        fft_rec_f(&p->pN, 0, N, full, 1, bt, +1);
        for (int r = 0; r < N; ++r) acc[r] += bt[2 * r];
    }
    const float den = sqrtf(sqr * sqsum_ptcl);
    for (int r = 0; r < N; ++r) cc[r] = (acc[r] / (float)(2 * N)) / den;
    free(pr); free(work); free(acc); free(sh8);
}

/* every correlation of one particle against nrefs references x nshifts shifts through the
 * FP32 FFT path (gencorrs_cc_2 :1502-1534 per (reference, shift) pair, the particle's
 * transforms memoized once as memoize_fft :864-877 does), OpenMP over the pairs.
 * out[(r * nshifts + s) * nrots + irot - 1]; the error of the reference's own FP32 loop
 * is measured on this output. */
int orc_fftpath_allcorrs(const orc_geom *g, int nrefs, const float *refs, const float *ptcl, const float *ctfmat,
                         int nshifts, const float *shifts, float *out, int nthreads)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    float *polar = (float *)malloc(sizeof(float) * 2 * N * K);
    double *at = (double *)malloc(sizeof(double) * N * K);
    double *at1 = (double *)malloc(sizeof(double) * N);
    orc_tables(g, polar, at, at1);
    orc_fftpath *fp0 = orc_fftpath_new(g);
    float *memo = (float *)malloc(sizeof(float) * orc_fftpath_memo_size(g));
    orc_fftpath_memoize(fp0, ptcl, memo);
    float sqp = 0.0f;
    for (int j = 0; j < 2 * Ks * P; ++j) sqp += ptcl[j] * ptcl[j];
    int used = 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    #pragma omp parallel
    {
#ifdef _OPENMP
        #pragma omp single
        used = omp_get_num_threads();
#endif
        orc_fftpath *fp = orc_fftpath_new(g);
        #pragma omp for schedule(dynamic, 4)
        for (int rs = 0; rs < nrefs * nshifts; ++rs) {
            const int r = rs / nshifts, s = rs % nshifts;
            orc_fftpath_gencorrs(fp, refs + (size_t)r * 2 * K * P, memo, sqp, ctfmat, shifts + 2 * s, at, at1,
                                 out + (size_t)rs * N);
        }
        orc_fftpath_free(fp);
    }
    orc_fftpath_free(fp0);
    free(memo); free(polar); free(at); free(at1);
    return used;
}

/* exhaustive search: the greedy strategy's loop over all references
 * (simple_strategy2D_greedy.f90:33-58) with the shift grid of the exhaustive
 * in-plane search (simple_pftcc_shsrch_grad.f90:182-199), each call a
 * gencorrs_cc_2 through the FFT path and a maxloc over rotations; OpenMP over
 * particles as in the 3D matcher (simple_strategy3D_matcher.f90:204). */
int orc_cpu_search(const orc_geom *g, int nrefs, const float *refs, int nptcls, const float *ptcls,
                   const float *ctfmats, int nshifts, const float *shifts,
                   int *best_ref, int *best_rot, int *best_shift, float *best_cc, int nthreads)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    float *polar = (float *)malloc(sizeof(float) * 2 * N * K);
    double *at = (double *)malloc(sizeof(double) * N * K);
    double *at1 = (double *)malloc(sizeof(double) * N);
    orc_tables(g, polar, at, at1);
    int used = 1;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#endif
    #pragma omp parallel
    {
#ifdef _OPENMP
        #pragma omp single
        used = omp_get_num_threads();
#endif
        orc_fftpath *fp = orc_fftpath_new(g);
        float *memo = (float *)malloc(sizeof(float) * orc_fftpath_memo_size(g));
        float *cc = (float *)malloc(sizeof(float) * N);
        #pragma omp for schedule(static)
        for (int i = 0; i < nptcls; ++i) {
            const float *pt = ptcls + (size_t)i * 2 * K * P;
            orc_fftpath_memoize(fp, pt, memo);
            float sqp = 0.0f;
            for (int j = 0; j < 2 * Ks * P; ++j) sqp += pt[j] * pt[j];
            float bcc = -INFINITY; int br = -1, bro = -1, bs = -1;
            for (int r = 0; r < nrefs; ++r)
                for (int s = 0; s < nshifts; ++s) {
                    orc_fftpath_gencorrs(fp, refs + (size_t)r * 2 * K * P, memo, sqp,
                                         ctfmats ? ctfmats + (size_t)i * K * P : NULL,
                                         shifts + 2 * s, at, at1, cc);
                    for (int rot = 0; rot < N; ++rot)
                        if (cc[rot] > bcc) { bcc = cc[rot]; br = r; bro = rot + 1; bs = s; }
                }
            best_ref[i] = br; best_rot[i] = bro; best_shift[i] = bs; best_cc[i] = bcc;
        }
        free(memo); free(cc);
        orc_fftpath_free(fp);
    }
    free(polar); free(at); free(at1);
    return used;
}

/* ------------------------------------------------------------------------- */
/* Euclidean objective (cc_objfun = OBJFUN_EUCLID), reference frame.
 * setup_pxls_p_shell (:879-893): pixels of the positive quadrant h, k = 1..kto whose
 * rounded radius nint(sqrt(h^2 + k^2)) is a shell in kfrom..kto. */
void orc_pxls_p_shell(int kfrom, int kto, double *pxls)
{
    for (int i = 0; i < kto - kfrom + 1; ++i) pxls[i] = 0.0;
    for (int h = 1; h <= kto; ++h)
        for (int k = 1; k <= kto; ++k) {
            const int sh = (int)lround(sqrt((double)(h * h + k * k)));
            if (sh >= kfrom && sh <= kto) pxls[sh - kfrom] += 1.0;
        }
}

/* calc_euclidk_for_rot (:1392-1415): sum_n |ref(n) - ptcl~(n + irot - 1)|^2 with the
 * same cyclic extension as corrk_for_rot (the reference's four-way split on irot) */
static double euclidk_for_rot(int P, const double *ref_k, const float *ptcl_k, int irot)
{
    const int N = 2 * P, s = irot - 1;
    double acc = 0.0;
    for (int n = 0; n < P; ++n) {
        const int j = (n + s) % N;
        double qr, qi;
        if (j < P) { qr = ptcl_k[2 * j]; qi = ptcl_k[2 * j + 1]; }
        else { qr = ptcl_k[2 * (j - P)]; qi = -ptcl_k[2 * (j - P) + 1]; }
        const double dr = ref_k[2 * n] - qr, di = ref_k[2 * n + 1] - qi;
        acc += dr * dr + di * di;
    }
    return acc;
}

/* gencorrs_euclid_1/_2: for every rotation
 *   sum_{k = kfrom..kstop} pxls(k) / P * (2 kcorrs_k(irot) - S_ptcl(k) - S_ref(k)) / (2 sigma2(k))
 * with kcorrs_k the per-shell correlation of calc_k_corrs (:1164-1188, the same cyclic
 * correlation as corrk_for_rot) and S the shell's square sums (:1550-1551, :1587-1588).
 * Both variants prepare the reference as ref * ctf (* shmat); gencorrs_euclid_1 goes
 * through prep_ref4corr, whose shell normalisation applies only with match_filt, which
 * the Euclidean objective does not use. */
void orc_gencorrs_euclid(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                         const double *shvec, const double *argtransf, const double *argtransf_shellone,
                         const double *sigma2, const double *pxls, double *euclids)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    prep_ref(g, ref, ctfmat, shvec, argtransf, argtransf_shellone, pr);
    for (int irot = 1; irot <= N; ++irot) euclids[irot - 1] = 0.0;
    for (int ik = 0; ik < Ks; ++ik) {
        const double sp = sqsum_kf(P, ptcl + 2 * ik * P), sr = sqsum_k(P, pr + 2 * ik * P);
        const double w = pxls[ik] / (double)P / (2.0 * sigma2[ik]);
        for (int irot = 1; irot <= N; ++irot)
            euclids[irot - 1] += w * (2.0 * corrk_for_rot(P, pr + 2 * ik * P, ptcl + 2 * ik * P, irot) - sp - sr);
    }
    free(pr);
}

/* f = -sum_{k<=kstop} k * euclidk(irot) / (2 sigma2(k)) * pxls(k) / P (calc_euclid_for_rot_8
 * :1308-1334); grad(d) = sum_{k<=kstop} k * (corrk(T_d, irot) - Re sum_n T_d(n) conj(ref(n)))
 * / sigma2(k) * pxls(k) / P with T_d = i * argtransf_d * ref, argtransf_x the first P rows of
 * argtransf and argtransf_y the last P (:2090-2108) */
void orc_gencorr_euclid_grad_for_rot(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                                     const double *shvec, int irot, const double *argtransf,
                                     const double *argtransf_shellone, const double *sigma2, const double *pxls,
                                     double *f, double *grad)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    double *t = (double *)malloc(sizeof(double) * 2 * P);
    prep_ref(g, ref, ctfmat, shvec, argtransf, argtransf_shellone, pr);
    double fs = 0.0, gx = 0.0, gy = 0.0;
    for (int ik = 0; ik < Ks; ++ik) {
        const double k = (double)(g->kfrom + ik);
        const double *a = pr + 2 * ik * P;
        const float *q = ptcl + 2 * ik * P;
        fs -= k * euclidk_for_rot(P, a, q, irot) / (2.0 * sigma2[ik]) * pxls[ik] / (double)P;
        for (int d = 0; d < 2; ++d) {
            double self = 0.0;
            for (int n = 0; n < P; ++n) {
                const double at = argtransf[ik * N + d * P + n];
                t[2 * n] = -at * a[2 * n + 1];   /* i * at * (ar + i ai) */
                t[2 * n + 1] = at * a[2 * n];
                self += t[2 * n] * a[2 * n] + t[2 * n + 1] * a[2 * n + 1];
            }
            const double diffsq = corrk_for_rot(P, t, q, irot) - self;
            const double contrib = k * diffsq / sigma2[ik] * pxls[ik] / (double)P;
            if (d == 0) gx += contrib; else gy += contrib;
        }
    }
    *f = fs;
    grad[0] = gx;
    grad[1] = gy;
    free(t);
    free(pr);
}

/* sigma_contrib(k) = 0.5 * euclidk(irot) / P, ptcl_sumsq(k) = sum_n |ptcl(n,k)|^2,
 * ref_sumsq(k) = sum_n |ref_prep(n,k)|^2, every shell kfrom..kto (:2177-2187) */
void orc_sigma_contrib(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                       const double *shvec, int irot, const double *argtransf, const double *argtransf_shellone,
                       double *sigma_contrib, double *ptcl_sumsq, double *ref_sumsq)
{
    const int P = g->pftsz, K = K_OF(g);
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    prep_ref(g, ref, ctfmat, shvec, argtransf, argtransf_shellone, pr);
    for (int ik = 0; ik < K; ++ik) {
        sigma_contrib[ik] = 0.5 * euclidk_for_rot(P, pr + 2 * ik * P, ptcl + 2 * ik * P, irot) / (double)P;
        if (ptcl_sumsq) ptcl_sumsq[ik] = sqsum_kf(P, ptcl + 2 * ik * P);
        if (ref_sumsq) ref_sumsq[ik] = sqsum_k(P, pr + 2 * ik * P);
    }
    free(pr);
}

/* ------------------------------------------------------------------------- */
/* Orientation derivatives.  drotmat (simple_ori_light.f90:107-146): d rotmat / d angle with
 * the angle in radians. */
static void drotmat3(double ang_deg, int choice, double r[9])
{
    const double a = ang_deg * 3.14159265358979323846 / 180.0, c = cos(a), s = sin(a);
    for (int i = 0; i < 9; ++i) r[i] = 0.0;
    if (choice == 1) { r[4] = -s; r[5] = -c; r[7] = c; r[8] = -s; }
    else if (choice == 2) { r[0] = -s; r[2] = -c; r[6] = c; r[8] = -s; }
    else { r[0] = -s; r[1] = c; r[3] = -c; r[4] = -s; }
}

/* euler2dm: with R = r3 r2 r1, dR/de1 = r3 r2 dr1, dR/de2 = r3 dr2 r1, dR/de3 = dr3 r2 r1 */
void orc_euler2dm(const double eul[3], double dR[27])
{
    double r1[9], r2[9], r3[9], d1[9], d2[9], d3[9], t[9];
    rotmat3(eul[0], 3, r1);
    rotmat3(eul[1], 2, r2);
    rotmat3(eul[2], 3, r3);
    drotmat3(eul[0], 3, d1);
    drotmat3(eul[1], 2, d2);
    drotmat3(eul[2], 3, d3);
    matmul3(r3, r2, t);
    matmul3(t, d1, dR);
    matmul3(r3, d2, t);
    matmul3(t, r1, dR + 9);
    matmul3(d3, r2, t);
    matmul3(t, r1, dR + 18);
}

/* I1 by the Abramowitz & Stegun 9.8.3 / 9.8.4 polynomial approximations (bessi1,
 * simple_kbinterpol.f90:282-308); x >= 0 */
static double bessi1(double x)
{
    if (x < 3.75) {
        double y = x / 3.75;
        y *= y;
        return x * (0.5 + y * (0.87890594 + y * (0.51498869 + y * (0.15084934 + y * (0.2658733e-1 +
                    y * (0.301532e-2 + y * 0.32411e-3))))));
    }
    const double y = 3.75 / x;
    return (0.39894228 + y * (-0.3988024e-1 + y * (-0.362018e-2 + y * (0.163801e-2 + y * (-0.1031555e-1 +
            y * (0.2282967e-1 + y * (-0.2895312e-1 + y * (0.1787654e-1 + y * (-0.420059e-2))))))))) *
           exp(x) / sqrt(x);
}

/* d apod / dx = -4 beta x I1(beta s) / (s W^3), s = sqrt(1 - (2x/W)^2); 0 where s^2 <= 0 */
double orc_kb_dapod(double x)
{
    const double W = 3.0, beta = 7.4;
    double arg = (2.0 / W) * x;
    arg = 1.0 - arg * arg;
    if (arg <= 0.0) return 0.0;
    const double s = sqrt(arg);
    return -4.0 * beta * x * bessi1(beta * s) / s / (W * W * W);
}

/* fdf_interp_fcomp for every sample of the reference: the window and weights of
 * interp_fcomp_norm, N = sum w c, D = sum w, and for each angle e_j the weight derivative
 * wd_j = sum over the axes d of (-dapod(win_d - loc_d) * dloc_d/de_j) times the other two
 * axes' apod, dloc/de_j = vec dR_j; fcomp = N / D, dfcomp_j = (sum wd_j c * D - N sum wd_j) / D^2.
 * Every shell kfrom..kto, no mask (fdf_project_polar :257-266). */
void orc_fdf_project_polar(const orc_geom *g, const float *polar, int box, const float *cmat_exp,
                           const double eul[3], double *pft, double *dpft)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g);
    const int E = box / 2 + 2, S = 2 * E + 1;
    double R[9], dR[27];
    orc_euler2m(eul, R);
    orc_euler2dm(eul, dR);
    for (int ik = 0; ik < K; ++ik)
        for (int i = 0; i < P; ++i) {
            const double vx = polar[ik * 2 * N + i], vy = polar[ik * 2 * N + N + i];
            double loc[3], dl[3][3];
            for (int d = 0; d < 3; ++d) {
                loc[d] = vx * R[d] + vy * R[3 + d];
                for (int j = 0; j < 3; ++j) dl[j][d] = vx * dR[9 * j + d] + vy * dR[9 * j + 3 + d];
            }
            int w0[3];
            double wa[3][3], da[3][3];
            for (int d = 0; d < 3; ++d) {
                w0[d] = f_nint(loc[d]) - 1;
                for (int l = 0; l < 3; ++l) {
                    wa[d][l] = orc_kb_apod((double)(w0[d] + l) - loc[d]);
                    da[d][l] = orc_kb_dapod((double)(w0[d] + l) - loc[d]);
                }
            }
            double nr = 0.0, ni = 0.0, D = 0.0, njr[3] = {0, 0, 0}, nji[3] = {0, 0, 0}, dj[3] = {0, 0, 0};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b)
                    for (int c = 0; c < 3; ++c) {
                        const size_t e = ((size_t)(w0[2] + c + E) * S + (w0[1] + b + E)) * S + (w0[0] + a + E);
                        const double cr = cmat_exp[2 * e], ci = cmat_exp[2 * e + 1];
                        const double w = wa[0][a] * wa[1][b] * wa[2][c];
                        nr += w * cr; ni += w * ci; D += w;
                        for (int j = 0; j < 3; ++j) {
                            const double wd = -da[0][a] * dl[j][0] * wa[1][b] * wa[2][c]
                                              - wa[0][a] * da[1][b] * dl[j][1] * wa[2][c]
                                              - wa[0][a] * wa[1][b] * da[2][c] * dl[j][2];
                            njr[j] += wd * cr; nji[j] += wd * ci; dj[j] += wd;
                        }
                    }
            pft[2 * (ik * P + i)] = nr / D;
            pft[2 * (ik * P + i) + 1] = ni / D;
            for (int j = 0; j < 3; ++j) {
                const size_t o = 2 * ((size_t)j * K * P + ik * P + i);
                dpft[o] = (njr[j] * D - nr * dj[j]) / (D * D);
                dpft[o + 1] = (nji[j] * D - ni * dj[j]) / (D * D);
            }
        }
}

void orc_gencorr_cont_shift_grad(const orc_geom *g, const float *ref, const float *dref, const float *ptcl,
                                 const double *ctfmat, const double *shvec, int irot, const double *argtransf,
                                 const double *argtransf_shellone, double *f, double *grad5)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    double *pd = (double *)malloc(sizeof(double) * 2 * K * P);
    double *t = (double *)malloc(sizeof(double) * 2 * P);
    prep_ref(g, ref, ctfmat, shvec, argtransf, argtransf_shellone, pr);
    double y = 0.0, sqr = 0.0, sqp = 0.0, T1[3] = {0, 0, 0}, T2[3] = {0, 0, 0};
    for (int ik = 0; ik < Ks; ++ik) {
        y += corrk_for_rot(P, pr + 2 * ik * P, ptcl + 2 * ik * P, irot);
        sqr += sqsum_k(P, pr + 2 * ik * P);
        sqp += sqsum_kf(P, ptcl + 2 * ik * P);
    }
    for (int j = 0; j < 3; ++j) {
        /* pft_dref(:,:,j) * ctf * shmat, the prepared reference's own operations */
        prep_ref(g, dref + (size_t)j * 2 * K * P, ctfmat, shvec, argtransf, argtransf_shellone, pd);
        for (int ik = 0; ik < Ks; ++ik) {
            const double *a = pd + 2 * ik * P, *b = pr + 2 * ik * P;
            T1[j] += corrk_for_rot(P, a, ptcl + 2 * ik * P, irot);
            for (int n = 0; n < P; ++n) T2[j] += a[2 * n] * b[2 * n] + a[2 * n + 1] * b[2 * n + 1];
        }
    }
    const double den = sqrt(sqr * sqp);
    *f = y / den;
    for (int j = 0; j < 3; ++j) grad5[j] = (T1[j] - y * T2[j] / sqr) / den;
    for (int d = 0; d < 2; ++d) {
        double c = 0.0;
        for (int ik = 0; ik < Ks; ++ik) {
            const double *a = pr + 2 * ik * P;
            for (int n = 0; n < P; ++n) {
                const double at = argtransf[ik * N + d * P + n];
                t[2 * n] = -at * a[2 * n + 1];
                t[2 * n + 1] = at * a[2 * n];
            }
            c += corrk_for_rot(P, t, ptcl + 2 * ik * P, irot);
        }
        grad5[3 + d] = c / den;
    }
    free(t);
    free(pd);
    free(pr);
}

/* ------------------------------------------------------------------------- */
/* Particle ingestion, prepimg4align (simple_strategy2D3D_common.f90:316-366), stated step by
 * step as the reference's image methods run:
 *  noise_norm (simple_image.f90:6623-6640) against the background, the pixels outside the disc
 *    of radius msk (disc_2 :506-523; cendist :2719-2748 measures from B/2 + 1, 1-based);
 *  fft (fwd_ft :5773-5782): shift_phorig (quadrant swap), r2c, / B^2;
 *  shift2Dserial([-x, -y]) (:6149-6174) when |x| or |y| > SHTHRESH = 0.001 (:31): cmat(h, k) times
 *    exp(i (h sh1 + k sh2)), sh = shvec * shconst in single precision, shconst = PI / (B/2)
 *    (:445), the phase in double and rounded to single;
 *  phase flip (simple_ctf.f90 apply_serial 'flip' :312-403): sign(1, tval), tval = sin(evalPhSh
 *    (+ phshift) + amp_contr_const) at spaFreqSq = (h/B)^2 + (k/B)^2, ang = atan2(k, h);
 *  ifft (bwd_ft :5784-5791): c2r, shift_phorig;
 *  clip (:6471-6516): the centred boxmatch window from (B - Bm)/2 + 1;
 *  mask 'soft' (:6208-6300): zero_background (:5176-5203) -- the mean of the k-th smallest values,
 *    k = Bm/2 (selec, simple_math.f90:2204), of the four border lines, subtracted when its
 *    magnitude exceeds TINY = 1e-10 -- then cosedge (simple_math.f90:1089-1103) with box
 *    minlen = min(nint(2 (msk + COSMSKHALFWIDTH)), Bm), COSMSKHALFWIDTH = 6 (simple_defs.f90:130),
 *    evaluated at (cis(i), cjs(j)) = (-Bm/2 + i - 1, -Bm/2 + j - 1) for i, j <= Bm/2 and applied to
 *    the four mirrored pixels, skipped where e > 0.9999;
 *  fft and the factor Bm^2 / B^2 (:364-365). */
static void fft2d(int B, double *z, int sign)
{
    double *a = (double *)malloc(sizeof(double) * 2 * B), *b = (double *)malloc(sizeof(double) * 2 * B);
    for (int r = 0; r < B; ++r) {   /* along x */
        orc_cfft(B, z + 2 * (size_t)r * B, b, sign);
        memcpy(z + 2 * (size_t)r * B, b, sizeof(double) * 2 * B);
    }
    for (int c = 0; c < B; ++c) {   /* along y */
        for (int r = 0; r < B; ++r) { a[2 * r] = z[2 * ((size_t)r * B + c)]; a[2 * r + 1] = z[2 * ((size_t)r * B + c) + 1]; }
        orc_cfft(B, a, b, sign);
        for (int r = 0; r < B; ++r) { z[2 * ((size_t)r * B + c)] = b[2 * r]; z[2 * ((size_t)r * B + c) + 1] = b[2 * r + 1]; }
    }
    free(a);
    free(b);
}

/* shift_phorig (:6016-6114) of an even square image: swap quadrant (i, j) with (i + B/2, j + B/2) */
static void phorig(int B, double *r)
{
    const int H = B / 2;
    for (int j = 0; j < H; ++j)
        for (int i = 0; i < B; ++i) {
            const int i2 = (i + H) % B, j2 = j + H;
            const double t = r[(size_t)j * B + i];
            r[(size_t)j * B + i] = r[(size_t)j2 * B + i2];
            r[(size_t)j2 * B + i2] = t;
        }
}

static int cmp_dbl(const void *a, const void *b)
{
    const double x = *(const double *)a, y = *(const double *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* kbinterpol%instr (simple_kbinterpol.f90:211-225) for the window of half-width 1.5 (W = 3,
 * beta = 7.4, :97-103): sinh(y) / y, y = sqrt(beta^2 - (pi W x)^2) (|x| <= 1/2 lies below the
 * threshold beta / (pi W)); the single-precision constants and argument of the reference */
static double kb_instr(double x)
{
    const double piW = (double)(3.14159265f * 3.0f), betasq = (double)(7.4f * 7.4f);
    const double y = sqrt(betasq - (piW * x) * (piW * x));
    return y < 1e-10 ? 1.0 : sinh(y) / y;
}

void orc_prepimg4align(int box, int boxmatch, const float *img, double msk, double x, double y, const orc_ctf *ctf,
                       double *cmat_out)
{
    orc_prepimg4align_opts(box, boxmatch, img, msk, 0.0, 0.0, 0.0, 0, x, y, ctf, cmat_out);
}

void orc_prepimg4align_opts(int box, int boxmatch, const float *img, double msk, double inner, double width,
                            double focusmsk, int griddev, double x, double y, const orc_ctf *ctf, double *cmat_out)
{
    const int B = box, Bm = boxmatch, hB = B / 2 + 1, hBm = Bm / 2 + 1;
    double *r = (double *)malloc(sizeof(double) * B * B);
    double *z = (double *)malloc(sizeof(double) * 2 * B * B);
    for (int e = 0; e < B * B; ++e) r[e] = img[e];
    /* noise_norm */
    {
        const double c = B / 2 + 1;
        long npix = 0;
        double s = 0.0;
        unsigned char *bg = (unsigned char *)malloc((size_t)B * B);
        for (int j = 0; j < B; ++j)
            for (int i = 0; i < B; ++i) {
                const double di = (i + 1) - c, dj = (j + 1) - c;
                bg[(size_t)j * B + i] = !(sqrt(di * di + dj * dj) <= msk);
                if (bg[(size_t)j * B + i]) { ++npix; s += r[(size_t)j * B + i]; }
            }
        const double ave = s / (double)npix;
        if (fabs(ave) > 1e-10)
            for (int e = 0; e < B * B; ++e) r[e] -= ave;
        double ep = 0.0, var = 0.0;
        for (int e = 0; e < B * B; ++e)
            if (bg[e]) { ep += r[e]; var += r[e] * r[e]; }
        var = (var - ep * ep / (double)npix) / ((double)npix - 1.0);
        if (var == var && var > 0.0) {
            const double sd = sqrt(var);
            for (int e = 0; e < B * B; ++e) r[e] /= sd;
        }
        free(bg);
    }
    /* fft */
    phorig(B, r);
    for (int e = 0; e < B * B; ++e) { z[2 * e] = r[e] / ((double)B * B); z[2 * e + 1] = 0.0; }
    fft2d(B, z, -1);
    /* shift and phase flip on the half plane h = 0..B/2, k = -B/2..B/2-1, mirrored onto the
     * Friedel mates so that the inverse transform stays real */
    const int do_shift = fabs(x) > 0.001 || fabs(y) > 0.001;
    const float shconst = (float)3.14159265358979323846 / (float)(B / 2);
    const double sh1 = (double)((float)(-x) * shconst), sh2 = (double)((float)(-y) * shconst);
    ctf_consts kc;
    if (ctf) { kc = ctf_setup(ctf); kc.phshift = ctf->phshift; }
    for (int kphys = 0; kphys < B; ++kphys) {
        const int k = kphys < B / 2 ? kphys : kphys - B;
        for (int h = 0; h <= B / 2; ++h) {
            double fr = 1.0, fi = 0.0;
            if (do_shift) {
                const double a = h * sh1 + k * sh2;
                fr = (double)(float)cos(a);
                fi = (double)(float)sin(a);
            }
            if (ctf) {
                const double hinv = (double)h / B, kinv = (double)k / B;
                const double t = sin(ctf_chi(&kc, hinv * hinv + kinv * kinv, atan2((double)k, (double)h)));
                const double sg = t >= 0.0 ? 1.0 : -1.0;
                fr *= sg; fi *= sg;
            }
            double *v = z + 2 * ((size_t)kphys * B + h);
            const double vr = v[0] * fr - v[1] * fi, vi = v[0] * fi + v[1] * fr;
            v[0] = vr; v[1] = vi;
            if (h > 0 && h < B / 2) {   /* Friedel mate (-h, -k) */
                double *w = z + 2 * ((size_t)((B - kphys) % B) * B + (B - h));
                w[0] = vr; w[1] = -vi;
            }
        }
    }
    /* ifft: c2r of the half plane (the full spectrum is Hermitian), then shift_phorig */
    fft2d(B, z, +1);
    for (int e = 0; e < B * B; ++e) r[e] = z[2 * e];
    phorig(B, r);
    /* clip */
    double *m = (double *)malloc(sizeof(double) * Bm * Bm);
    const int st = (B - Bm) / 2;
    for (int j = 0; j < Bm; ++j)
        for (int i = 0; i < Bm; ++i) m[(size_t)j * Bm + i] = r[(size_t)(j + st) * B + (i + st)];
    /* zero_background */
    {
        double *line = (double *)malloc(sizeof(double) * Bm);
        double med = 0.0;
        for (int which = 0; which < 4; ++which) {
            for (int t = 0; t < Bm; ++t) {
                switch (which) {
                case 0: line[t] = m[(size_t)t * Bm + 0]; break;              /* rmat(1, :)  */
                case 1: line[t] = m[(size_t)t * Bm + (Bm - 1)]; break;       /* rmat(Bm, :) */
                case 2: line[t] = m[t]; break;                                /* rmat(:, 1)  */
                default: line[t] = m[(size_t)(Bm - 1) * Bm + t]; break;      /* rmat(:, Bm) */
                }
            }
            qsort(line, Bm, sizeof(double), cmp_dbl);
            med += line[Bm / 2 - 1];
        }
        med /= 4.0;
        if (fabs(med) > 1e-10)
            for (int e = 0; e < Bm * Bm; ++e) m[e] -= med;
        free(line);
    }
    /* cosine edge: mask(msk, 'soft', inner, width) with l_innermsk, else mask(focusmsk, 'soft')
     * with l_focusmsk, else mask(msk, 'soft') (prepimg4align :349-358; mask :6208-6300) */
    {
        const double mrad = inner > 0.0 ? msk : (focusmsk > 0.0 ? focusmsk : msk);
        const double iw = width > 0.0 ? width : 10.0;
        int minlen = (int)f_nint(2.0 * (mrad + 6.0));
        if (minlen > Bm) minlen = Bm;
        const double maxrad = (double)(minlen / 2), cwidth = 2.0 * (maxrad - mrad);
        for (int i = 1; i <= Bm / 2; ++i)
            for (int j = 1; j <= Bm / 2; ++j) {
                const double cx = -Bm / 2.0 + (i - 1), cy = -Bm / 2.0 + (j - 1);
                const double rad = sqrt(cx * cx + cy * cy);
                double e = 1.0;
                if (rad >= maxrad) e = 0.0;
                else if (rad >= maxrad - cwidth) e = (cos(((rad - (maxrad - cwidth)) / cwidth) * 3.14159265358979323846) + 1.0) / 2.0;
                if (inner > 0.0) {   /* cosedge_inner (simple_math.f90:1128-1140) */
                    double wi;
                    if (rad < inner - iw) wi = 0.0;
                    else if (rad > inner) wi = 1.0;
                    else wi = (1.0 + cos(3.14159265358979323846 * (inner - rad) / iw)) / 2.0;
                    e *= wi;
                }
                if (e > 0.9999) continue;
                const int ir = Bm + 1 - i, jr = Bm + 1 - j;
                m[(size_t)(j - 1) * Bm + (i - 1)] *= e;
                m[(size_t)(jr - 1) * Bm + (i - 1)] *= e;
                m[(size_t)(j - 1) * Bm + (ir - 1)] *= e;
                m[(size_t)(jr - 1) * Bm + (ir - 1)] *= e;
            }
    }
    /* griddev 'yes': div_by_instrfun (simple_polarizer.f90:111-116) with the instrument function
     * image of gen_instrfun_img (simple_gridding.f90:18-55): w(i) w(j), w(i) = instr((i - c) / Bm),
     * c = Bm/2 + 1, 1-based i */
    if (griddev) {
        for (int j = 1; j <= Bm; ++j)
            for (int i = 1; i <= Bm; ++i) {
                const double wi = kb_instr((double)(float)((float)(i - (Bm / 2 + 1)) / (float)Bm));
                const double wj = kb_instr((double)(float)((float)(j - (Bm / 2 + 1)) / (float)Bm));
                m[(size_t)(j - 1) * Bm + (i - 1)] /= wi * wj;
            }
    }
    /* fft and the box factor */
    phorig(Bm, m);
    double *zm = (double *)malloc(sizeof(double) * 2 * Bm * Bm);
    const double f = 1.0 / ((double)Bm * Bm) * ((double)Bm * Bm) / ((double)B * B);
    for (int e = 0; e < Bm * Bm; ++e) { zm[2 * e] = m[e] * f; zm[2 * e + 1] = 0.0; }
    fft2d(Bm, zm, -1);
    for (int kphys = 0; kphys < Bm; ++kphys)
        for (int h = 0; h < hBm; ++h) {
            cmat_out[2 * ((size_t)kphys * hBm + h)] = zm[2 * ((size_t)kphys * Bm + h)];
            cmat_out[2 * ((size_t)kphys * hBm + h) + 1] = zm[2 * ((size_t)kphys * Bm + h) + 1];
        }
    (void)hB;
    free(zm);
    free(m);
    free(z);
    free(r);
}

void orc_gencorrs_euclid_ptclframe(const orc_geom *g, const float *ref, const float *ptcl, const double *ctfmat,
                                   const double *shvec, const double *argtransf, const double *argtransf_shellone,
                                   const double *sigma2, const double *pxls, double *euclids)
{
    const int N = g->nrots, P = g->pftsz, K = K_OF(g), Ks = g->kstop - g->kfrom + 1;
    double *pr = (double *)malloc(sizeof(double) * 2 * K * P);
    prep_ref(g, ref, NULL, shvec, argtransf, argtransf_shellone, pr);   /* A = ref * shmat */
    for (int s = 0; s < N; ++s) {
        double acc = 0.0;
        for (int ik = 0; ik < Ks; ++ik) {
            const double w = pxls[ik] / (double)P / sigma2[ik];
            const double *a = pr + 2 * ik * P;
            const float *q = ptcl + 2 * ik * P;
            double e = 0.0;
            for (int n = 0; n < P; ++n) {
                const int j = (n + s) % N, jp = j % P;
                const double c = ctfmat ? ctfmat[ik * P + jp] : 1.0;
                const double qr = q[2 * jp], qi = j < P ? q[2 * jp + 1] : -q[2 * jp + 1];
                const double dr = a[2 * n] * c - qr, di = a[2 * n + 1] * c - qi;
                e += dr * dr + di * di;
            }
            acc += w * e;
        }
        euclids[s] = -0.5 * acc;
    }
    free(pr);
}

/* ------------------------------------------------------------------------- */
/* The matched-filter mode.  shellnorm_and_filter_ref_8 (:783-807), l_match_filt branch. */
void orc_shellnorm_factors(const orc_geom *g, const float *ref, const float *optlp, double *scale)
{
    orc_shellnorm_factors_mode(g, ref, optlp, 0, scale);
}

/* pssnr = 1: the l_pssnr branch of shellnorm_and_filter_ref(_8) (:763-770, :789-796):
 * sqrt(ssnr k) / sqrt(pw) (sqrt(ssnr k) where pw <= 1e-12), ssnr = ref_optlp(k, iref), k the
 * shell number */
void orc_shellnorm_factors_mode(const orc_geom *g, const float *ref, const float *optlp, int pssnr, double *scale)
{
    const int P = g->pftsz, Ks = g->kstop - g->kfrom + 1;
    for (int ik = 0; ik < Ks; ++ik) {
        const double pw = sqsum_kf(P, ref + 2 * ik * P) / (double)P;
        const double o = optlp ? (double)optlp[ik] : 1.0;
        const double w = pssnr ? sqrt(o * (double)(g->kfrom + ik)) : o;
        scale[ik] = pw > 1e-12 ? w / sqrt(pw) : w;
    }
}

/* prep_matchfilt (:999-1019), the l_pssnr branch: every shell k <= kstop of the particle times
 * sqrt(k) / sqrt(pw_ptcl) (sqrt(k) where pw_ptcl <= 1e-12) and, sample by sample,
 * sqrt(1 + ssnr |CTF(n,k)|^2) (sqrt(1 + ssnr) without CTF), ssnr = ref_optlp(k, iref) */
void orc_prep_matchfilt_pssnr(const orc_geom *g, const double *ctfmat, const float *optlp, float *ptcl)
{
    const int P = g->pftsz, Ks = g->kstop - g->kfrom + 1;
    for (int ik = 0; ik < Ks; ++ik) {
        const double pw = sqsum_kf(P, ptcl + 2 * ik * P) / (double)P;
        const double ssnr = optlp ? (double)optlp[ik] : 1.0;
        double w = sqrt((double)(g->kfrom + ik));
        if (pw > 1e-12) w /= sqrt(pw);
        for (int n = 0; n < P; ++n) {
            const double c = ctfmat ? ctfmat[ik * P + n] : 1.0;
            const double f = w * sqrt(1.0 + ssnr * c * c);
            ptcl[2 * (ik * P + n)] = (float)(f * ptcl[2 * (ik * P + n)]);
            ptcl[2 * (ik * P + n) + 1] = (float)(f * ptcl[2 * (ik * P + n) + 1]);
        }
    }
}

/* The Savitzky & Golay (1964) least-squares smoothing coefficients for a 7-point window and a
 * quartic, c_{-3..3} = (5, -30, 75, 131, 75, -30, 5) / 231 (the values savgol's normal equations
 * give for nl = nr = 3, m = 4, ld = 0); y(i) = sum_k c_k y(i + k) for i <= n - 3 with the points
 * left of the first skipped, as SavitzkyGolay_filter applies them. */
void orc_savgol7(int n, double *y)
{
    static const double c[7] = {5.0 / 231.0, -30.0 / 231.0, 75.0 / 231.0, 131.0 / 231.0,
                                75.0 / 231.0, -30.0 / 231.0, 5.0 / 231.0};
    double *ys = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    for (int i = 0; i < n; ++i) ys[i] = y[i];
    for (int i = 0; i < n - 3; ++i) {
        double v = 0.0;
        for (int k = -3; k <= 3; ++k)
            if (i + k >= 0) v += c[k + 3] * ys[i + k];
        y[i] = v;
    }
    free(ys);
}

void orc_prep_matchfilt(const orc_geom *g, const float *ref, const double *ctfmat, const float *optlp, int irot,
                        float *ptcl)
{
    const int P = g->pftsz, Ks = g->kstop - g->kfrom + 1, N = g->nrots;
    double *pr = (double *)malloc(sizeof(double) * 2 * Ks * P);
    double *pp = (double *)malloc(sizeof(double) * 2 * Ks * P);
    double *diff = (double *)malloc(sizeof(double) * Ks), *fit = (double *)malloc(sizeof(double) * Ks);
    /* reference times |CTF|, particle as held; both shell-normalised by optlp / sqrt(power) */
    for (int ik = 0; ik < Ks; ++ik) {
        const double o = optlp ? (double)optlp[ik] : 1.0;
        double pwr = 0.0, pwp = 0.0;
        for (int n = 0; n < P; ++n) {
            const double c = ctfmat ? ctfmat[ik * P + n] : 1.0;
            const double rr = ref[2 * (ik * P + n)] * c, ri = ref[2 * (ik * P + n) + 1] * c;
            pr[2 * (ik * P + n)] = rr; pr[2 * (ik * P + n) + 1] = ri;
            pwr += rr * rr + ri * ri;
            const double qr = ptcl[2 * (ik * P + n)], qi = ptcl[2 * (ik * P + n) + 1];
            pp[2 * (ik * P + n)] = qr; pp[2 * (ik * P + n) + 1] = qi;
            pwp += qr * qr + qi * qi;
        }
        pwr /= P;
        pwp /= P;
        const double wp = pwp > 1e-12 ? o / sqrt(pwp) : o, wr = pwr > 1e-12 ? o / sqrt(pwr) : o;
        for (int n = 0; n < 2 * P; ++n) { pp[2 * ik * P + n] *= wp; pr[2 * ik * P + n] *= wr; }
    }
    /* power of the difference at irot: ref(n) - ptcl~(n + irot - 1) (the reference's case split) */
    for (int ik = 0; ik < Ks; ++ik) {
        double d = 0.0;
        for (int n = 0; n < P; ++n) {
            const int j = (n + irot - 1) % N, jp = j % P;
            const double qr = pp[2 * (ik * P + jp)], qi = j < P ? pp[2 * (ik * P + jp) + 1] : -pp[2 * (ik * P + jp) + 1];
            const double dr = pr[2 * (ik * P + n)] - qr, di = pr[2 * (ik * P + n) + 1] - qi;
            d += dr * dr + di * di;
        }
        diff[ik] = d / P;
        fit[ik] = diff[ik];
    }
    orc_savgol7(Ks, fit);
    for (int ik = 0; ik < Ks; ++ik)
        if (fit[ik] <= 0.0) fit[ik] = diff[ik];
    for (int ik = 0; ik < 3 && ik < Ks; ++ik) fit[ik] = diff[ik];
    /* filter: the normalised particle times 1/sqrt(its power) and sqrt(ssnr / (ssnr + 1)) */
    for (int ik = 0; ik < Ks; ++ik) {
        double pwp = 0.0, pwr = 0.0;
        for (int n = 0; n < P; ++n) {
            pwp += pp[2 * (ik * P + n)] * pp[2 * (ik * P + n)] + pp[2 * (ik * P + n) + 1] * pp[2 * (ik * P + n) + 1];
            pwr += pr[2 * (ik * P + n)] * pr[2 * (ik * P + n)] + pr[2 * (ik * P + n) + 1] * pr[2 * (ik * P + n) + 1];
        }
        pwp /= P;
        pwr /= P;
        double w = pwp > 1e-12 ? 1.0 / sqrt(pwp) : 1.0;
        if (fit[ik] > 1e-12) {
            const double ssnr = pwr / fit[ik];
            w *= sqrt(ssnr / (ssnr + 1.0));
        }
        for (int n = 0; n < 2 * P; ++n) ptcl[2 * ik * P + n] = (float)(w * pp[2 * ik * P + n]);
    }
    free(fit); free(diff); free(pp); free(pr);
}
