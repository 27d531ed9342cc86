// k_matchfilt.cu -- the matched-filter mode (params_glob%l_match_filt, with its l_pssnr
// variant) of simple_polarft_corrcalc.f90:
//   k_shellnorm       the factors of shellnorm_and_filter_ref(_8) (:756-807): shell k <= kstop of
//                     a raw reference scaled by ref_optlp(k, iref) / sqrt(pw), pw its mean power
//                     sum_n |ref(n,k)|^2 / P (FP64), or by ref_optlp(k, iref) where pw <= 1e-12;
//                     one block per (set, reference) -> snorm[set][iref][k];
//   k_shellnorm_apply the same factors on the m-domain search's reference spectra (UA: the
//                     reference times shift phases, linear in the reference; RU: |ref|^2, by
//                     the factor squared), rows r * nshifts + s of reference r;
//   k_prep_matchfilt  prep_matchfilt (:987-1095), l_match_filt branch: the held particle and the
//                     reference times |CTF| both shell-normalised by ref_optlp / sqrt(power); the
//                     power of their difference at irot, smoothed over the shells by the 7-point
//                     quartic Savitzky-Golay filter (SavitzkyGolay_filter, simple_math.f90:
//                     3511-3588; the first three shells and non-positive fits keep the raw
//                     difference); the particle rescaled by 1/sqrt(its power) sqrt(ssnr/(ssnr+1)),
//                     ssnr = reference power / fitted difference power; written back with its
//                     square sum over kfrom..kstop (set_ptcl_pft + memoize_sqsum_ptcl).
//                     One block per request, FP64 sums.
#include "pftcc_internal.cuh"

#include <algorithm>

namespace pftcc {

constexpr int MF_THREADS = 256;

__device__ __forceinline__ double mf_block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < MF_THREADS / 32; ++w) t += red[w];
    return t;
}

// per-shell sums of |x|^2 over the P samples of each shell k < Ks into out[k] (shared memory),
// one warp per shell
__device__ void mf_shell_power(const float2 *x, int Ks, int P, double *out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = warp; k < Ks; k += MF_THREADS / 32) {
        double s = 0.0;
        for (int n = lane; n < P; n += 32) {
            const float2 v = x[(size_t)k * P + n];
            s += (double)v.x * v.x + (double)v.y * v.y;
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) out[k] = s;
    }
}

// pssnr (params_glob%l_pssnr, :763-770 / :789-796): sqrt(ssnr k) / sqrt(pw) in place of
// optlp / sqrt(pw), ssnr = ref_optlp(k, iref), k the shell number
__global__ void __launch_bounds__(MF_THREADS) k_shellnorm(Geom g, const float2 *__restrict__ refs_even,
                                                          const float2 *__restrict__ refs_odd,
                                                          const float *__restrict__ optlp, int nrefs, int r0, int n,
                                                          int pssnr, float *__restrict__ snorm)
{
    extern __shared__ double pw[];   // [Ks]
    const int set = blockIdx.x / n, r = r0 + blockIdx.x % n;
    const float2 *ref = (set == 0 ? refs_even : refs_odd) + (size_t)r * g.K * g.P;
    mf_shell_power(ref, g.Ks, g.P, pw);
    __syncthreads();
    for (int k = threadIdx.x; k < g.Ks; k += blockDim.x) {
        const double p = pw[k] / (double)g.P, o = (double)optlp[(size_t)r * g.Ks + k];
        const double w = pssnr ? sqrt(o * (double)(g.kfrom + k)) : o;
        snorm[((size_t)set * nrefs + r) * g.Ks + k] = (float)(p > 1e-12 ? w / sqrt(p) : w);
    }
}

// prep_matchfilt's l_pssnr branch (:999-1019): shell k <= kstop of the held particle times
// sqrt(k) / sqrt(pw) (sqrt(k) where pw <= 1e-12) and sqrt(1 + ssnr |CTF(n,k)|^2) per sample,
// ssnr = ref_optlp(k, iref); written back with its square sum (set_ptcl_pft); one block per request
__global__ void __launch_bounds__(MF_THREADS) k_prep_pssnr(Geom g, const int4 *__restrict__ reqs,
                                                           const float *__restrict__ ctfmats,
                                                           const float *__restrict__ optlp, float2 *__restrict__ ptcls,
                                                           float *__restrict__ sqsums)
{
    extern __shared__ double pw[];   // [Ks]
    __shared__ double red[MF_THREADS / 32];
    const int4 rq = reqs[blockIdx.x];   // iref (0-based), slot, irot, pad
    const int P = g.P, Ks = g.Ks;
    float2 *q = ptcls + (size_t)rq.y * g.K * P;
    const float *ctf = ctfmats ? ctfmats + (size_t)rq.y * g.K * P : nullptr;
    const float *o = optlp + (size_t)rq.x * Ks;
    mf_shell_power(q, Ks, P, pw);
    __syncthreads();
    double s = 0.0;
    for (int e = threadIdx.x; e < Ks * P; e += blockDim.x) {
        const int k = e / P;
        const double p = pw[k] / (double)P;
        double w = sqrt((double)(g.kfrom + k));
        if (p > 1e-12) w /= sqrt(p);
        const double c = ctf ? (double)ctf[e] : 1.0;
        const float f = (float)(w * sqrt(1.0 + (double)o[k] * c * c));
        float2 v = q[e];
        v = make_float2(v.x * f, v.y * f);
        q[e] = v;
        s += (double)v.x * v.x + (double)v.y * v.y;
    }
    s = mf_block_sum(s, red);
    if (threadIdx.x == 0) sqsums[rq.y] = (float)s;
}

__global__ void k_shellnorm_apply(int M, int Ks, int J, int nrs, int rows_pad, int nshifts, int nrefs,
                                  const float *__restrict__ s, float2 *__restrict__ UA, double2 *__restrict__ RU)
{
    const long long nua = (long long)M * nrs * Ks, nru = (long long)nrefs * J * Ks;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nua + nru;
         e += (long long)gridDim.x * blockDim.x) {
        if (e < nua) {
            const int k = (int)(e % Ks);
            const long long mr = e / Ks;
            const int row = (int)(mr % nrs), m = (int)(mr / nrs);
            const float f = s[(size_t)(row / nshifts) * Ks + k];
            float2 *u = UA + ((size_t)m * rows_pad + row) * Ks + k;
            *u = make_float2(u->x * f, u->y * f);
        } else {
            const long long q = e - nua;
            const int k = (int)(q % Ks), r = (int)(q / ((long long)J * Ks));
            const double f = (double)s[(size_t)r * Ks + k];
            double2 *v = RU + q;
            *v = make_double2(v->x * f * f, v->y * f * f);
        }
    }
}

struct MatchReq { int iref, slot, irot, pad; };

__global__ void __launch_bounds__(MF_THREADS) k_prep_matchfilt(Geom g, const MatchReq *__restrict__ reqs,
                                                               const float2 *__restrict__ refs_even,
                                                               const float2 *__restrict__ refs_odd,
                                                               const float *__restrict__ ctfmats,
                                                               const uint8_t *__restrict__ iseven,
                                                               const float *__restrict__ optlp, float2 *__restrict__ ptcls,
                                                               float *__restrict__ sqsums)
{
    extern __shared__ double mfs[];   // 6 arrays of Ks
    __shared__ double red[MF_THREADS / 32];
    const MatchReq rq = reqs[blockIdx.x];
    const int P = g.P, N = g.N, Ks = g.Ks;
    double *pwq = mfs, *pwr = mfs + Ks, *dif = mfs + 2 * Ks, *fit = mfs + 3 * Ks, *wq = mfs + 4 * Ks, *wr = mfs + 5 * Ks;
    float2 *q = ptcls + (size_t)rq.slot * g.K * P;
    const float2 *r = (iseven[rq.slot] ? refs_even : refs_odd) + (size_t)rq.iref * g.K * P;
    const float *ctf = ctfmats ? ctfmats + (size_t)rq.slot * g.K * P : nullptr;
    const float *o = optlp + (size_t)rq.iref * Ks;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // powers of the particle and of the reference times |CTF|, one warp per shell
    for (int k = warp; k < Ks; k += MF_THREADS / 32) {
        double sq = 0.0, sr = 0.0;
        for (int n = lane; n < P; n += 32) {
            const float2 a = q[(size_t)k * P + n], b = r[(size_t)k * P + n];
            const double c = ctf ? (double)ctf[(size_t)k * P + n] : 1.0;
            sq += (double)a.x * a.x + (double)a.y * a.y;
            sr += c * c * ((double)b.x * b.x + (double)b.y * b.y);
        }
        for (int s = 16; s > 0; s >>= 1) {
            sq += __shfl_xor_sync(0xffffffffu, sq, s);
            sr += __shfl_xor_sync(0xffffffffu, sr, s);
        }
        if (lane == 0) {
            const double pq = sq / P, pr = sr / P, ok = (double)o[k];
            wq[k] = pq > 1e-12 ? ok / sqrt(pq) : ok;
            wr[k] = pr > 1e-12 ? ok / sqrt(pr) : ok;
            pwq[k] = pq * wq[k] * wq[k];   // powers after the normalisation
            pwr[k] = pr * wr[k] * wr[k];
        }
    }
    __syncthreads();
    // the difference power at irot: wr ref(n) c(n) - wq ptcl~(n + irot - 1)
    for (int k = warp; k < Ks; k += MF_THREADS / 32) {
        double d = 0.0;
        for (int n = lane; n < P; n += 32) {
            int j = n + rq.irot - 1;
            if (j >= N) j -= N;
            const int jp = j < P ? j : j - P;
            const float2 a = q[(size_t)k * P + jp], b = r[(size_t)k * P + n];
            const double c = ctf ? (double)ctf[(size_t)k * P + n] : 1.0;
            const double qr = wq[k] * a.x, qi = wq[k] * (j < P ? a.y : -a.y);
            const double dr = wr[k] * c * b.x - qr, di = wr[k] * c * b.y - qi;
            d += dr * dr + di * di;
        }
        for (int s = 16; s > 0; s >>= 1) d += __shfl_xor_sync(0xffffffffu, d, s);
        if (lane == 0) dif[k] = d / P;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // Savitzky & Golay 7-point quartic smoothing, c_{-3..3} = (5, -30, 75, 131, 75, -30, 5) / 231
        const double c[7] = {5.0 / 231.0, -30.0 / 231.0, 75.0 / 231.0, 131.0 / 231.0, 75.0 / 231.0, -30.0 / 231.0,
                             5.0 / 231.0};
        for (int k = 0; k < Ks; ++k) {
            double v = dif[k];
            if (k < Ks - 3) {
                v = 0.0;
                for (int t = -3; t <= 3; ++t)
                    if (k + t >= 0) v += c[t + 3] * dif[k + t];
            }
            fit[k] = v <= 0.0 || k < 3 ? dif[k] : v;
        }
        for (int k = 0; k < Ks; ++k) {
            double w = pwq[k] > 1e-12 ? 1.0 / sqrt(pwq[k]) : 1.0;
            if (fit[k] > 1e-12) {
                const double ssnr = pwr[k] / fit[k];
                w *= sqrt(ssnr / (ssnr + 1.0));
            }
            wq[k] *= w;   // the particle's total factor
        }
    }
    __syncthreads();
    double s = 0.0;
    for (int e = threadIdx.x; e < Ks * P; e += blockDim.x) {
        const float f = (float)wq[e / P];
        float2 v = q[e];
        v = make_float2(v.x * f, v.y * f);
        q[e] = v;
        s += (double)v.x * v.x + (double)v.y * v.y;
    }
    s = mf_block_sum(s, red);
    if (threadIdx.x == 0) sqsums[rq.slot] = (float)s;
}

// calc_ptcl_pspec (:897-904): sum_n |ptcl(n,k)|^2 / P for every shell kfrom..kto, a warp per shell
__global__ void __launch_bounds__(MF_THREADS) k_ptcl_pspec(Geom g, const float2 *__restrict__ ptcls, int slot,
                                                           float *__restrict__ pspec)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const float2 *q = ptcls + (size_t)slot * g.K * g.P;
    for (int k = warp; k < g.K; k += MF_THREADS / 32) {
        double s = 0.0;
        for (int n = lane; n < g.P; n += 32) {
            const float2 v = q[(size_t)k * g.P + n];
            s += (double)v.x * v.x + (double)v.y * v.y;
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) pspec[k] = (float)(s / g.P);
    }
}

cudaError_t launch_ptcl_pspec(pftcc_handle *h, int slot, float *pspec_dev)
{
    PFTCC_LAUNCH(h);
    k_ptcl_pspec<<<1, MF_THREADS, 0, h->stream>>>(h->g, h->ptcls, slot, pspec_dev);
    return cudaGetLastError();
}

cudaError_t launch_shellnorm(pftcc_handle *h, int r0, int n)
{
    if (n <= 0) return cudaSuccess;
    PFTCC_LAUNCH(h);
    k_shellnorm<<<2 * n, MF_THREADS, (size_t)h->g.Ks * sizeof(double), h->stream>>>(
        h->g, h->refs_even, h->refs_odd, h->d_optlp, h->nrefs, r0, n, h->pssnr, h->d_snorm);
    return cudaGetLastError();
}

cudaError_t launch_shellnorm_apply(pftcc_handle *h, int M, int nrs, int rows_pad, int nshifts, int set, float2 *UA,
                                   double2 *RU)
{
    const Geom &g = h->g;
    const int J = g.P / 2 + 1;
    const long long tot = (long long)M * nrs * g.Ks + (long long)h->nrefs * J * g.Ks;
    PFTCC_LAUNCH(h);
    k_shellnorm_apply<<<(int)std::min<long long>((tot + 255) / 256, 8192), 256, 0, h->stream>>>(
        M, g.Ks, J, nrs, rows_pad, nshifts, h->nrefs, h->d_snorm + (size_t)set * h->nrefs * g.Ks, UA, RU);
    return cudaGetLastError();
}

cudaError_t launch_prep_matchfilt(pftcc_handle *h, const void *reqs_dev, int nreq)
{
    if (nreq <= 0) return cudaSuccess;
    const float *ctf = (h->cfg.with_ctf && h->ctf_ready) ? h->ctfmats : nullptr;
    static_assert(sizeof(MatchReq) == sizeof(int4), "request layout");
    if (h->pssnr) {
        PFTCC_LAUNCH(h);
        k_prep_pssnr<<<nreq, MF_THREADS, (size_t)h->g.Ks * sizeof(double), h->stream>>>(
            h->g, static_cast<const int4 *>(reqs_dev), ctf, h->d_optlp, h->ptcls, h->sqsums);
        return cudaGetLastError();
    }
    PFTCC_LAUNCH(h);
    k_prep_matchfilt<<<nreq, MF_THREADS, (size_t)6 * h->g.Ks * sizeof(double), h->stream>>>(h->g, static_cast<const MatchReq *>(reqs_dev), h->refs_even,
                                                         h->refs_odd, ctf, h->d_iseven, h->d_optlp, h->ptcls,
                                                         h->sqsums);
    return cudaGetLastError();
}

}  // namespace pftcc
