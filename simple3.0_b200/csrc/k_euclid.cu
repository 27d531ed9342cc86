// k_euclid.cu -- the Euclidean objective at one rotation, reference frame, FP64
// (simple_polarft_corrcalc.f90): gencorr_euclid_for_rot(_8) :2002-2048 with
// calc_euclid_for_rot(_8) :1280-1334, gencorr_euclid_grad_for_rot_8 / _grad_only_ :2071-2148,
// gencorr_sigma_contrib :2150-2188 with calc_euclidk_for_rot :1392-1415.
//
// The reference is prepared as ref * ctf * shmat (shmat by gen_shmat_8's recurrence: the
// first shell's phases analytic, each later shell the previous one times the shell-one
// phase vector) and the particle extended over the full circle, ptcl~(j + P) = conj(ptcl(j)).
// With d(n, k) = ref_prep(n, k) - ptcl~(n + irot - 1, k) and w(k) = k pxls(k) / (P sigma2(k)):
//   f      = -sum_{k<=kstop} w(k) sum_n |d|^2 / 2
//   grad_x =  sum_{k<=kstop} w(k) (Re sum_n T(n) conj(ptcl~) - Re sum_n T(n) conj(ref_prep)),
//             T = i argtransf_x ref_prep (argtransf_y for grad_y)
//   shells =  per shell k = kfrom..kto: sum_n |d|^2 / (2P), sum_n |ptcl|^2, sum_n |ref_prep|^2
// One block per request, threads over the polar angles n, each thread walking the shells;
// the per-shell sums meet in shared FP64 accumulators.
#include "pftcc_internal.cuh"

namespace pftcc {

constexpr int EU_THREADS = 256;

__device__ __forceinline__ double eu_block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < EU_THREADS / 32; ++w) t += red[w];
    return t;
}

__global__ void __launch_bounds__(EU_THREADS) k_euclid_rot(
    Geom g, const EuclidReq *__restrict__ reqs, const float2 *__restrict__ refs_even,
    const float2 *__restrict__ refs_odd, const float2 *__restrict__ ptcls, const float *__restrict__ ctfmats,
    const uint8_t *__restrict__ iseven, const double *__restrict__ argtransf, const double *__restrict__ argtransf1,
    const float *__restrict__ sig2, const float *__restrict__ pxls, int want_shells, double *__restrict__ out3,
    double *__restrict__ shells)
{
    extern __shared__ double shk[];   // [3][K] when want_shells
    __shared__ double red[EU_THREADS / 32];
    const EuclidReq rq = reqs[blockIdx.x];
    const int N = g.N, P = g.P, K = g.K;
    if (want_shells)
        for (int e = threadIdx.x; e < 3 * K; e += blockDim.x) shk[e] = 0.0;
    __syncthreads();
    const float2 *q = ptcls + (long long)rq.slot * K * P;
    const float2 *r = (iseven[rq.slot] ? refs_even : refs_odd) + (long long)rq.iref * K * P;
    const float *ctf = ctfmats ? ctfmats + (long long)rq.slot * K * P : nullptr;
    const float *sg = sig2 ? sig2 + (long long)rq.slot * K : nullptr;
    const int s = rq.irot - 1;
    const int kend = want_shells ? K : g.Ks;
    double f = 0.0, gx = 0.0, gy = 0.0;
    for (int n = threadIdx.x; n < P; n += blockDim.x) {
        double st_r, st_i, v_r, v_i;
        sincos(argtransf[n] * rq.sx + argtransf[P + n] * rq.sy, &st_i, &st_r);
        sincos(argtransf1[n] * rq.sx + argtransf1[P + n] * rq.sy, &v_i, &v_r);
        int j = s + n;
        if (j >= N) j -= N;
        const int jp = j < P ? j : j - P;
        const double qs = j < P ? 1.0 : -1.0;
        for (int ik = 0; ik < kend; ++ik) {
            const double c = ctf ? (double)ctf[ik * P + n] : 1.0;
            const float2 rv = r[(long long)ik * P + n];
            const double rr = (double)rv.x * c, ri = (double)rv.y * c;
            const double ar = rr * st_r - ri * st_i, ai = rr * st_i + ri * st_r;   // prepared reference
            const float2 qv = q[(long long)ik * P + jp];
            const double qr = qv.x, qi = qs * qv.y;                                // ptcl~(j)
            const double dr = ar - qr, di = ai - qi, d2 = dr * dr + di * di;
            if (sg && ik < g.Ks) {
                const double wk = (double)(g.kfrom + ik) * (double)pxls[ik] / ((double)P * (double)sg[ik]);
                f -= 0.5 * wk * d2;
                const double ax = argtransf[ik * N + n], ay = argtransf[ik * N + P + n];
                // T = i a A = (-a ai, a ar): Re T conj(ptcl~) - Re T conj(A)
                gx += wk * ((-ax * ai * qr + ax * ar * qi) - (-ax * ai * ar + ax * ar * ai));
                gy += wk * ((-ay * ai * qr + ay * ar * qi) - (-ay * ai * ar + ay * ar * ai));
            }
            if (want_shells) {
                atomicAdd(&shk[ik], d2);
                atomicAdd(&shk[K + ik], (double)qv.x * qv.x + (double)qv.y * qv.y);
                atomicAdd(&shk[2 * K + ik], ar * ar + ai * ai);
            }
            const double nr = st_r * v_r - st_i * v_i, ni = st_r * v_i + st_i * v_r;
            st_r = nr;
            st_i = ni;
        }
    }
    f = eu_block_sum(f, red);
    gx = eu_block_sum(gx, red);
    gy = eu_block_sum(gy, red);
    if (threadIdx.x == 0 && out3) {
        out3[3 * blockIdx.x] = f;
        out3[3 * blockIdx.x + 1] = gx;
        out3[3 * blockIdx.x + 2] = gy;
    }
    if (want_shells) {
        const double half_over_p = 0.5 / (double)P;
        for (int e = threadIdx.x; e < 3 * K; e += blockDim.x)
            shells[(long long)blockIdx.x * 3 * K + e] = e < K ? shk[e] * half_over_p : shk[e];
    }
}

cudaError_t launch_euclid_rot(pftcc_handle *h, const EuclidReq *reqs_dev, int nreq, int with_f, int want_shells,
                              double *out3, double *shells)
{
    if (nreq <= 0) return cudaSuccess;
    const size_t smem = want_shells ? (size_t)3 * h->g.K * sizeof(double) : 0;
    cudaError_t e = smem_limit((const void *)k_euclid_rot, smem);
    if (e != cudaSuccess) return e;
    const float *ctf = (h->cfg.with_ctf && h->ctf_ready) ? h->ctfmats : nullptr;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_EXACT);
    k_euclid_rot<<<nreq, EU_THREADS, smem, h->stream>>>(h->g, reqs_dev, h->refs_even, h->refs_odd, h->ptcls, ctf,
                                                        h->d_iseven, h->argtransf, h->argtransf1,
                                                        with_f ? h->d_sig2 : nullptr, h->d_pxls, want_shells,
                                                        out3, shells);
    return cudaGetLastError();
}

}  // namespace pftcc
