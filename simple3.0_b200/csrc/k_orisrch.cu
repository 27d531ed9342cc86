// k_orisrch.cu -- the orientation-gradient correlator, reference frame, FP64:
// gencorr_cont_shift_grad_cc_for_rot_8 (simple_polarft_corrcalc.f90:1788-1847) and
// gencorr_cont_grad_cc_for_rot_8 (:1735-1786) with calc_T1_T2_for_rot_8 (:1246-1278).
//
// With A = ref * ctf * shmat and dA_j = dref_j * ctf * shmat (the derivative references of
// fdf_project_polar, j = e1, e2, e3), ptcl~ the particle extended over the full circle and sums
// over the shells kfrom..kstop:
//   y = Re sum_n A(n) conj(ptcl~(n + irot - 1)),  S = sum |A|^2,  den = sqrt(S * sqsum_ptcl)
//   T1_j = Re sum_n dA_j(n) conj(ptcl~(n + irot - 1)),  T2_j = Re sum_n dA_j(n) conj(A(n))
//   f = y / den,  grad_j = (T1_j - y T2_j / S) / den,
//   grad_{4,5} = Re sum_n (i argtransf_{x,y} A)(n) conj(ptcl~(n + irot - 1)) / den.
// T1 correlates with the particle being scored (the reference passes iref to
// calc_T1_T2_for_rot_8 as the particle slot, :1776 / :1831, which names that particle only
// when the two indices coincide).  One block per request, threads over the polar angles.
#include "pftcc_internal.cuh"

namespace pftcc {

constexpr int OG_THREADS = 256;

__device__ __forceinline__ double og_block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < OG_THREADS / 32; ++w) t += red[w];
    return t;
}

__global__ void __launch_bounds__(OG_THREADS) k_cont_shift_grad(
    Geom g, const EuclidReq *__restrict__ reqs, const float2 *__restrict__ refs_even,
    const float2 *__restrict__ refs_odd, const float2 *__restrict__ drefs_even, const float2 *__restrict__ drefs_odd,
    const float2 *__restrict__ ptcls, const float *__restrict__ ctfmats, const uint8_t *__restrict__ iseven,
    const float *__restrict__ sqsums, const double *__restrict__ argtransf, const double *__restrict__ argtransf1,
    double *__restrict__ out6 /* [nreq][6]: f, d/de1, d/de2, d/de3, d/dsx, d/dsy */)
{
    __shared__ double red[OG_THREADS / 32];
    const EuclidReq rq = reqs[blockIdx.x];
    const int N = g.N, P = g.P, K = g.K;
    const bool ev = iseven[rq.slot] != 0;
    const float2 *q = ptcls + (long long)rq.slot * K * P;
    const float2 *r = (ev ? refs_even : refs_odd) + (long long)rq.iref * K * P;
    const float2 *dr = (ev ? drefs_even : drefs_odd) + (long long)rq.iref * 3 * K * P;
    const float *ctf = ctfmats ? ctfmats + (long long)rq.slot * K * P : nullptr;
    const int s = rq.irot - 1;
    double y = 0.0, sqr = 0.0, gx = 0.0, gy = 0.0, t1[3] = {0.0, 0.0, 0.0}, t2[3] = {0.0, 0.0, 0.0};
    for (int n = threadIdx.x; n < P; n += blockDim.x) {
        double st_r, st_i, v_r, v_i;
        sincos(argtransf[n] * rq.sx + argtransf[P + n] * rq.sy, &st_i, &st_r);
        sincos(argtransf1[n] * rq.sx + argtransf1[P + n] * rq.sy, &v_i, &v_r);
        int j = s + n;
        if (j >= N) j -= N;
        const int jp = j < P ? j : j - P;
        const double qs = j < P ? 1.0 : -1.0;
        for (int ik = 0; ik < g.Ks; ++ik) {
            const double c = ctf ? (double)ctf[ik * P + n] : 1.0;
            const float2 rv = r[(long long)ik * P + n];
            const double rr = (double)rv.x * c, ri = (double)rv.y * c;
            const double ar = rr * st_r - ri * st_i, ai = rr * st_i + ri * st_r;
            const float2 qv = q[(long long)ik * P + jp];
            const double qr = qv.x, qi = qs * qv.y;
            y += ar * qr + ai * qi;
            sqr += ar * ar + ai * ai;
            const double ax = argtransf[ik * N + n], ay = argtransf[ik * N + P + n];
            gx += ax * (-ai * qr + ar * qi);
            gy += ay * (-ai * qr + ar * qi);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float2 dv = dr[((long long)d * K + ik) * P + n];
                const double pr = (double)dv.x * c, pi = (double)dv.y * c;
                const double br = pr * st_r - pi * st_i, bi = pr * st_i + pi * st_r;
                t1[d] += br * qr + bi * qi;
                t2[d] += br * ar + bi * ai;
            }
            const double nr = st_r * v_r - st_i * v_i, ni = st_r * v_i + st_i * v_r;
            st_r = nr;
            st_i = ni;
        }
    }
    y = og_block_sum(y, red);
    sqr = og_block_sum(sqr, red);
    gx = og_block_sum(gx, red);
    gy = og_block_sum(gy, red);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        t1[d] = og_block_sum(t1[d], red);
        t2[d] = og_block_sum(t2[d], red);
    }
    if (threadIdx.x == 0) {
        const double den = sqrt(sqr * (double)sqsums[rq.slot]);
        double *o = out6 + 6 * blockIdx.x;
        o[0] = y / den;
#pragma unroll
        for (int d = 0; d < 3; ++d) o[1 + d] = (t1[d] - y * t2[d] / sqr) / den;
        o[4] = gx / den;
        o[5] = gy / den;
    }
}

cudaError_t launch_cont_shift_grad(pftcc_handle *h, const EuclidReq *reqs_dev, int nreq, double *out6)
{
    if (nreq <= 0) return cudaSuccess;
    if (!h->drefs_even || !h->drefs_odd) return cudaErrorInvalidValue;
    const float *ctf = (h->cfg.with_ctf && h->ctf_ready) ? h->ctfmats : nullptr;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_EXACT);
    k_cont_shift_grad<<<nreq, OG_THREADS, 0, h->stream>>>(h->g, reqs_dev, h->refs_even, h->refs_odd, h->drefs_even,
                                                          h->drefs_odd, h->ptcls, ctf, h->d_iseven, h->sqsums,
                                                          h->argtransf, h->argtransf1, out6);
    return cudaGetLastError();
}

}  // namespace pftcc
