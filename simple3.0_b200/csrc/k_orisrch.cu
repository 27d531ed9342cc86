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
// calc_T1_T2_for_rot_8 as the particle slot, :1781 / :1836, which names that particle only
// when the two indices coincide).  One block per request, threads over the polar angles.
#include "pftcc_internal.cuh"
#include "lbfgsb.h"

#include <cmath>
#include <vector>

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
    int scratch, const float *__restrict__ snorm, int nrefs,
    double *__restrict__ out6 /* [nreq][6]: f, d/de1, d/de2, d/de3, d/dsx, d/dsy */)
{
    __shared__ double red[OG_THREADS / 32];
    const EuclidReq rq = reqs[blockIdx.x];
    const int N = g.N, P = g.P, K = g.K;
    const bool ev = iseven[rq.slot] != 0;
    const float2 *q = ptcls + (long long)rq.slot * K * P;
    // scratch: request b's own section and derivatives at refs_even / drefs_even + b
    const float2 *r = scratch ? refs_even + (long long)blockIdx.x * K * P
                              : (ev ? refs_even : refs_odd) + (long long)rq.iref * K * P;
    const float2 *dr = scratch ? drefs_even + (long long)blockIdx.x * 3 * K * P
                               : (ev ? drefs_even : drefs_odd) + (long long)rq.iref * 3 * K * P;
    const float *ctf = ctfmats ? ctfmats + (long long)rq.slot * K * P : nullptr;
    // matched-filter mode: the reference (not its derivatives) shell-normalised, as
    // gencorr_cont_shift_grad_cc_for_rot_8 applies shellnorm_and_filter_ref_8 to pft_ref alone
    const float *sn = (snorm && !scratch) ? snorm + ((size_t)(ev ? 0 : 1) * nrefs + rq.iref) * g.Ks : nullptr;
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
            const double f = sn ? (double)sn[ik] : 1.0;
            const double rr = (double)rv.x * f * c, ri = (double)rv.y * f * c;
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
                                                          h->argtransf, h->argtransf1, 0, snorm_ptr(h), h->nrefs, out6);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// pftcc_orisrch_grad%minimize (simple_pftcc_orisrch_grad.f90:60-122) for n particles at once:
// variables (e1, e2, e3 in degrees, sx, sy), box e +- angerr_deg and |s| <= maxHWshift, start
// (e_in, 0, 0), cost -corr and gradient -grad of gencorr_cont_shift_grad_cc_for_rot_8 at
// irot = 1 on the sections fdf_project_polar makes at the trial angles (fdfcostfun :178-207).
// The gradient's angle components are per radian while the variables are degrees, as the
// reference pairs them.  Every round, the pending trial points of all unfinished problems are
// projected by ONE k_fdf_project_polar launch into per-request scratch sections and scored by
// ONE k_cont_shift_grad launch.  A problem whose final cost is not below its starting cost keeps
// its angles and returns a zero shift (:101-117); the shift found is rotated into the reference
// frame by rotmat2d(e3) (:106-109).
static int orisrch_eval(pftcc_handle *h, int nb, const int *slots, const double *xt, double *f, double *g5,
                        float2 *scr_ref, float2 *scr_dref, double *dRD, EuclidReq *dreq, double *dout,
                        std::vector<double> &RD, std::vector<EuclidReq> &rq, std::vector<double> &o)
{
    RD.resize((size_t)nb * 36);
    rq.resize(nb);
    for (int b = 0; b < nb; ++b) {
        host_euler2m(&xt[5 * b], &RD[(size_t)b * 36], &RD[(size_t)b * 36 + 9]);
        rq[b] = EuclidReq{0, slots[b], 1, 0, xt[5 * b + 3], xt[5 * b + 4]};
    }
    cudaError_t e = cudaMemcpyAsync(dRD, RD.data(), RD.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dreq, rq.data(), (size_t)nb * sizeof(EuclidReq), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = launch_fdf_project_polar(h, h->vol_box, h->vol_cube, dRD, nb, scr_ref, scr_dref);
    if (e == cudaSuccess) {
        const float *ctf = (h->cfg.with_ctf && h->ctf_ready) ? h->ctfmats : nullptr;
        PFTCC_LAUNCH(h);
        KTimer kt(h, PFTCC_K_EXACT);
        k_cont_shift_grad<<<nb, OG_THREADS, 0, h->stream>>>(h->g, dreq, scr_ref, scr_ref, scr_dref, scr_dref,
                                                             h->ptcls, ctf, h->d_iseven, h->sqsums, h->argtransf,
                                                             h->argtransf1, 1, nullptr, 0, dout);
        e = cudaGetLastError();
    }
    o.resize((size_t)nb * 6);
    if (e == cudaSuccess) e = cudaMemcpyAsync(o.data(), dout, o.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "orisrch evaluation");
    for (int b = 0; b < nb; ++b) {
        f[b] = -o[6 * (size_t)b];
        for (int v = 0; v < 5; ++v) g5[5 * (size_t)b + v] = -o[6 * (size_t)b + 1 + v];
    }
    return PFTCC_OK;
}

int orisrch_batch(pftcc_handle *h, int n, const pftcc_orisrch_req *req, int maxits, double pgtol, double factr,
                  pftcc_orisrch_out *out)
{
    constexpr int NV = 5;
    std::vector<int> slot(n);
    std::vector<double> x0((size_t)n * NV), lb((size_t)n * NV), ub((size_t)n * NV);
    for (int i = 0; i < n; ++i) {
        slot[i] = -1;
        if (req[i].iptcl >= h->pfrom && req[i].iptcl <= h->pto) slot[i] = h->pinds[req[i].iptcl - h->pfrom] - 1;
        if (slot[i] < 0) return set_err(h, PFTCC_ERR_INDEX, "orisrch: particle not held");
        for (int v = 0; v < 3; ++v) {
            x0[(size_t)i * NV + v] = req[i].e[v];
            lb[(size_t)i * NV + v] = req[i].e[v] - req[i].angerr_deg;
            ub[(size_t)i * NV + v] = req[i].e[v] + req[i].angerr_deg;
        }
        for (int v = 3; v < 5; ++v) {
            x0[(size_t)i * NV + v] = 0.0;
            lb[(size_t)i * NV + v] = -req[i].maxhwshift;
            ub[(size_t)i * NV + v] = req[i].maxhwshift;
        }
    }
    // scratch for the largest round: n sections, their derivatives, matrices, requests, results
    const size_t KP = (size_t)h->g.K * h->g.P;
    float2 *scr = nullptr;
    double *dRD = nullptr, *dout = nullptr;
    EuclidReq *dreq = nullptr;
    int st = dev_alloc(h, (void **)&scr, (size_t)n * 4 * KP * sizeof(float2), "orisrch sections");
    if (st == PFTCC_OK) st = dev_alloc(h, (void **)&dRD, (size_t)n * 36 * sizeof(double), "orisrch matrices");
    if (st == PFTCC_OK) st = dev_alloc(h, (void **)&dreq, (size_t)n * sizeof(EuclidReq), "orisrch requests");
    if (st == PFTCC_OK) st = dev_alloc(h, (void **)&dout, (size_t)n * 6 * sizeof(double), "orisrch results");
    std::vector<double> f0(n, 0.0);
    std::vector<char> have_f0(n, 0);
    if (st == PFTCC_OK) {
        std::vector<int> sl;
        std::vector<double> RD, o;
        std::vector<EuclidReq> rq;
        auto eval = [&](int nb, const int *idx, const double *xt, double *f, double *g) -> int {
            sl.resize(nb);
            for (int b = 0; b < nb; ++b) sl[b] = slot[idx[b]];
            const int s2 = orisrch_eval(h, nb, sl.data(), xt, f, g, scr, scr + (size_t)n * KP, dRD, dreq, dout, RD,
                                        rq, o);
            if (s2 != PFTCC_OK) return s2;
            for (int b = 0; b < nb; ++b)
                if (!have_f0[idx[b]]) { have_f0[idx[b]] = 1; f0[idx[b]] = f[b]; }
            return 0;
        };
        std::vector<lbfgsb::Result<NV>> res(n);
        st = lbfgsb::minimize_batch(n, x0.data(), lb.data(), ub.data(), maxits, pgtol, factr, eval, res.data());
        if (st == PFTCC_OK) {
            for (int i = 0; i < n; ++i) {
                pftcc_orisrch_out &q = out[i];
                const bool better = res[i].f < f0[i];
                q.found_better = better ? 1 : 0;
                q.corr = better ? -res[i].f : -f0[i];
                q.corr_init = -f0[i];
                for (int v = 0; v < 3; ++v) q.e[v] = better ? res[i].x[v] : req[i].e[v];
                q.shift[0] = q.shift[1] = 0.0;
                if (better) {   // cxy(2:) = matmul(x(4:5), rotmat2d(x(3))), rotmat2d = [c s; -s c]
                    const double a = res[i].x[2] * 3.14159265358979323846 / 180.0, c = std::cos(a), sn = std::sin(a);
                    q.shift[0] = res[i].x[3] * c - res[i].x[4] * sn;
                    q.shift[1] = res[i].x[3] * sn + res[i].x[4] * c;
                }
                q.nevals = res[i].nevals;
                q.niter = res[i].niter;
                q.converged = res[i].converged;
                q.pad = 0;
            }
        }
    }
    dev_free(h, scr);
    dev_free(h, dRD);
    dev_free(h, dreq);
    dev_free(h, dout);
    return st;
}

}  // namespace pftcc
