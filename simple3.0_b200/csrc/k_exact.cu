// k_exact.cu -- gridding, CTF matrices and the exact FP32 correlation kernels.
//
// The exact kernels evaluate the reference's correlation sums directly,
//   corr(irot) = Re sum_k sum_n pft_ref(n,k) * conj(ptcl~(n + irot - 1, k))
// (calc_corr_for_rot, simple_polarft_corrcalc.f90:1190-1216, with ptcl~ the
// particle extended over the full circle by conjugate symmetry), for every
// rotation at once, with the reference prepared exactly as gencorrs_cc_1/_2 do
// (prep_ref4corr :961-985, gen_shmat_8 :1098-1120, :1526-1531).
#include "pftcc_internal.cuh"

#include <cstddef>
#include <cmath>

namespace pftcc {

// ---------------------------------------------------------------------------
// polarize: pft(i,k) = sum_taps w * F(h,k) with the Hermitian half-plane gather
// (simple_polarizer.f90:120-151, simple_image.f90:1894-1907).  One block per image:
// the whole half-plane FT is staged into shared memory with coalesced 16-byte loads,
// then every (irot, k) sample gathers its 9 taps from shared memory.  Tap tables
// (offsets, with the conjugation flag as a bitwise complement, and weights) come
// from init_polarizer and live in L2.  The particle square sum over kfrom..kstop
// (memoize_sqsum_ptcl :841-845) is reduced in the same kernel.
__global__ void __launch_bounds__(256) k_polarize(Geom g, const float2 *__restrict__ cmats, long long img_elems,
                                                   const int *__restrict__ tap_off, const float *__restrict__ tap_w,
                                                   float2 *__restrict__ out, float *__restrict__ sqsums)
{
    extern __shared__ float4 smem4[];
    float2 *img = reinterpret_cast<float2 *>(smem4);
    __shared__ float red[32];
    const int i = blockIdx.x;
    const float2 *src = cmats + (long long)i * img_elems;
    // stage the image: img_elems float2 = img_elems/2 float4 (img_elems is even for even box)
    const float4 *src4 = reinterpret_cast<const float4 *>(src);
    for (long long e = threadIdx.x; e < img_elems / 2; e += blockDim.x) smem4[e] = __ldg(src4 + e);
    __syncthreads();
    const int npts = g.K * g.P;
    float2 *dst = out + (long long)i * npts;
    float sq = 0.f;
    for (int e = threadIdx.x; e < npts; e += blockDim.x) {
        const int *o = tap_off + e * 9;
        const float *w = tap_w + e * 9;
        float ar = 0.f, ai = 0.f;
#pragma unroll
        for (int t = 0; t < 9; ++t) {
            const int off = o[t];
            const float2 v = img[off >= 0 ? off : ~off];
            const float vi = off >= 0 ? v.y : -v.y;
            ar = fmaf(w[t], v.x, ar);
            ai = fmaf(w[t], vi, ai);
        }
        dst[e] = make_float2(ar, ai);
        if (e / g.P < g.Ks) sq += ar * ar + ai * ai;
    }
    // block reduction of the square sum
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0 && sqsums) sqsums[i] = v;
    }
}

cudaError_t launch_polarize(pftcc_handle *h, const float2 *cmats, int n, int first_slot)
{
    const Geom &g = h->g;
    const long long img_elems = (long long)g.box * (g.box / 2 + 1);
    const size_t smem = (size_t)img_elems * sizeof(float2);
    cudaError_t e = smem_limit((const void *)k_polarize, smem);
    if (e != cudaSuccess) return e;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_POLARIZE);
    k_polarize<<<n, 256, smem, h->stream>>>(g, cmats, img_elems, h->pol_off, h->pol_w,
                                           h->ptcls + (size_t)first_slot * g.K * g.P, h->sqsums + first_slot);
    return cudaGetLastError();
}

// square sums of particles set directly (set_ptcl_pft -> memoize_sqsum_ptcl :841-845)
__global__ void k_sqsums(Geom g, const float2 *__restrict__ ptcls, float *__restrict__ sqsums)
{
    __shared__ float red[32];
    const float2 *p = ptcls + (long long)blockIdx.x * g.K * g.P;
    float sq = 0.f;
    for (int e = threadIdx.x; e < g.Ks * g.P; e += blockDim.x) {
        const float2 v = p[e];
        sq += v.x * v.x + v.y * v.y;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_xor_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x < 32) {
        float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (threadIdx.x == 0) sqsums[blockIdx.x] = v;
    }
}

cudaError_t launch_sqsums(pftcc_handle *h, int first_slot, int n)
{
    PFTCC_LAUNCH(h);
    k_sqsums<<<n, 256, 0, h->stream>>>(h->g, h->ptcls + (size_t)first_slot * h->g.K * h->g.P, h->sqsums + first_slot);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// |CTF| on the polar grid in single precision, following the reference's
// arithmetic: create_polar_absctfmats :926-935 (spaFreqSq from polar * 1/ldim,
// ang = atan2(y, x)), simple_ctf.f90 constructor :54-70, init :73-81,
// evalPhSh :88-98, eval_df :185-189, kV2wl :522-525, eval :147-153 / :154-160.
// derivative != 0 writes d|CTF|/d(defocus[micron]) (dfx and dfy moved together).
__device__ __forceinline__ float ctf_abs_f(const pftcc_ctfparams &c, float spafreqsq, float ang, float ddf,
                                           int derivative)
{
    const float kv = 1000.0f * c.kv;
    const float wl = (12.26f / sqrtf(kv + (0.9784f * kv * kv) / 1.0e6f)) / c.smpd;
    const float cs = (c.cs * 1.0e7f) / c.smpd;
    const float phaseq = sqrtf(1.0f - c.fraca * c.fraca);
    const float ampc = atanf(c.fraca / phaseq);
    const float dfx = ((c.dfx + ddf) * 1.0e4f) / c.smpd;
    const float dfy = ((c.dfy + ddf) * 1.0e4f) / c.smpd;
    const float angast = (c.angast / 180.0f) * 3.14159265358979f;
    const float df = 0.5f * (dfx + dfy + cosf(2.0f * (ang - angast)) * (dfx - dfy));
    const float pi = 3.14159265358979f;
    float chi = pi * wl * spafreqsq * (df - 0.5f * wl * wl * spafreqsq * cs);
    if (c.l_phaseplate) chi += c.phshift;
    chi += ampc;
    const float s = sinf(chi);
    if (!derivative) return fabsf(s);
    const float dchi = pi * wl * spafreqsq * (1.0e4f / c.smpd);
    return (s >= 0.f ? 1.f : -1.f) * cosf(chi) * dchi;
}

__global__ void k_ctfmat(Geom g, const float *__restrict__ polar, const pftcc_ctfparams *__restrict__ params,
                         float *__restrict__ out, float ddf, int derivative)
{
    const int i = blockIdx.y;
    const pftcc_ctfparams c = params[i];
    const float inv_ldim = 1.0f / (float)g.box;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < g.K * g.P; e += gridDim.x * blockDim.x) {
        const int ik = e / g.P, irot = e - ik * g.P;
        const float x = polar[ik * 2 * g.N + irot], y = polar[ik * 2 * g.N + g.N + irot];
        const float hinv = x * inv_ldim, kinv = y * inv_ldim;
        const float s2 = hinv * hinv + kinv * kinv;
        const float ang = atan2f(y, x);
        out[(long long)i * g.K * g.P + e] = ctf_abs_f(c, s2, ang, ddf, derivative);
    }
}

cudaError_t launch_ctfmat(pftcc_handle *h, const pftcc_ctfparams *params, int n, float *out, float ddf, int derivative)
{
    const int per = h->g.K * h->g.P;
    dim3 grid((per + 255) / 256, n);
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_CTFMAT);
    k_ctfmat<<<grid, 256, 0, h->stream>>>(h->g, h->polar, params, out, ddf, derivative);
    return cudaGetLastError();
}

// zero_refs_beyond_kstop :747-754
__global__ void k_zero_beyond(Geom g, int nrefs, float2 *even, float2 *odd)
{
    const int nz = (g.K - g.Ks) * g.P;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)nrefs * nz;
         e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / nz, o = e - r * nz;
        const long long idx = r * g.K * g.P + (long long)g.Ks * g.P + o;
        even[idx] = make_float2(0.f, 0.f);
        odd[idx] = make_float2(0.f, 0.f);
    }
}

cudaError_t launch_zero_beyond_kstop(pftcc_handle *h)
{
    if (h->g.K == h->g.Ks) return cudaSuccess;
    PFTCC_LAUNCH(h);
    k_zero_beyond<<<296, 256, 0, h->stream>>>(h->g, h->nrefs, h->refs_even, h->refs_odd);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// exact correlations for a list of (reference, shift) work items per particle.
//
// One block per particle group, 256 threads; thread t owns rotations s = t + 256 r.
// Shells are processed in chunks of KC: the prepared reference A(n,k) and the
// extended particle Qt(j,k), j < N, sit in shared memory; the shift phases follow
// gen_shmat_8 (first shell analytic in double, later shells by the double
// precision de Moivre recurrence, cast to single precision as gen_shmat does).
//
// FRAME_REF:  A = (ref * ctf(n)) * shmat(n), Qt = ptcl~,
//             cc = corr / sqrt(sum|A|^2 * sqsum_ptcl)   (sum over kstop for cc_1,
//             over all shells for cc_2, exactly as the reference)
// FRAME_PTCL: A = ref * shmat(n), Qt = ctf~(j) ptcl~(j),
//             cc = corr / sqrt(sum_n |ref(n)|^2 ctf~(n+s)^2 * sqsum_ptcl)
// FRAME_EUCLID: A and Qt as FRAME_REF, shell weights W(k) = pxls(k) / (P sigma2(k)),
//             euclid = sum_{k<=kstop} W(k) (corr_k - (sum_n |A|^2 + sum_n |ptcl|^2) / 2)
//             (gencorrs_euclid_1/_2 :1536-1592: pxls/P (2 kcorrs - sumsqptcl - sumsqref) / (2 sigma2))
constexpr int EX_THREADS = 256;
__host__ __device__ constexpr size_t al16(size_t b) { return (b + 15) & ~size_t(15); }
constexpr int EX_RPT = 3;      // rotations per thread: N <= 768

template <int FRAME>
__global__ void __launch_bounds__(EX_THREADS) k_exact(
    Geom g, int KC, const float2 *__restrict__ refs_even, const float2 *__restrict__ refs_odd,
    const float2 *__restrict__ ptcls, const float *__restrict__ ctfmats, const uint8_t *__restrict__ iseven,
    const float *__restrict__ sqsums, const double *__restrict__ argtransf, const double *__restrict__ argtransf1,
    const Group *__restrict__ groups, const Work *__restrict__ work, const float *__restrict__ shifts, int mode,
    int cc1_kstop, const float *__restrict__ sig2, const float *__restrict__ pxls, const float *__restrict__ snorm,
    int nrefs, float *__restrict__ out, pftcc_best *__restrict__ best, const uint8_t *__restrict__ rotmask)
{
    extern __shared__ float4 smem4[];
    const int N = g.N, P = g.P;
    // shared layout (16-byte aligned sections, see exact_smem): sh [P] double2 running
    // shmat, sv [P] double2 shell-one phase vector, Qt [KC][N] float2, A [KC][P] float2,
    // then for the particle frame C2t [KC][N] float and R2 [KC][P] float, for the Euclidean
    // objective the shell weights W [K] double in their place
    char *base = reinterpret_cast<char *>(smem4);
    double2 *sh = reinterpret_cast<double2 *>(base);
    double2 *sv = sh + P;
    float2 *Qt = reinterpret_cast<float2 *>(base + al16(2 * P * sizeof(double2)));
    float2 *A = reinterpret_cast<float2 *>(reinterpret_cast<char *>(Qt) + al16(KC * N * sizeof(float2)));
    float *C2t = reinterpret_cast<float *>(reinterpret_cast<char *>(A) + al16(KC * P * sizeof(float2)));
    float *R2 = reinterpret_cast<float *>(reinterpret_cast<char *>(C2t) + al16(KC * N * sizeof(float)));
    double *W = reinterpret_cast<double *>(C2t);
    __shared__ double red[EX_THREADS / 32];
    __shared__ float bcc[EX_THREADS / 32];
    __shared__ int brot[EX_THREADS / 32];

    const Group grp = groups[blockIdx.x];
    const int slot = grp.slot;
    const float2 *q = ptcls + (long long)slot * g.K * P;
    const float *ctf = ctfmats ? ctfmats + (long long)slot * g.K * P : nullptr;
    const float2 *refs = iseven[slot] ? refs_even : refs_odd;
    const float sqp = sqsums[slot];
    if (FRAME == FRAME_EUCLID)   // read after the __syncthreads() that opens the first shell chunk
        for (int ik = threadIdx.x; ik < g.K; ik += blockDim.x)
            W[ik] = (double)pxls[ik] / ((double)P * (double)sig2[(long long)slot * g.K + ik]);
    float run_best = -INFINITY;
    int run_rot = 0, run_item = -1;

    for (int it = 0; it < grp.count; ++it) {
        const Work w = work[grp.first + it];
        const float2 *r = refs + (long long)w.iref * g.K * P;
        const bool has_shift = w.ishift >= 0;
        // matched-filter mode: the reference's shell factors (shellnorm_and_filter_ref), which
        // gencorrs_cc_1/_2 apply and, of the Euclidean pair, gencorrs_euclid_1 alone
        const float *sn = (snorm && (FRAME != FRAME_EUCLID || !has_shift))
                              ? snorm + ((size_t)(iseven[slot] ? 0 : 1) * nrefs + w.iref) * g.Ks
                              : nullptr;
        if (has_shift) {
            const double sx = (double)shifts[2 * w.ishift], sy = (double)shifts[2 * w.ishift + 1];
            for (int n = threadIdx.x; n < P; n += blockDim.x) {
                const double a = argtransf[n] * sx + argtransf[P + n] * sy;
                const double a1 = argtransf1[n] * sx + argtransf1[P + n] * sy;
                double s, c;
                sincos(a, &s, &c);
                sh[n] = make_double2(c, s);
                sincos(a1, &s, &c);
                sv[n] = make_double2(c, s);
            }
        }
        double acc[EX_RPT], dacc[EX_RPT];
#pragma unroll
        for (int u = 0; u < EX_RPT; ++u) { acc[u] = 0.0; dacc[u] = 0.0; }
        double sqr = 0.0;
        const int ksq = (has_shift || !cc1_kstop) ? g.K : g.Ks;   // cc_2 sums all shells, cc_1 to kstop
        for (int k0 = 0; k0 < g.K; k0 += KC) {
            const int kc = min(KC, g.K - k0);
            __syncthreads();
            // prepared reference for the chunk (thread per n, sequential over shells)
            for (int n = threadIdx.x; n < P; n += blockDim.x) {
                double2 st = has_shift ? sh[n] : make_double2(1.0, 0.0);
                const double2 v = has_shift ? sv[n] : make_double2(1.0, 0.0);
                for (int kk = 0; kk < kc; ++kk) {
                    const int ik = k0 + kk;
                    float2 rv = r[(long long)ik * P + n];
                    if (sn && ik < g.Ks) { rv.x *= sn[ik]; rv.y *= sn[ik]; }
                    float ar = rv.x, ai = rv.y;
                    if (FRAME != PFTCC_FRAME_PTCL && ctf) {
                        const float c = ctf[ik * P + n];
                        ar *= c; ai *= c;
                    }
                    if (FRAME == PFTCC_FRAME_PTCL) R2[kk * P + n] = rv.x * rv.x + rv.y * rv.y;
                    if (has_shift) {
                        const float sr = (float)st.x, si = (float)st.y;
                        const float tr = ar * sr - ai * si, ti = ar * si + ai * sr;
                        ar = tr; ai = ti;
                        // advance the recurrence: shmat(:,k+1) = shmat(:,k) * shvec
                        const double nr = st.x * v.x - st.y * v.y, ni = st.x * v.y + st.y * v.x;
                        st = make_double2(nr, ni);
                    }
                    A[kk * P + n] = make_float2(ar, ai);
                    if (FRAME == FRAME_EUCLID) {
                        if (ik < g.Ks) sqr += W[ik] * ((double)ar * ar + (double)ai * ai);
                    } else if (ik < ksq) {
                        sqr += (double)ar * ar + (double)ai * ai;
                    }
                }
                if (has_shift) sh[n] = st;
            }
            // extended particle for the chunk
            for (int e = threadIdx.x; e < kc * N; e += blockDim.x) {
                const int kk = e / N, j = e - kk * N, ik = k0 + kk;
                if (ik >= g.Ks) continue;
                const int jp = j < P ? j : j - P;
                float2 v = q[(long long)ik * P + jp];
                if (j >= P) v.y = -v.y;
                if (FRAME == PFTCC_FRAME_PTCL) {
                    const float c = ctf ? ctf[ik * P + jp] : 1.f;
                    v.x *= c; v.y *= c;
                    C2t[kk * N + j] = c * c;
                }
                if (FRAME == FRAME_EUCLID && j < P) sqr += W[ik] * ((double)v.x * v.x + (double)v.y * v.y);
                Qt[kk * N + j] = v;
            }
            __syncthreads();
            const int kend = min(kc, g.Ks - k0);
#pragma unroll
            for (int u = 0; u < EX_RPT; ++u) {
                const int s = threadIdx.x + u * EX_THREADS;
                if (s >= N) break;
                // products of the FP32 operands accumulated in FP64: the accumulation then
                // adds no rounding beyond the operands' own (FP32 sums over P*Ks terms
                // would add ~1e-5 relative on correlations near 1e-3)
                double a_tot = 0.0, d_tot = 0.0;
                for (int kk = 0; kk < kend; ++kk) {
                    const float2 *Ak = A + kk * P;
                    const float2 *Qk = Qt + kk * N;
                    int j = s;
                    // the Euclidean objective weights each shell's correlation
                    double a_k = FRAME == FRAME_EUCLID ? 0.0 : a_tot;
                    for (int n = 0; n < P; ++n) {
                        const float2 av = Ak[n];
                        const float2 qv = Qk[j];
                        a_k = fma((double)av.x, (double)qv.x, a_k);
                        a_k = fma((double)av.y, (double)qv.y, a_k);
                        if (FRAME == PFTCC_FRAME_PTCL) d_tot = fma((double)R2[kk * P + n], (double)C2t[kk * N + j], d_tot);
                        if (++j == N) j = 0;
                    }
                    if (FRAME == FRAME_EUCLID) a_tot = fma(W[k0 + kk], a_k, a_tot);
                    else a_tot = a_k;
                }
                acc[u] += a_tot;
                dacc[u] += d_tot;
            }
        }
        // square sum of the prepared reference
        for (int o = 16; o > 0; o >>= 1) sqr += __shfl_xor_sync(0xffffffffu, sqr, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sqr;
        __syncthreads();
        double sqr_tot = 0.0;
#pragma unroll
        for (int wi = 0; wi < EX_THREADS / 32; ++wi) sqr_tot += red[wi];
        float my_best = -INFINITY;
        int my_rot = 0;
#pragma unroll
        for (int u = 0; u < EX_RPT; ++u) {
            const int s = threadIdx.x + u * EX_THREADS;
            if (s >= N) break;
            float cc;
            if (FRAME == FRAME_EUCLID) {
                cc = (float)(acc[u] - 0.5 * sqr_tot);
            } else {
                const double den = FRAME == PFTCC_FRAME_REF ? sqrt(sqr_tot * sqp) : sqrt(dacc[u] * sqp);
                cc = (float)(acc[u] / den);
            }
            if (mode == MODE_FULL) out[w.out + s] = cc;
            // rotmask [group][N] (optional): rotations outside the mask take no part in the maximum
            if (cc > my_best && (!rotmask || rotmask[(size_t)blockIdx.x * N + s])) { my_best = cc; my_rot = s; }
        }
        if (mode == MODE_BEST || mode == MODE_ITEMMAX) {
            // block argmax, lowest rotation on ties (maxloc)
            for (int o = 16; o > 0; o >>= 1) {
                const float ob = __shfl_xor_sync(0xffffffffu, my_best, o);
                const int orot = __shfl_xor_sync(0xffffffffu, my_rot, o);
                if (ob > my_best || (ob == my_best && orot < my_rot)) { my_best = ob; my_rot = orot; }
            }
            if ((threadIdx.x & 31) == 0) { bcc[threadIdx.x >> 5] = my_best; brot[threadIdx.x >> 5] = my_rot; }
            __syncthreads();
            float bb = bcc[0];
            int br = brot[0];
            for (int wi = 1; wi < EX_THREADS / 32; ++wi)
                if (bcc[wi] > bb || (bcc[wi] == bb && brot[wi] < br)) { bb = bcc[wi]; br = brot[wi]; }
            if (bb > run_best) { run_best = bb; run_rot = br; run_item = it; }
            if (mode == MODE_ITEMMAX && threadIdx.x == 0) out[w.out] = bb;
        }
        __syncthreads();
    }
    if (mode == MODE_BEST && threadIdx.x == 0) {
        pftcc_best b;
        if (run_item >= 0) {
            const Work w = work[grp.first + run_item];
            b.iref = w.iref + 1;
            b.irot = run_rot + 1;
            b.ishift = w.ishift;
            b.corr = run_best;
        } else {
            b.iref = 0; b.irot = 0; b.ishift = -1; b.corr = -INFINITY;
        }
        best[grp.out_best] = b;
    }
}

static size_t exact_smem(const Geom &g, int frame, int kc)
{
    size_t b = al16(2 * g.P * sizeof(double2)) + al16((size_t)kc * g.N * sizeof(float2)) +
               al16((size_t)kc * g.P * sizeof(float2));
    if (frame == PFTCC_FRAME_PTCL) b += al16((size_t)kc * g.N * sizeof(float)) + al16((size_t)kc * g.P * sizeof(float));
    if (frame == FRAME_EUCLID) b += al16((size_t)g.K * sizeof(double));
    return b;
}

static int exact_kc(const Geom &g, int frame, size_t *smem)
{
    int kc = 8;
    while (kc > 1 && exact_smem(g, frame, kc) > 100 * 1024) --kc;
    *smem = exact_smem(g, frame, kc);
    return kc;
}

template <int FRAME>
static cudaError_t launch_exact_t(pftcc_handle *h, int kc, size_t smem, const Group *groups, int ngroups,
                                  const Work *work, const float *shifts, int mode, int cc1_kstop, float *out,
                                  pftcc_best *best, const uint8_t *rotmask)
{
    cudaError_t e = smem_limit((const void *)k_exact<FRAME>, smem);
    if (e != cudaSuccess) return e;
    const float *ctf = (h->cfg.with_ctf && h->ctf_ready) ? h->ctfmats : nullptr;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_EXACT);
    k_exact<FRAME><<<ngroups, EX_THREADS, smem, h->stream>>>(
        h->g, kc, h->refs_even, h->refs_odd, h->ptcls, ctf, h->d_iseven, h->sqsums, h->argtransf, h->argtransf1,
        groups, work, shifts, mode, cc1_kstop, h->d_sig2, h->d_pxls, snorm_ptr(h), h->nrefs, out, best, rotmask);
    return cudaGetLastError();
}

cudaError_t launch_exact(pftcc_handle *h, const Group *groups, int ngroups, const Work *work, const float *shifts,
                         int mode, int frame, int cc1_kstop, float *out, pftcc_best *best, const uint8_t *rotmask)
{
    if (frame == FRAME_EUCLID && (!h->d_sig2 || !h->d_pxls)) return cudaErrorInvalidValue;
    size_t smem;
    const int kc = exact_kc(h->g, frame, &smem);
    if (frame == PFTCC_FRAME_PTCL)
        return launch_exact_t<PFTCC_FRAME_PTCL>(h, kc, smem, groups, ngroups, work, shifts, mode, cc1_kstop, out, best,
                                                rotmask);
    if (frame == FRAME_EUCLID)
        return launch_exact_t<FRAME_EUCLID>(h, kc, smem, groups, ngroups, work, shifts, mode, cc1_kstop, out, best,
                                            rotmask);
    return launch_exact_t<PFTCC_FRAME_REF>(h, kc, smem, groups, ngroups, work, shifts, mode, cc1_kstop, out, best,
                                           rotmask);
}

// ---------------------------------------------------------------------------
// single-rotation correlation and its shift / defocus derivatives in double
// precision: gencorr_cc_for_rot_8 (:1690-1733) and gencorr_cc_grad_for_rot_8
// (:1863-1925), both branches (match_filt: unweighted sums normalised with
// sqsums over kstop; otherwise shell weights k in numerator and both norms).
// The derivative with respect to the defocus multiplies the reference by
// d|CTF|/d(df) instead of |CTF| and applies the quotient rule to the norm.
//
// One block per request.  ctf_mode 0: stored ctfmats (the drop-in calls);
// ctf_mode 1: |CTF| and its derivative recomputed at defocus + ddf.
struct RotReq { int iref, slot, irot, ctf_mode; double sx, sy, ddf; };
static_assert(sizeof(RotReq) == sizeof(RotReqH) && offsetof(RotReq, sx) == offsetof(RotReqH, sx),
              "RotReqH mirrors RotReq");

__device__ __forceinline__ double ctf_abs_d(const pftcc_ctfparams &c, double s2, double ang, double ddf, double *dctf)
{
    const double kv = 1000.0 * (double)c.kv;
    const double wl = (12.26 / sqrt(kv + (0.9784 * kv * kv) / 1.0e6)) / (double)c.smpd;
    const double cs = ((double)c.cs * 1.0e7) / (double)c.smpd;
    const double ampc = atan((double)c.fraca / sqrt(1.0 - (double)c.fraca * c.fraca));
    const double sc = 1.0e4 / (double)c.smpd;
    const double dfx = ((double)c.dfx + ddf) * sc, dfy = ((double)c.dfy + ddf) * sc;
    const double angast = (double)c.angast / 180.0 * 3.141592653589793;
    const double df = 0.5 * (dfx + dfy + cos(2.0 * (ang - angast)) * (dfx - dfy));
    double chi = 3.141592653589793 * wl * s2 * (df - 0.5 * wl * wl * s2 * cs) + ampc;
    if (c.l_phaseplate) chi += (double)c.phshift;
    double s, co;
    sincos(chi, &s, &co);
    *dctf = (s >= 0.0 ? 1.0 : -1.0) * co * 3.141592653589793 * wl * s2 * sc;
    return fabs(s);
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < NT / 32; ++w) t += red[w];
    return t;
}

constexpr int FR_THREADS = 256;

__global__ void __launch_bounds__(FR_THREADS) k_for_rot(
    Geom g, const RotReq *__restrict__ reqs, const float2 *__restrict__ refs_even,
    const float2 *__restrict__ refs_odd, const float2 *__restrict__ ptcls, const float *__restrict__ ctfmats,
    const pftcc_ctfparams *__restrict__ ctfp, const uint8_t *__restrict__ iseven, const float *__restrict__ polar,
    const double *__restrict__ argtransf, const double *__restrict__ argtransf1, int with_ctf, int match_filt,
    const float *__restrict__ snorm, int nrefs, double *__restrict__ out /* [nreq][5]: f, d/dsx, d/dsy, d/ddf, unused */)
{
    __shared__ double red[FR_THREADS / 32];
    const RotReq rq = reqs[blockIdx.x];
    const int N = g.N, P = g.P;
    const float2 *q = ptcls + (long long)rq.slot * g.K * P;
    const float2 *r = (iseven[rq.slot] ? refs_even : refs_odd) + (long long)rq.iref * g.K * P;
    // matched-filter mode: shellnorm_and_filter_ref_8's factors
    const float *sn = snorm ? snorm + ((size_t)(iseven[rq.slot] ? 0 : 1) * nrefs + rq.iref) * g.Ks : nullptr;
    const int s = rq.irot - 1;
    double corr = 0, sqr = 0, sqp = 0, gx = 0, gy = 0, gd = 0, dsq = 0;
    // thread per n; the shift phase of every shell follows the de Moivre recurrence
    for (int n = threadIdx.x; n < P; n += blockDim.x) {
        const double a = argtransf[n] * rq.sx + argtransf[P + n] * rq.sy;
        const double a1 = argtransf1[n] * rq.sx + argtransf1[P + n] * rq.sy;
        double st_r, st_i, v_r, v_i;
        sincos(a, &st_i, &st_r);
        sincos(a1, &v_i, &v_r);
        int j = s + n;
        if (j >= N) j -= N;
        const int jp = j < P ? j : j - P;
        const double qs = j < P ? 1.0 : -1.0;
        for (int ik = 0; ik < g.Ks; ++ik) {
            const double wgt = match_filt ? 1.0 : (double)(g.kfrom + ik);
            double c = 1.0, dc = 0.0;
            if (with_ctf) {
                if (rq.ctf_mode == 0) {
                    c = (double)ctfmats[((long long)rq.slot * g.K + ik) * P + n];
                } else {
                    const double x = polar[ik * 2 * N + n], y = polar[ik * 2 * N + N + n];
                    const double hinv = x / g.box, kinv = y / g.box;
                    c = ctf_abs_d(ctfp[rq.slot], hinv * hinv + kinv * kinv, atan2(y, x), rq.ddf, &dc);
                }
            }
            const float2 rv = r[(long long)ik * P + n];
            const double f = sn ? (double)sn[ik] : 1.0;
            const double rr = (double)rv.x * f * c, ri = (double)rv.y * f * c;
            const double ar = rr * st_r - ri * st_i, ai = rr * st_i + ri * st_r;   // prepared reference
            const float2 qv = q[(long long)ik * P + jp];
            const double qr = qv.x, qi = qs * qv.y;                                // ptcl~(j)
            corr += wgt * (ar * qr + ai * qi);
            sqr += wgt * (ar * ar + ai * ai);
            sqp += wgt * ((double)qv.x * qv.x + (double)qv.y * qv.y);
            // i * argtransf * A
            const double ax = argtransf[ik * N + n], ay = argtransf[ik * N + P + n];
            gx += wgt * ax * (-ai * qr + ar * qi);
            gy += wgt * ay * (-ai * qr + ar * qi);
            if (with_ctf && rq.ctf_mode == 1) {
                const double dr = (double)rv.x * f * dc, di = (double)rv.y * f * dc;
                const double br = dr * st_r - di * st_i, bi = dr * st_i + di * st_r;
                gd += wgt * (br * qr + bi * qi);
                dsq += wgt * 2.0 * (ar * br + ai * bi);
            }
            const double nr = st_r * v_r - st_i * v_i, ni = st_r * v_i + st_i * v_r;
            st_r = nr; st_i = ni;
        }
    }
    corr = block_sum<FR_THREADS>(corr, red);
    sqr = block_sum<FR_THREADS>(sqr, red);
    sqp = block_sum<FR_THREADS>(sqp, red);
    gx = block_sum<FR_THREADS>(gx, red);
    gy = block_sum<FR_THREADS>(gy, red);
    gd = block_sum<FR_THREADS>(gd, red);
    dsq = block_sum<FR_THREADS>(dsq, red);
    if (threadIdx.x == 0) {
        const double den = sqrt(sqr * sqp);
        const double f = corr / den;
        double *o = out + 5 * blockIdx.x;
        o[0] = f;
        o[1] = gx / den;
        o[2] = gy / den;
        o[3] = (with_ctf && rq.ctf_mode == 1) ? (gd / den - 0.5 * f * dsq / sqr) : 0.0;
        o[4] = 0.0;
    }
}

cudaError_t launch_for_rot(pftcc_handle *h, int iref, int slot, double sx, double sy, int irot, int match_filt,
                           int want_grad, double ddf, double *out5)
{
    // a single request: stage it through the small device buffer used for work items
    RotReq rq{iref, slot, irot, 0, sx, sy, ddf};
    (void)want_grad;
    cudaError_t e = cudaMemcpyAsync(h->d_work, &rq, sizeof(rq), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return e;
    PFTCC_LAUNCH(h);
    k_for_rot<<<1, FR_THREADS, 0, h->stream>>>(h->g, reinterpret_cast<const RotReq *>(h->d_work), h->refs_even,
                                                h->refs_odd, h->ptcls, h->ctfmats, h->d_ctfp, h->d_iseven, h->polar,
                                                h->argtransf, h->argtransf1, h->cfg.with_ctf && h->ctf_ready,
                                                match_filt, snorm_ptr(h), h->nrefs, out5);
    return cudaGetLastError();
}

// n single-rotation requests already on the device (reqs_dev: RotReq layout, see
// pftcc_internal.cuh), out5 [n][5] = f, df/dsx, df/dsy, df/ddf, unused
cudaError_t launch_rot_reqs(pftcc_handle *h, const void *reqs_dev, int n, double *out5)
{
    PFTCC_LAUNCH(h);
    k_for_rot<<<n, FR_THREADS, 0, h->stream>>>(h->g, reinterpret_cast<const RotReq *>(reqs_dev), h->refs_even,
                                                h->refs_odd, h->ptcls, h->ctfmats, h->d_ctfp, h->d_iseven, h->polar,
                                                h->argtransf, h->argtransf1, h->cfg.with_ctf && h->ctf_ready,
                                                h->cfg.match_filt, snorm_ptr(h), h->nrefs, out5);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// genfrc / calc_frc (:1417-1484) and specscore_1/_2 (:2190-2205): for each shell
// k <= kstop the correlation at irot over sqrt(sum_n |ptcl(n,k)|^2 * sum_n |ref(n,k)|^2),
// the reference prepared as ref * ctf * shmat (reference frame, as prep_ref4corr and
// calc_frc do; FP64 like the single-rotation correlators), 0 where that denominator is
// below 1e-12; the score is max(0, median) with median_nocopy's rule
// (simple_math.f90:2111-2130).  One block per request: threads over the polar angles,
// warps reduce their per-shell partial sums into the block's FP64 accumulators.
__global__ void __launch_bounds__(FR_THREADS) k_specscore(
    Geom g, const FrcReq *__restrict__ reqs, const float2 *__restrict__ refs_even, const float2 *__restrict__ refs_odd,
    const float2 *__restrict__ ptcls, const float *__restrict__ ctfmats, const uint8_t *__restrict__ iseven,
    const double *__restrict__ argtransf, const double *__restrict__ argtransf1, int with_ctf,
    float *__restrict__ frc_out /* [nreq][Ks] or null */, float *__restrict__ score_out)
{
    extern __shared__ double acc[];   // [3][Ks]: correlation, |ref|^2, |ptcl|^2
    const FrcReq rq = reqs[blockIdx.x];
    const int N = g.N, P = g.P, Ks = g.Ks, lane = threadIdx.x & 31;
    for (int e = threadIdx.x; e < 3 * Ks; e += blockDim.x) acc[e] = 0.0;
    __syncthreads();
    const float2 *q = ptcls + (long long)rq.slot * g.K * P;
    const float2 *r = (iseven[rq.slot] ? refs_even : refs_odd) + (long long)rq.iref * g.K * P;
    const int s = rq.irot - 1;
    for (int n0 = 0; n0 < P; n0 += blockDim.x) {
        const int n = n0 + threadIdx.x;
        const bool on = n < P;
        double st_r = 1.0, st_i = 0.0, v_r = 1.0, v_i = 0.0, qs = 1.0;
        int jp = 0;
        if (on) {
            if (rq.has_shift) {
                const double a = argtransf[n] * rq.sx + argtransf[P + n] * rq.sy;
                const double a1 = argtransf1[n] * rq.sx + argtransf1[P + n] * rq.sy;
                sincos(a, &st_i, &st_r);
                sincos(a1, &v_i, &v_r);
            }
            int j = s + n;
            if (j >= N) j -= N;
            jp = j < P ? j : j - P;
            qs = j < P ? 1.0 : -1.0;
        }
        for (int ik = 0; ik < Ks; ++ik) {
            double cr = 0.0, r2 = 0.0, p2 = 0.0;
            if (on) {
                const double c = with_ctf ? (double)ctfmats[((long long)rq.slot * g.K + ik) * P + n] : 1.0;
                const float2 rv = r[(long long)ik * P + n];
                const double rr = (double)rv.x * c, ri = (double)rv.y * c;
                const double ar = rr * st_r - ri * st_i, ai = rr * st_i + ri * st_r;
                const float2 qv = q[(long long)ik * P + jp];
                const double qr = qv.x, qi = qs * qv.y;
                cr = ar * qr + ai * qi;
                r2 = ar * ar + ai * ai;
                p2 = (double)qv.x * qv.x + (double)qv.y * qv.y;
                const double nr = st_r * v_r - st_i * v_i, ni = st_r * v_i + st_i * v_r;
                st_r = nr; st_i = ni;
            }
            for (int o = 16; o > 0; o >>= 1) {
                cr += __shfl_xor_sync(0xffffffffu, cr, o);
                r2 += __shfl_xor_sync(0xffffffffu, r2, o);
                p2 += __shfl_xor_sync(0xffffffffu, p2, o);
            }
            if (lane == 0) {
                atomicAdd(acc + ik, cr);
                atomicAdd(acc + Ks + ik, r2);
                atomicAdd(acc + 2 * Ks + ik, p2);
            }
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int ik = 0; ik < Ks; ++ik) {
            const double den = sqrt(acc[2 * Ks + ik] * acc[Ks + ik]);
            acc[ik] = den < 1e-12 ? 0.0 : acc[ik] / den;
            if (frc_out) frc_out[(long long)blockIdx.x * Ks + ik] = (float)acc[ik];
        }
        for (int a = 1; a < Ks; ++a) {      // insertion sort of the Ks shell values
            const double v = acc[a];
            int b = a - 1;
            while (b >= 0 && acc[b] > v) { acc[b + 1] = acc[b]; --b; }
            acc[b + 1] = v;
        }
        const double med = (Ks & 1) ? acc[Ks / 2] : 0.5 * (acc[Ks / 2 - 1] + acc[Ks / 2]);
        score_out[blockIdx.x] = (float)(med > 0.0 ? med : 0.0);
    }
}

cudaError_t launch_specscore(pftcc_handle *h, const FrcReq *reqs_dev, int nreq, float *frc_dev, float *score_dev)
{
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_EXACT);
    k_specscore<<<nreq, FR_THREADS, 3 * h->g.Ks * sizeof(double), h->stream>>>(
        h->g, reqs_dev, h->refs_even, h->refs_odd, h->ptcls, h->ctfmats, h->d_iseven, h->argtransf, h->argtransf1,
        h->cfg.with_ctf && h->ctf_ready, frc_dev, score_dev);
    return cudaGetLastError();
}

__global__ void k_grad_reqs(const pftcc_grad_req *__restrict__ in, const int *__restrict__ slots, int n,
                            RotReq *__restrict__ out)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const pftcc_grad_req r = in[i];
    out[i] = RotReq{r.iref - 1, slots[i], r.irot, 1, r.sx, r.sy, r.ddf};
}

cudaError_t launch_grad_batch(pftcc_handle *h, const pftcc_grad_req *req_dev, const int *slots_dev, int nreq,
                              double *out5)
{
    RotReq *rq = reinterpret_cast<RotReq *>(h->d_work);
    PFTCC_LAUNCH(h);
    k_grad_reqs<<<(nreq + 255) / 256, 256, 0, h->stream>>>(req_dev, slots_dev, nreq, rq);
    PFTCC_LAUNCH(h);
    k_for_rot<<<nreq, FR_THREADS, 0, h->stream>>>(h->g, rq, h->refs_even, h->refs_odd, h->ptcls, h->ctfmats,
                                                   h->d_ctfp, h->d_iseven, h->polar, h->argtransf, h->argtransf1,
                                                   h->cfg.with_ctf && h->ctf_ready, h->cfg.match_filt, snorm_ptr(h),
                                                   h->nrefs, out5);
    return cudaGetLastError();
}

}  // namespace pftcc
