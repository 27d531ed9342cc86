// k_search.cu -- the m-domain correlation search (particle-frame CTF).
//
// The reference correlates one (reference, particle) pair at a time with K FFT
// triples (calc_corrs_over_k, simple_polarft_corrcalc.f90:1132-1162).  Writing
// that computation out: with x~ the half-circle polar FT extended to the full
// circle by conjugate symmetry and U(m,k) = sum_{n<P} v_m(n,k) w_N^{-mn}
// (v_m = Re x for even m, Im x for odd m -- the r2c(P) and fft_factors-weighted
// c2c(P) transforms of memoize_fft :869-876 interleaved), the correlation is
//     corr(rot) = (2/N) * sum_{m<N} X(m) w_N^{-m rot},
//     X(m)      = sum_k U_A(m,k) conj(U_B(m,k))     (Hermitian in m),
// so for every angular frequency m = 0..P the work over all (ref, shift) x
// particle pairs is one complex contraction over the shells k, followed by one
// real inverse transform of length N per pair.  A is the reference times the
// shift phases of gen_shmat_8 (:1098-1120, reference side), B the particle times
// its |CTF| at the particle's own polar index (the particle frame; identical to
// the reference's prep_ref4corr :982 for an isotropic CTF), and the normaliser
// D(rot) = sum_k sum_n |ref(n,k)|^2 CTF^2(n+rot,k), P-periodic in rot, is the
// same kind of contraction over the P-point spectra of |ref|^2 and CTF^2, in FP64.
//
// Pipeline per call (all on the handle's stream):
//   k_spec_ptcl   particle spectra UB[m][col][k] (FP32) and CTF^2 spectra CV (FP64)
//   k_spec_r2     |ref|^2 spectra RU (FP64)
//   for each parity group (even/odd references, prep_ref4corr :970-974):
//     k_spec_ref  (ref, shift) spectra UA[m][rs][k] (FP32)
//     for each wave of rows (rs) x columns (particles):
//       stage 1   X[m][col][rs] = 4 sum_k UA conj(UB)   (FP32 CUDA cores, or tcgen05)
//       k_norm    D[r][col][rho] for the wave's references (FP64)
//       k_stage2  per (col, rs): length-P complex FFT of the packed Hermitian X,
//                 cc = (2/N) y / sqrt(D sqsum_ptcl), argmax over rotations, merge
//                 into the particle's running top-8 (cc, rs*N + rot)
//   k_finish      top-1, or the exact FP32 re-score of the top-ntop (ref, shift)
#include "pftcc_internal.cuh"
#include "spec_fft.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace pftcc {

int umma_stage1(pftcc_handle *h, int M, int Ks, const float2 *UA, int rs0, int nrs_w, int rows_pad,
                const float2 *UB, int c0, int ncols_w, int cols_pad, float2 *X, int prepare, int parity_group);
bool stage2_fast_supported(int P);
int stage2_fast_p2(int P);
int stage2_fast_dlen(int P);
cudaError_t launch_stage2_fast(pftcc_handle *h, int P, int rows, int xrows, int xcols, int row0, int nshifts, int r0,
                               int dcols, int col0, int cols, int nrs_total, const float2 *X, const float *Dinv,
                               float2 *cand, float *ccall, const int *perm, int eu);
cudaError_t launch_rescore_md(pftcc_handle *h, int P, int ncols, int ntop, int Ks, int nshifts, int has_shifts,
                              const float2 *UA, int rows_pad, const float2 *UB, int cols_pad, const double2 *RU,
                              const double2 *CV, const float *sqp, const float2 *cand, const int *perm, int c0,
                              pftcc_best *out, int eu);

static constexpr int MAXF = 12;
struct FFTPlan {
    int nf;
    int f[MAXF];     // radices, top level first
};

static FFTPlan make_plan(int P)
{
    FFTPlan p{};
    int m = P;
    const int rad[4] = {4, 2, 3, 5};
    for (int r = 0; r < 4; ++r)
        while (m % rad[r] == 0 && p.nf < MAXF) { p.f[p.nf++] = rad[r]; m /= rad[r]; }
    for (int q = 7; m > 1 && p.nf < MAXF; q += 2)
        while (m % q == 0) { p.f[p.nf++] = q; m /= q; }
    return p;
}

// position of input element i after the mixed-radix digit reversal that makes the
// in-place decimation-in-time passes produce natural-order output
static int digit_rev(const FFTPlan &p, int P, int i)
{
    int pos = 0, n = P;
    for (int l = 0; l < p.nf; ++l) {
        const int r = p.f[l];
        n /= r;
        pos += (i % r) * n;
        i /= r;
    }
    return pos;
}

// ---------------------------------------------------------------------------
// spectra of the (reference, shift) rows: U(m,k) = sum_n v_m(n,k) w_N^{-mn}
constexpr int SPEC_THREADS = 256;

__global__ void __launch_bounds__(SPEC_THREADS) k_spec_ref(
    Geom g, int nshifts, const float2 *__restrict__ refs, const float *__restrict__ shifts,
    const double *__restrict__ argtransf, const double *__restrict__ argtransf1, int rs0, int nrs, int rows_pad,
    float2 *__restrict__ UA)
{
    extern __shared__ float4 smem4[];
    const int N = g.N, P = g.P, Ks = g.Ks, M = P + 1;
    double2 *tw = reinterpret_cast<double2 *>(smem4);   // [N] w_N^{-e}
    float2 *a = reinterpret_cast<float2 *>(tw + N);      // [P][Ks]: the threads of a DFT step read consecutive k
    const int row = blockIdx.x;                          // local row
    const int rs = rs0 + row;
    float2 *dst = UA;
    if (rs >= nrs) {   // zero padding rows
        for (int e = threadIdx.x; e < M * Ks; e += blockDim.x) {
            const int m = e / Ks, k = e - m * Ks;
            dst[((size_t)m * rows_pad + row) * Ks + k] = make_float2(0.f, 0.f);
        }
        return;
    }
    const int r = rs / nshifts, s = rs - r * nshifts;
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * e / N, &sn, &cs);
        tw[e] = make_double2(cs, sn);
    }
    const float2 *R = refs + (size_t)r * g.K * P;
    const double sx = shifts ? (double)shifts[2 * s] : 0.0, sy = shifts ? (double)shifts[2 * s + 1] : 0.0;
    for (int n = threadIdx.x; n < P; n += blockDim.x) {
        // gen_shmat_8: analytic first shell, de Moivre recurrence, cast to single precision
        double sr, si, vr, vi;
        sincos(argtransf[n] * sx + argtransf[P + n] * sy, &si, &sr);
        sincos(argtransf1[n] * sx + argtransf1[P + n] * sy, &vi, &vr);
        for (int k = 0; k < Ks; ++k) {
            const float2 x = R[(size_t)k * P + n];
            const float fr = (float)sr, fi = (float)si;
            a[n * Ks + k] = make_float2(x.x * fr - x.y * fi, x.x * fi + x.y * fr);
            const double nr = sr * vr - si * vi, ni = sr * vi + si * vr;
            sr = nr; si = ni;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < M * Ks; e += blockDim.x) {
        const int m = e / Ks, k = e - m * Ks;
        const float2 *ak = a + k;
        // FP64 twiddles and accumulation: the spectra carry no more than the operands' FP32 rounding
        double ur = 0.0, ui = 0.0;
        int idx = 0;
        if (m & 1) {
            for (int n = 0; n < P; ++n) {
                const double v = ak[n * Ks].y;
                ur = fma(v, tw[idx].x, ur);
                ui = fma(v, tw[idx].y, ui);
                idx += m; if (idx >= N) idx -= N;
            }
        } else {
            for (int n = 0; n < P; ++n) {
                const double v = ak[n * Ks].x;
                ur = fma(v, tw[idx].x, ur);
                ui = fma(v, tw[idx].y, ui);
                idx += m; if (idx >= N) idx -= N;
            }
        }
        dst[((size_t)m * rows_pad + row) * Ks + k] = make_float2((float)ur, (float)ui);
    }
}

// particle-side spectra: B = |CTF| * ptcl (particle frame), UB[m][col][k]; and the
// FP64 spectra of CTF^2 over P points, CV[col][j][k], j = 0..P/2
__global__ void __launch_bounds__(SPEC_THREADS) k_spec_ptcl(
    Geom g, const float2 *__restrict__ ptcls, const float *__restrict__ ctfmats, const int *__restrict__ perm,
    int ncols, int cols_pad, float2 *__restrict__ UB, double2 *__restrict__ CV, float *__restrict__ sqp_out,
    const float *__restrict__ sqsums)
{
    extern __shared__ float4 smem4[];
    const int N = g.N, P = g.P, Ks = g.Ks, M = P + 1, J = P / 2 + 1;
    double2 *tw = reinterpret_cast<double2 *>(smem4);  // [N]
    float2 *b = reinterpret_cast<float2 *>(tw + N);     // [P][Ks]: DFT steps read consecutive k
    float *c2 = reinterpret_cast<float *>(b + Ks * P);  // [P][Ks]
    const int col = blockIdx.x;
    if (col >= ncols) {
        for (int e = threadIdx.x; e < M * Ks; e += blockDim.x) {
            const int m = e / Ks, k = e - m * Ks;
            UB[((size_t)m * cols_pad + col) * Ks + k] = make_float2(0.f, 0.f);
        }
        for (int e = threadIdx.x; e < J * Ks; e += blockDim.x) CV[(size_t)col * J * Ks + e] = make_double2(0.0, 0.0);
        if (threadIdx.x == 0) sqp_out[col] = 1.f;
        return;
    }
    const int slot = perm[col];
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * e / N, &sn, &cs);
        tw[e] = make_double2(cs, sn);
    }
    const float2 *Q = ptcls + (size_t)slot * g.K * P;
    const float *C = ctfmats ? ctfmats + (size_t)slot * g.K * P : nullptr;
    for (int e = threadIdx.x; e < Ks * P; e += blockDim.x) {
        const float c = C ? C[e] : 1.f;
        const float2 q = Q[e];
        const int k = e / P, n = e - k * P;
        b[n * Ks + k] = make_float2(c * q.x, c * q.y);
        c2[n * Ks + k] = c * c;
    }
    if (threadIdx.x == 0) sqp_out[col] = sqsums[slot];
    __syncthreads();
    for (int e = threadIdx.x; e < M * Ks; e += blockDim.x) {
        const int m = e / Ks, k = e - m * Ks;
        const float2 *bk = b + k;
        double ur = 0.0, ui = 0.0;
        int idx = 0;
        for (int n = 0; n < P; ++n) {
            const double v = (m & 1) ? bk[n * Ks].y : bk[n * Ks].x;
            ur = fma(v, tw[idx].x, ur);
            ui = fma(v, tw[idx].y, ui);
            idx += m; if (idx >= N) idx -= N;
        }
        UB[((size_t)m * cols_pad + col) * Ks + k] = make_float2((float)ur, (float)ui);
    }
    // CTF^2 spectra over P points in FP64: w_P^{-jn} = w_N^{-2jn}, read from the w_N table
    for (int e = threadIdx.x; e < J * Ks; e += blockDim.x) {
        const int j = e / Ks, k = e - j * Ks;
        double ur = 0.0, ui = 0.0;
        int idx = 0;
        for (int n = 0; n < P; ++n) {
            const double v = (double)c2[n * Ks + k];
            ur = fma(v, tw[idx].x, ur);
            ui = fma(v, tw[idx].y, ui);
            idx += 2 * j; if (idx >= N) idx -= N;
        }
        CV[(size_t)col * J * Ks + (size_t)j * Ks + k] = make_double2(ur, ui);
    }
}

// The same spectra by FP64 transforms of length N = N1 * N2 (spec_fft.cuh), shells in
// batches of sfft::KB: (reference, shift) rows UA[m][rs][k], one block per row.  The shifted
// polar samples a(n, k) are formed exactly as in k_spec_ref (FP32 products with the
// single-precision shift phases of the de Moivre recurrence), a batch of shells at a time
// ([shell][n] in shared memory), the recurrence state kept per angular sample n.
template <int N1, int N2>
__global__ void __launch_bounds__(SPEC_THREADS) k_spec_ref_fft(
    Geom g, int nshifts, const float2 *__restrict__ refs, const float *__restrict__ shifts,
    const double *__restrict__ argtransf, const double *__restrict__ argtransf1, int rs0, int nrs, int rows_pad,
    float2 *__restrict__ UA, int kb_per_block)
{
    constexpr int N = N1 * N2, P = N / 2, NPT = (P + SPEC_THREADS - 1) / SPEC_THREADS;
    extern __shared__ float4 smem4[];
    const int Ks = g.Ks, M = P + 1;
    // this block's shells [ka, kz): blockIdx.y selects kb_per_block batches of sfft::KB
    const int ka = blockIdx.y * kb_per_block * sfft::KB, kz = min(Ks, ka + kb_per_block * sfft::KB);
    double2 *tw = reinterpret_cast<double2 *>(smem4);                              // [N] w_N^{-e}
    double2 *buf = tw + N;                                                          // the transform buffer
    float2 *a = reinterpret_cast<float2 *>(buf + sfft::buf_elems<N1, N2>());       // [KB][P]
    const int row = blockIdx.x;
    const int rs = rs0 + row;
    if (rs >= nrs) {   // zero padding rows
        const int nk = kz - ka;
        for (int e = threadIdx.x; e < M * nk; e += blockDim.x) {
            const int m = e / nk, k = ka + e - m * nk;
            UA[((size_t)m * rows_pad + row) * Ks + k] = make_float2(0.f, 0.f);
        }
        return;
    }
    const int r = rs / nshifts, s = rs - r * nshifts;
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * e / N, &sn, &cs);
        tw[e] = make_double2(cs, sn);
    }
    const float2 *R = refs + (size_t)r * g.K * P;
    const double sx = shifts ? (double)shifts[2 * s] : 0.0, sy = shifts ? (double)shifts[2 * s + 1] : 0.0;
    // gen_shmat_8 per angular sample: analytic first shell, de Moivre recurrence over k
    double pr[NPT], pi[NPT], qr[NPT], qi[NPT];
#pragma unroll
    for (int i = 0; i < NPT; ++i) {
        const int n = threadIdx.x + i * SPEC_THREADS;
        pr[i] = 1.0; pi[i] = 0.0; qr[i] = 1.0; qi[i] = 0.0;
        if (n < P) {
            sincos(argtransf[n] * sx + argtransf[P + n] * sy, &pi[i], &pr[i]);
            sincos(argtransf1[n] * sx + argtransf1[P + n] * sy, &qi[i], &qr[i]);
            // the recurrence carried to the block's first shell by the same steps as below
            for (int k = 0; k < ka; ++k) {
                const double nr = pr[i] * qr[i] - pi[i] * qi[i], ni = pr[i] * qi[i] + pi[i] * qr[i];
                pr[i] = nr; pi[i] = ni;
            }
        }
    }
    for (int k0 = ka; k0 < kz; k0 += sfft::KB) {
        const int nk = min(sfft::KB, kz - k0);
#pragma unroll
        for (int i = 0; i < NPT; ++i) {
            const int n = threadIdx.x + i * SPEC_THREADS;
            if (n >= P) continue;
            for (int kl = 0; kl < nk; ++kl) {
                const float2 x = R[(size_t)(k0 + kl) * P + n];
                const float fr = (float)pr[i], fi = (float)pi[i];
                a[kl * P + n] = make_float2(x.x * fr - x.y * fi, x.x * fi + x.y * fr);
                const double nr = pr[i] * qr[i] - pi[i] * qi[i], ni = pr[i] * qi[i] + pi[i] * qr[i];
                pr[i] = nr; pi[i] = ni;
            }
        }
        auto getf = [&](int kl, int n) {
            const float2 v = a[kl * P + (n < P ? n : n - P)];
            return make_double2((double)v.x, n < P ? (double)v.y : -(double)v.y);
        };
        auto put = [&](int kl, int m, double2 F) {
            if (m <= P) {
                const float2 u = (m & 1) ? make_float2((float)(0.5 * F.y), (float)(-0.5 * F.x))
                                         : make_float2((float)(0.5 * F.x), (float)(0.5 * F.y));
                UA[((size_t)m * rows_pad + row) * Ks + k0 + kl] = u;
            }
        };
        sfft::batch_fft<N1, N2>(nk, getf, put, buf, tw);
    }
}

// particle-side spectra by the FP64 transforms: UB[m][col][k] of B = |CTF| * ptcl and the
// CTF^2 spectra CV[col][j][k] = sum_{n<P} CTF^2(n, k) w_P^{-jn} (the even outputs F(2j) / 2
// of the transform of the real sequence continued periodically over the full circle)
template <int N1, int N2>
__global__ void __launch_bounds__(SPEC_THREADS) k_spec_ptcl_fft(
    Geom g, const float2 *__restrict__ ptcls, const float *__restrict__ ctfmats, const int *__restrict__ perm,
    int ncols, int cols_pad, float2 *__restrict__ UB, double2 *__restrict__ CV, float *__restrict__ sqp_out,
    const float *__restrict__ sqsums, int kb_per_block)
{
    constexpr int N = N1 * N2, P = N / 2, J = P / 2 + 1;
    extern __shared__ float4 smem4[];
    const int Ks = g.Ks, M = P + 1;
    const int ka = blockIdx.y * kb_per_block * sfft::KB, kz = min(Ks, ka + kb_per_block * sfft::KB);
    double2 *tw = reinterpret_cast<double2 *>(smem4);                              // [N]
    double2 *buf = tw + N;
    float2 *b = reinterpret_cast<float2 *>(buf + sfft::buf_elems<N1, N2>());       // [KB][P]
    float *c2 = reinterpret_cast<float *>(b + sfft::KB * P);                        // [KB][P]
    const int col = blockIdx.x;
    if (col >= ncols) {
        const int nk = kz - ka;
        for (int e = threadIdx.x; e < M * nk; e += blockDim.x) {
            const int m = e / nk, k = ka + e - m * nk;
            UB[((size_t)m * cols_pad + col) * Ks + k] = make_float2(0.f, 0.f);
        }
        for (int e = threadIdx.x; e < J * nk; e += blockDim.x) {
            const int j = e / nk, k = ka + e - j * nk;
            CV[(size_t)col * J * Ks + (size_t)j * Ks + k] = make_double2(0.0, 0.0);
        }
        if (threadIdx.x == 0 && blockIdx.y == 0) sqp_out[col] = 1.f;
        return;
    }
    const int slot = perm[col];
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * e / N, &sn, &cs);
        tw[e] = make_double2(cs, sn);
    }
    const float2 *Q = ptcls + (size_t)slot * g.K * P;
    const float *C = ctfmats ? ctfmats + (size_t)slot * g.K * P : nullptr;
    if (threadIdx.x == 0 && blockIdx.y == 0) sqp_out[col] = sqsums[slot];
    for (int k0 = ka; k0 < kz; k0 += sfft::KB) {
        const int nk = min(sfft::KB, kz - k0);
        for (int e = threadIdx.x; e < nk * P; e += blockDim.x) {   // e = kl P + n
            const float c = C ? C[(size_t)k0 * P + e] : 1.f;
            const float2 q = Q[(size_t)k0 * P + e];
            b[e] = make_float2(c * q.x, c * q.y);
            c2[e] = c * c;
        }
        auto getf = [&](int kl, int n) {
            const float2 v = b[kl * P + (n < P ? n : n - P)];
            return make_double2((double)v.x, n < P ? (double)v.y : -(double)v.y);
        };
        auto put = [&](int kl, int m, double2 F) {
            if (m <= P) {
                const float2 u = (m & 1) ? make_float2((float)(0.5 * F.y), (float)(-0.5 * F.x))
                                         : make_float2((float)(0.5 * F.x), (float)(0.5 * F.y));
                UB[((size_t)m * cols_pad + col) * Ks + k0 + kl] = u;
            }
        };
        sfft::batch_fft<N1, N2>(nk, getf, put, buf, tw);
        auto getc = [&](int kl, int n) { return make_double2((double)c2[kl * P + (n < P ? n : n - P)], 0.0); };
        auto putc = [&](int kl, int m, double2 F) {
            if (!(m & 1) && m <= P) CV[(size_t)col * J * Ks + (size_t)(m >> 1) * Ks + k0 + kl] = make_double2(0.5 * F.x, 0.5 * F.y);
        };
        sfft::batch_fft<N1, N2>(nk, getc, putc, buf, tw);
    }
}

// shell batches per spectra block: all of a row's batches in one block when the rows fill the
// GPU many times over (the transform tables are then built once per row), one batch per block
// when they do not (a search without shifts has one row per reference)
static int spec_batches(const Geom &g) { return (g.Ks + sfft::KB - 1) / sfft::KB; }
static int spec_kb_per_block(const Geom &g, int rows) { return rows >= 16 * 148 ? spec_batches(g) : 1; }

template <int N1, int N2> static size_t spec_ref_fft_smem(int)
{
    return (size_t)N1 * N2 * sizeof(double2) + (size_t)sfft::buf_elems<N1, N2>() * sizeof(double2) +
           (size_t)sfft::KB * (N1 * N2 / 2) * sizeof(float2);
}
template <int N1, int N2> static size_t spec_ptcl_fft_smem(int)
{
    return spec_ref_fft_smem<N1, N2>(0) + (size_t)sfft::KB * (N1 * N2 / 2) * sizeof(float);
}

// launches of the spectra kernels: the FFT forms for the supported lengths, the direct
// sums otherwise (identical spectra up to FP64 rounding before the final FP32 / FP64 store)
template <int N1, int N2>
static cudaError_t launch_spec_ref_fft(pftcc_handle *h, const Geom &g, int ns, const float2 *refs, const float *shifts,
                                       int nrs, int rows_pad, float2 *UA)
{
    const size_t smem = spec_ref_fft_smem<N1, N2>(0);
    cudaError_t e = smem_limit((const void *)k_spec_ref_fft<N1, N2>, smem);
    if (e != cudaSuccess) return e;
    const int kbpb = spec_kb_per_block(g, rows_pad);
    const dim3 grid(rows_pad, (spec_batches(g) + kbpb - 1) / kbpb);
    PFTCC_LAUNCH(h);
    k_spec_ref_fft<N1, N2><<<grid, SPEC_THREADS, smem, h->stream>>>(g, ns, refs, shifts, h->argtransf, h->argtransf1, 0,
                                                                    nrs, rows_pad, UA, kbpb);
    return cudaGetLastError();
}

static cudaError_t launch_spec_ref(pftcc_handle *h, const Geom &g, int ns, const float2 *refs, const float *shifts,
                                   int nrs, int rows_pad, float2 *UA)
{
    switch (g.P) {
    case 64: return launch_spec_ref_fft<16, 8>(h, g, ns, refs, shifts, nrs, rows_pad, UA);
    case 180: return launch_spec_ref_fft<24, 15>(h, g, ns, refs, shifts, nrs, rows_pad, UA);
    case 300: return launch_spec_ref_fft<24, 25>(h, g, ns, refs, shifts, nrs, rows_pad, UA);
    default: break;
    }
    const size_t smem = g.N * sizeof(double2) + (size_t)g.Ks * g.P * sizeof(float2);
    cudaError_t e = smem_limit((const void *)k_spec_ref, smem);
    if (e != cudaSuccess) return e;
    PFTCC_LAUNCH(h);
    k_spec_ref<<<rows_pad, SPEC_THREADS, smem, h->stream>>>(g, ns, refs, shifts, h->argtransf, h->argtransf1, 0, nrs,
                                                            rows_pad, UA);
    return cudaGetLastError();
}

template <int N1, int N2>
static cudaError_t launch_spec_ptcl_fft(pftcc_handle *h, const Geom &g, const float *ctf, const int *perm, int np,
                                        int cols_pad, float2 *UB, double2 *CV, float *sqp)
{
    const size_t smem = spec_ptcl_fft_smem<N1, N2>(0);
    cudaError_t e = smem_limit((const void *)k_spec_ptcl_fft<N1, N2>, smem);
    if (e != cudaSuccess) return e;
    const int kbpb = spec_kb_per_block(g, cols_pad);
    const dim3 grid(cols_pad, (spec_batches(g) + kbpb - 1) / kbpb);
    PFTCC_LAUNCH(h);
    k_spec_ptcl_fft<N1, N2><<<grid, SPEC_THREADS, smem, h->stream>>>(g, h->ptcls, ctf, perm, np, cols_pad, UB, CV, sqp,
                                                                     h->sqsums, kbpb);
    return cudaGetLastError();
}

static cudaError_t launch_spec_ptcl(pftcc_handle *h, const Geom &g, const float *ctf, const int *perm, int np,
                                    int cols_pad, float2 *UB, double2 *CV, float *sqp)
{
    switch (g.P) {
    case 64: return launch_spec_ptcl_fft<16, 8>(h, g, ctf, perm, np, cols_pad, UB, CV, sqp);
    case 180: return launch_spec_ptcl_fft<24, 15>(h, g, ctf, perm, np, cols_pad, UB, CV, sqp);
    case 300: return launch_spec_ptcl_fft<24, 25>(h, g, ctf, perm, np, cols_pad, UB, CV, sqp);
    default: break;
    }
    const size_t smem = g.N * sizeof(double2) + (size_t)g.Ks * g.P * (sizeof(float2) + sizeof(float));
    cudaError_t e = smem_limit((const void *)k_spec_ptcl, smem);
    if (e != cudaSuccess) return e;
    PFTCC_LAUNCH(h);
    k_spec_ptcl<<<cols_pad, SPEC_THREADS, smem, h->stream>>>(g, h->ptcls, ctf, perm, np, cols_pad, UB, CV, sqp,
                                                             h->sqsums);
    return cudaGetLastError();
}

// |ref|^2 spectra over P points (FP64): RU[r][j][k]
__global__ void __launch_bounds__(SPEC_THREADS) k_spec_r2(Geom g, const float2 *__restrict__ refs,
                                                          double2 *__restrict__ RU)
{
    const int P = g.P, Ks = g.Ks, J = P / 2 + 1;
    const int r = blockIdx.x;
    const float2 *R = refs + (size_t)r * g.K * P;
    for (int e = threadIdx.x; e < J * Ks; e += blockDim.x) {
        const int j = e / Ks, k = e - j * Ks;
        double ur = 0.0, ui = 0.0;
        for (int n = 0; n < P; ++n) {
            const float2 x = R[(size_t)k * P + n];
            const double u = (double)x.x * x.x + (double)x.y * x.y;
            double sn, cs;
            sincospi(-2.0 * (double)((j * n) % P) / P, &sn, &cs);
            ur += u * cs;
            ui += u * sn;
        }
        RU[(size_t)r * J * Ks + (size_t)j * Ks + k] = make_double2(ur, ui);
    }
}

// The same |ref|^2 spectra by the FP64 transforms of length N = 2P (spec_fft.cuh): RU(j) is
// F(2j) / 2 of the transform of |ref|^2 continued periodically over the full circle, as the
// CTF^2 spectra of k_spec_ptcl_fft.  Block (reference, kb_per_block batches of sfft::KB shells).
template <int N1, int N2>
__global__ void __launch_bounds__(SPEC_THREADS) k_spec_r2_fft(Geom g, const float2 *__restrict__ refs,
                                                              double2 *__restrict__ RU, int kb_per_block)
{
    constexpr int N = N1 * N2, P = N / 2, J = P / 2 + 1;
    extern __shared__ float4 smem4[];
    const int Ks = g.Ks;
    const int ka = blockIdx.y * kb_per_block * sfft::KB, kz = min(Ks, ka + kb_per_block * sfft::KB);
    double2 *tw = reinterpret_cast<double2 *>(smem4);                              // [N]
    double2 *buf = tw + N;
    double *u2 = reinterpret_cast<double *>(buf + sfft::buf_elems<N1, N2>());      // [KB][P]
    const int r = blockIdx.x;
    for (int e = threadIdx.x; e < N; e += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * e / N, &sn, &cs);
        tw[e] = make_double2(cs, sn);
    }
    const float2 *R = refs + (size_t)r * g.K * P;
    for (int k0 = ka; k0 < kz; k0 += sfft::KB) {
        const int nk = min(sfft::KB, kz - k0);
        for (int e = threadIdx.x; e < nk * P; e += blockDim.x) {   // e = kl P + n
            const float2 x = R[(size_t)k0 * P + e];
            u2[e] = (double)x.x * x.x + (double)x.y * x.y;
        }
        auto getc = [&](int kl, int n) { return make_double2(u2[kl * P + (n < P ? n : n - P)], 0.0); };
        auto putc = [&](int kl, int m, double2 F) {
            if (!(m & 1) && m <= P) RU[(size_t)r * J * Ks + (size_t)(m >> 1) * Ks + k0 + kl] = make_double2(0.5 * F.x, 0.5 * F.y);
        };
        sfft::batch_fft<N1, N2>(nk, getc, putc, buf, tw);
    }
}

template <int N1, int N2> static cudaError_t launch_spec_r2_fft(pftcc_handle *h, const Geom &g, const float2 *refs,
                                                                  double2 *RU)
{
    const size_t smem = (size_t)N1 * N2 * sizeof(double2) + (size_t)sfft::buf_elems<N1, N2>() * sizeof(double2) +
                        (size_t)sfft::KB * (N1 * N2 / 2) * sizeof(double);
    cudaError_t e = smem_limit((const void *)k_spec_r2_fft<N1, N2>, smem);
    if (e != cudaSuccess) return e;
    const int kbpb = spec_kb_per_block(g, h->nrefs);
    const dim3 grid(h->nrefs, (spec_batches(g) + kbpb - 1) / kbpb);
    PFTCC_LAUNCH(h);
    k_spec_r2_fft<N1, N2><<<grid, SPEC_THREADS, smem, h->stream>>>(g, refs, RU, kbpb);
    return cudaGetLastError();
}

// |ref|^2 spectra: the transforms for the supported lengths, the direct sums otherwise
static cudaError_t launch_spec_r2(pftcc_handle *h, const Geom &g, const float2 *refs, double2 *RU)
{
    switch (g.P) {
    case 64: return launch_spec_r2_fft<16, 8>(h, g, refs, RU);
    case 180: return launch_spec_r2_fft<24, 15>(h, g, refs, RU);
    case 300: return launch_spec_r2_fft<24, 25>(h, g, refs, RU);
    default: break;
    }
    PFTCC_LAUNCH(h);
    k_spec_r2<<<h->nrefs, SPEC_THREADS, 0, h->stream>>>(g, refs, RU);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// stage 1 on CUDA cores: X[m][col][row] = 4 * sum_k UA[m][row][k] * conj(UB[m][col][k])
// for the plane pair (m, P - m) of blockIdx.z (m = 0 pairs with P; m = P/2 with itself),
// stored as the packed spectrum of stage 2, Z(m) and Z(P - m) (make_z).  Block tile 64
// cols x 64 rows, 256 threads with 4 x 4 complex micro-tiles per plane, the whole shell
// range of both planes staged in shared memory (Ks <= 64).
constexpr int S1_TILE = 64;
constexpr int COL_TILE = 128;

__global__ void __launch_bounds__(256) k_stage1_fp32(int Ks, int P, const float2 *__restrict__ UA, int rows_pad,
                                                     int row0, const float2 *__restrict__ UB, int cols_pad, int col0,
                                                     float2 *__restrict__ Z, int xrows, int xcols)
{
    extern __shared__ float4 smem4[];
    float2 *sa = reinterpret_cast<float2 *>(smem4);   // [2 planes][Ks][64] rows
    float2 *sb = sa + 2 * Ks * S1_TILE;                // [2 planes][Ks][64] cols
    const int mp = blockIdx.z;
    const int mA = mp, mB = mp == 0 ? P : P - mp;
    const int rt = blockIdx.x * S1_TILE, ct = blockIdx.y * S1_TILE;
    for (int h = 0; h < 2; ++h) {
        const int m = h == 0 ? mA : mB;
        const float2 *A = UA + ((size_t)m * rows_pad + row0 + rt) * Ks;
        const float2 *B = UB + ((size_t)m * cols_pad + col0 + ct) * Ks;
        for (int e = threadIdx.x; e < S1_TILE * Ks; e += blockDim.x) {
            const int i = e / Ks, k = e - i * Ks;
            sa[(h * Ks + k) * S1_TILE + i] = A[e];
            sb[(h * Ks + k) * S1_TILE + i] = B[e];
        }
    }
    __syncthreads();
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;   // rows 4*tx.., cols 4*ty..
    float accr[2][4][4], acci[2][4][4];
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) { accr[h][i][j] = 0.f; acci[h][i][j] = 0.f; }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const float2 *sah = sa + h * Ks * S1_TILE, *sbh = sb + h * Ks * S1_TILE;
        for (int k = 0; k < Ks; ++k) {
            const float4 a01 = *reinterpret_cast<const float4 *>(sah + k * S1_TILE + 4 * tx);
            const float4 a23 = *reinterpret_cast<const float4 *>(sah + k * S1_TILE + 4 * tx + 2);
            const float4 b01 = *reinterpret_cast<const float4 *>(sbh + k * S1_TILE + 4 * ty);
            const float4 b23 = *reinterpret_cast<const float4 *>(sbh + k * S1_TILE + 4 * ty + 2);
            const float ar[4] = {a01.x, a01.z, a23.x, a23.z}, ai[4] = {a01.y, a01.w, a23.y, a23.w};
            const float br[4] = {b01.x, b01.z, b23.x, b23.z}, bi[4] = {b01.y, b01.w, b23.y, b23.w};
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    // a * conj(b)
                    accr[h][i][j] = fmaf(ar[i], br[j], fmaf(ai[i], bi[j], accr[h][i][j]));
                    acci[h][i][j] = fmaf(ai[i], br[j], fmaf(-ar[i], bi[j], acci[h][i][j]));
                }
        }
    }
    const int N = 2 * P;
    const float2 wA = wn_of(mA, N), wB = wn_of(mB, N);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        const int col = ct + 4 * ty + j;
        if (col >= xcols) continue;
        float2 *dA = Z + ((size_t)mA * xcols + col) * xrows + rt + 4 * tx;
        float2 *dB = Z + ((size_t)(mB < P ? mB : 0) * xcols + col) * xrows + rt + 4 * tx;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            if (rt + 4 * tx + i >= xrows) continue;
            float2 xa = make_float2(4.f * accr[0][i][j], 4.f * acci[0][i][j]);
            float2 xb = make_float2(4.f * accr[1][i][j], 4.f * acci[1][i][j]);
            if (mp == 0) {              // X(0) and X(P) are real
                xa.y = 0.f;
                xb.y = 0.f;
                dA[i] = make_z(xa, xb, wA);
            } else {
                dA[i] = make_z(xa, xb, wA);
                if (mB != mA) dB[i] = make_z(xb, xa, wB);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// rotation-dependent normaliser D(rho) = (1/P) sum_j wgt_j Re[Y(j) w_P^{+j rho}] with
// Y(j) = sum_k conj(RU[r][j][k]) CV[col][j][k] (wgt_j = 1 at j = 0 and j = P/2, else 2)
// (spectra FP64, products FP32, transform FP64); stored as the FP32 factor
// Dinv[rl][col][rho] = 1/sqrt(D(rho) * sqsum_ptcl(col)) the correlations are scaled by.
// Two kernels per wave:
//   k_norm_y2: Y for every (reference, particle) pair of the wave as a batched complex
//            product over the shells, from FP32 copies of the spectra transposed to
//            [j][k][reference] and [j][k][particle] (k_norm_cvt), two-lane FP32 FMAs (these
//            factors rank the search's candidates; the re-score forms its own normaliser in
//            FP64); Y[rl][cl][j] unscaled, FP32;
//   k_norm:  D from Y, one block per particle column, NORM_RB = 32 references at a time:
//            lane = reference, each thread NORM_GPT residues g < P/Q, and for each g the Q
//            rotations rho = g + q P/Q at once: with S_r = sum_{j = r mod Q} Y(j) w_P^{j g},
//            D(g + q P/Q) = Re sum_r i_Q^{q r} S_r (i_Q = exp(2 pi i/Q)); the twiddles
//            w_P^{j g} come from an FP64 table in shared memory and are the same for the
//            whole warp (broadcast reads).
// Layouts of the stored factor: p2 == 0, natural Dinv[rl][col][rho] (P values); p2 > 0,
// the order in which the split-radix stage 2 (P = P1 x p2) reads them, block pairs
// (l2, l2 + 1) of its pass B: Dinv[rl][col][l2 >> 1][l1][b][l2 & 1] for
// rot = 2 (l2 + p2 l1) + b (rho = rot mod P; for odd p2 lane 1 of the last pair repeats
// l2 = p2 - 1; 4 P1 ceil(p2 / 2) values), multiplied by dscale.
// FP32 copies of the normaliser's spectra, transposed so that the contraction below reads
// them coalesced: RUf[j][k][r] = RU[r][j][k] (|ref|^2 spectra), CVf[j][k][c] = CV[c][j][k]
// (CTF^2 spectra); the values the FP64 spectra round to, as the contraction always used
constexpr int CVT_BLOCKS = 8 * 148;   // grid-stride copy, 8 blocks per SM of a B200
__global__ void k_norm_cvt(int n, int J, int Ks, int n_pad, const double2 *__restrict__ src, float2 *__restrict__ dst)
{
    const long long tot = (long long)n_pad * J * Ks;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < tot; e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e % n_pad);
        const long long jk = e / n_pad;   // j * Ks + k
        float2 v = make_float2(0.f, 0.f);
        if (r < n) {
            const double2 u = src[(size_t)r * J * Ks + jk];
            v = make_float2((float)u.x, (float)u.y);
        }
        dst[e] = v;
    }
}

// Y(j) = sum_k conj(RU(j,k)) CV(j,k) for every (reference, particle) pair of a wave: FP32 products
// accumulated in FP32 as two lane-pair fmas per complex product, (u.x, u.x)(v.x, v.y) +
// (u.y, u.y)(v.y, -v.x), k in increasing order.  Block: one j, NY2_R = 8 references x 512
// particles, 4 warps; every thread takes the 8 references (their spectra read at one address per
// warp) and the particles l + 32 q (q < 4) of its warp's 128 (coalesced reads), 32 accumulators.
// Y[(rl * ncols + cl) * J + j] unscaled (the transform applies the weights wgt_j / P).
constexpr int NY2_R = 8, NY2_C = 512, NY2_KC = 8;   // references, particles and shells per chunk of a block
constexpr size_t NY2_SMEM = 2 * (size_t)NY2_KC * NY2_C * sizeof(float2);
__global__ void __launch_bounds__(128) k_norm_y2(int Ks, int J, const float2 *__restrict__ RUf, int nrefs_p,
                                                 const float2 *__restrict__ CVf, int cols_pad, int r0, int nr, int c0,
                                                 int ncols, float2 *__restrict__ Y)
{
    __shared__ float2 us[64][NY2_R];     // the block's references' spectra at this j, [k][reference]
    extern __shared__ float2 cvs[];      // [2][NY2_KC][NY2_C] its particles' spectra, NY2_KC shells per chunk
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int rb = blockIdx.y * NY2_R, cb0 = blockIdx.x * NY2_C, cb = cb0 + warp * 128, j = blockIdx.z;
    const float2 *ur = RUf + (size_t)j * Ks * nrefs_p;
    const float2 *vr = CVf + (size_t)j * Ks * cols_pad;
    for (int e = threadIdx.x; e < NY2_R * Ks; e += blockDim.x) {   // clamped reads (the stores are masked)
        const int k = e / NY2_R, i = e - k * NY2_R;
        us[k][i] = __ldg(ur + (size_t)k * nrefs_p + r0 + min(rb + i, nr - 1));
    }
    // the particles' spectra in chunks of NY2_KC shells by asynchronous 8-byte copies, the next chunk
    // in flight while this one is used (clamped columns; the stores are masked)
    const int nch = (Ks + NY2_KC - 1) / NY2_KC;
    auto fetch = [&](int ch) {
        float2 *dst = cvs + (size_t)(ch & 1) * NY2_KC * NY2_C;
        const int k0 = ch * NY2_KC, nk = min(NY2_KC, Ks - k0);
        for (int e = threadIdx.x; e < nk * NY2_C; e += blockDim.x) {
            const int kk = e / NY2_C, c = e - kk * NY2_C;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(dst + e)),
                         "l"(vr + (size_t)(k0 + kk) * cols_pad + c0 + min(cb0 + c, ncols - 1))
                         : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    fetch(0);
    const bool active = cb < ncols;
    float2 acc[NY2_R][4];
#pragma unroll
    for (int i = 0; i < NY2_R; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[i][q] = make_float2(0.f, 0.f);
    for (int ch = 0; ch < nch; ++ch) {
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();    // chunk ch landed for everyone; chunk ch - 1's buffer is free
        if (ch + 1 < nch) fetch(ch + 1);
        const float2 *cv = cvs + (size_t)(ch & 1) * NY2_KC * NY2_C + warp * 128 + lane;
        const int k0 = ch * NY2_KC, nk = min(NY2_KC, Ks - k0);
        if (active) {
#pragma unroll 4
            for (int kk = 0; kk < nk; ++kk) {
                float2 v[4], vb[4];
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    v[q] = cv[kk * NY2_C + 32 * q];
                    vb[q] = make_float2(v[q].y, -v[q].x);
                }
#pragma unroll
                for (int i = 0; i < NY2_R; ++i) {
                    const float2 u = us[k0 + kk][i];
                    const float2 ux = make_float2(u.x, u.x), uy = make_float2(u.y, u.y);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        acc[i][q] = __ffma2_rn(ux, v[q], acc[i][q]);
                        acc[i][q] = __ffma2_rn(uy, vb[q], acc[i][q]);
                    }
                }
            }
        }
    }
    if (!active) return;
#pragma unroll
    for (int i = 0; i < NY2_R; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int rl = rb + i, cl = cb + lane + 32 * q;
            if (rl < nr && cl < ncols) Y[((size_t)rl * ncols + cl) * J + j] = acc[i][q];
        }
}

constexpr int NORM_RB = 32;
constexpr int NORM_GPT = 3;
template <int Q>
__global__ void __launch_bounds__(256) k_norm(Geom g, const float2 *__restrict__ Yg, int nr, int c0, int ncols,
                                              int dcols, const float *__restrict__ sqp, float *__restrict__ D, int p2,
                                              double dscale)
{
    extern __shared__ double2 sd[];
    const int P = g.P, J = P / 2 + 1, G = P / Q, Jp = J | 1;
    const int p1 = p2 > 0 ? P / p2 : 0, dlen = p2 > 0 ? 4 * p1 * ((p2 + 1) / 2) : P;
    double2 *Y = sd;                            // [NORM_RB][Jp], scaled by wgt_j / P
    double2 *tw = Y + (size_t)NORM_RB * Jp;     // [P] w_P^{+e}
    const int cl = blockIdx.x;
    if (cl >= ncols) return;
    const int col = c0 + cl;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int e = threadIdx.x; e < P; e += blockDim.x) {
        double s, c;
        sincospi(2.0 * e / P, &s, &c);
        tw[e] = make_double2(c, s);
    }
    const double sq = (double)sqp[col];
    for (int rb0 = 0; rb0 < nr; rb0 += NORM_RB) {
        const int nb = min(NORM_RB, nr - rb0);
        __syncthreads();
        for (int it = threadIdx.x; it < nb * J; it += blockDim.x) {
            const int rb = it / J, j = it - rb * J;
            const float2 a = Yg[((size_t)(rb0 + rb) * ncols + cl) * J + j];
            const double wgt = ((j == 0 || 2 * j == P) ? 1.0 : 2.0) / P;
            Y[(size_t)rb * Jp + j] = make_double2(wgt * a.x, wgt * a.y);
        }
        __syncthreads();
        if (lane < nb) {
            const double2 *y = Y + (size_t)lane * Jp;
            float *dst = D + ((size_t)(rb0 + lane) * dcols + cl) * dlen;
            for (int g0 = warp * NORM_GPT; g0 < G; g0 += nwarps * NORM_GPT) {
                double sr[NORM_GPT][Q], si[NORM_GPT][Q];
                int idx[NORM_GPT];
#pragma unroll
                for (int t = 0; t < NORM_GPT; ++t) {
                    idx[t] = 0;
#pragma unroll
                    for (int q = 0; q < Q; ++q) sr[t][q] = si[t][q] = 0.0;
                }
                for (int j0 = 0; j0 < J; j0 += Q) {
#pragma unroll
                    for (int q = 0; q < Q; ++q) {
                        const int j = j0 + q;
                        if (j < J) {
                            const double2 a = y[j];
#pragma unroll
                            for (int t = 0; t < NORM_GPT; ++t) {
                                const double2 w = tw[idx[t]];
                                sr[t][q] = fma(a.x, w.x, fma(-a.y, w.y, sr[t][q]));
                                si[t][q] = fma(a.x, w.y, fma(a.y, w.x, si[t][q]));
                                idx[t] += g0 + t;                 // (j * g) mod P
                                if (idx[t] >= P) idx[t] -= P;
                            }
                        }
                    }
                }
#pragma unroll
                for (int t = 0; t < NORM_GPT; ++t) {
                    const int gg = g0 + t;
                    if (gg >= G) continue;
#pragma unroll
                    for (int q = 0; q < Q; ++q) {
                        // Re sum_r i_Q^{q r} S_r
                        double d = 0.0;
#pragma unroll
                        for (int r = 0; r < Q; ++r) {
                            const int e = (q * r) % Q;   // i_Q^e in {1, i, -1, -i} (Q = 4), {1, -1} (Q = 2)
                            if (Q == 1 || e == 0) d += sr[t][r];
                            else if (2 * e == Q) d -= sr[t][r];
                            else if (4 * e == Q) d -= si[t][r];
                            else d += si[t][r];            // 4 e == 3 Q
                        }
                        const int rho = gg + q * G;
                        if (p2 == 0) {
                            dst[rho] = (float)(1.0 / sqrt(d * sq));
                        } else {
                            const float v = (float)(dscale / sqrt(d * sq));
#pragma unroll
                            for (int h = 0; h < 2; ++h) {   // rot = rho and rho + P
                                const int rot = rho + h * P, l = rot >> 1, l2 = l % p2;
                                float *o = dst + ((((l2 >> 1) * p1 + l / p2) * 2 + (rot & 1)) * 2 + (l2 & 1));
                                o[0] = v;
                                if ((p2 & 1) && l2 == p2 - 1) o[1] = v;
                            }
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
}

// D from Y by an FP64 transform of length P/2 = N1 * N2 (spec_fft.cuh), the lengths with
// that split; same inputs, outputs and layouts as k_norm.  With c_j = Y(j) (j <= P/2, already
// scaled by wgt_j / P), D(rho) = sum_{j<P} H(j) w_P^{+j rho} for the Hermitian extension H
// (H(0) = Re c_0, H(P/2) = Re c_{P/2}, H(j) = c_j / 2, H(P - j) = conj(c_j) / 2), and
// z(l) = D(2l) + i D(2l + 1) is the length-P/2 inverse DFT of
// Zh(j) = [H(j) + H(j + P/2)] + i [H(j) - H(j + P/2)] w_P^{+j}, computed as conj of the
// forward transform of conj(Zh).  One block per particle column, NB references per batch:
//   pass 1, task (reference, n1): a length-N2 DFT over n2 of conj Zh(n1 + N1 n2), times
//           w_{P/2}^{-n1 k2}, into buf[reference][k2][n1];
//   pass 2, task (reference, k2): a length-N1 DFT over n1 -> conj z(k2 + N2 k1).
// P2C: the stage-2 split P = P1 x P2C the factors are laid out for (compile-time, so that the
// layout's index arithmetic divides by a constant), or 0 for the natural layout
template <int N1, int N2, int P2C>
__global__ void __launch_bounds__(256) k_norm_fft(const float2 *__restrict__ Yg, int nr, int c0, int ncols, int dcols,
                                                  const float *__restrict__ sqp, float *__restrict__ D, double dscale,
                                                  int eu)
{
    constexpr int H = N1 * N2, P = 2 * H, J = H + 1;
    constexpr int p2 = P2C;
    constexpr int NB = 256 / (N1 > N2 ? N1 : N2);
    extern __shared__ double2 sd[];
    double2 *tw = sd;                 // [H] w_{P/2}^{-e}
    double2 *wp = tw + H;             // [H] w_P^{+e}
    double2 *buf = wp + H;            // [NB][N2][N1 + 1]
    float2 *ys = reinterpret_cast<float2 *>(buf + NB * N2 * (N1 + 1));   // [NB][J] the batch's Y rows
    const int cl = blockIdx.x;
    if (cl >= ncols) return;
    const int col = c0 + cl;
    for (int e = threadIdx.x; e < H; e += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * e / H, &sn, &cs);
        tw[e] = make_double2(cs, sn);
        sincospi(2.0 * e / P, &sn, &cs);
        wp[e] = make_double2(cs, sn);
    }
    const double sq = (double)sqp[col];
    constexpr int p1 = p2 > 0 ? P / p2 : 0, dlen = p2 > 0 ? 4 * p1 * ((p2 + 1) / 2) : P;
    // a batch's Y rows (J values each, coalesced) by asynchronous 8-byte copies: the first batch's
    // before the loop, every later batch's while the previous batch's pass 2 runs (pass 1 has
    // consumed ys by then)
    auto fetch = [&](int b0) {
        const int n = min(NB, nr - b0);
        for (int e = threadIdx.x; e < n * J; e += blockDim.x) {
            const int kl = e / J, j = e - kl * J;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((uint32_t)__cvta_generic_to_shared(ys + e)),
                         "l"(Yg + ((size_t)(b0 + kl) * ncols + cl) * J + j)
                         : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    fetch(0);
    for (int rb0 = 0; rb0 < nr; rb0 += NB) {
        const int nb = min(NB, nr - rb0);
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        for (int t = threadIdx.x; t < nb * N1; t += blockDim.x) {
            const int kl = t / N1, n1 = t - kl * N1;
            const float2 *y = ys + (size_t)kl * J;
            // Y(j) times wgt_j / P: 1 / P at j = 0 and j = P/2, 2 / P otherwise
            const double w1 = 1.0 / P, w2 = 2.0 / P;
            double2 x[N2];
#pragma unroll
            for (int n2 = 0; n2 < N2; ++n2) {
                const int j = n1 + N1 * n2;
                double2 hj, hh;
                if (j == 0) {
                    hj = make_double2(w1 * y[0].x, 0.0);
                    hh = make_double2(w1 * y[H].x, 0.0);
                } else {
                    const float2 a = y[j], b = y[H - j];
                    hj = make_double2(0.5 * (w2 * a.x), 0.5 * (w2 * a.y));
                    hh = make_double2(0.5 * (w2 * b.x), -0.5 * (w2 * b.y));
                }
                const double2 ev = sfft::d_add(hj, hh), od = sfft::d_mul(sfft::d_sub(hj, hh), wp[j]);
                x[n2] = make_double2(ev.x - od.y, -(ev.y + od.x));   // conj(ev + i od)
            }
            sfft::DFFT<N2, N1>::run(x, tw);
            double2 *row = buf + (size_t)kl * N2 * (N1 + 1) + n1;
#pragma unroll
            for (int k2 = 0; k2 < N2; ++k2)
                row[k2 * (N1 + 1)] = (k2 == 0 || n1 == 0) ? x[k2] : sfft::d_mul(x[k2], tw[n1 * k2]);
        }
        __syncthreads();
        if (rb0 + NB < nr) fetch(rb0 + NB);
        for (int t = threadIdx.x; t < nb * N2; t += blockDim.x) {
            const int kl = t / N2, k2 = t - kl * N2;
            const double2 *row = buf + ((size_t)kl * N2 + k2) * (N1 + 1);
            double2 x[N1];
#pragma unroll
            for (int n1 = 0; n1 < N1; ++n1) x[n1] = row[n1];
            sfft::DFFT<N1, N2>::run(x, tw);
            float *dst = D + ((size_t)(rb0 + kl) * dcols + cl) * dlen;
#pragma unroll
            for (int k1 = 0; k1 < N1; ++k1) {
                const int l = k2 + N2 * k1;
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    const double d = b == 0 ? x[k1].x : -x[k1].y;   // D(2l + b)
                    const int rho = 2 * l + b;
                    // the FP32 factor 1/sqrt(D sqsum): D sqsum formed in FP64, its reciprocal square
                    // root in FP32 by rsqrtf and one Newton-Raphson step y (3 - a y^2) / 2
                    const float a = (float)(d * sq);
                    float y = rsqrtf(a);
                    y = y * fmaf(-0.5f * a, y * y, 1.5f);
                    if constexpr (p2 == 0) {
                        dst[rho] = y;
                    } else {
                        // the Euclidean objective: the additive term -(D + sum_k w_k |ptcl_k|^2) / 2,
                        // sq holding the weighted particle term
                        const float v = eu ? (float)(-0.5 * (d + sq)) : (float)dscale * y;
#pragma unroll
                        for (int hh = 0; hh < 2; ++hh) {   // rot = rho and rho + P
                            const int rot = rho + hh * P, lr = rot >> 1, l2 = lr % p2;
                            float *o = dst + ((((l2 >> 1) * p1 + lr / p2) * 2 + (rot & 1)) * 2 + (l2 & 1));
                            o[0] = v;
                            if ((p2 & 1) && l2 == p2 - 1) o[1] = v;
                        }
                    }
                }
            }
        }
    }
}

template <int N1, int N2, int P2C>
static cudaError_t launch_norm_fft_k(pftcc_handle *h, const float2 *Y, int nr, int c0, int ncols, int dcols,
                                     const float *sqp, float *D, double dscale, int eu)
{
    constexpr int H = N1 * N2, NB = 256 / (N1 > N2 ? N1 : N2);
    const size_t smem = (size_t)(2 * H + NB * N2 * (N1 + 1)) * sizeof(double2) + (size_t)NB * (H + 1) * sizeof(float2);
    cudaError_t e = smem_limit((const void *)k_norm_fft<N1, N2, P2C>, smem);
    if (e != cudaSuccess) return e;
    k_norm_fft<N1, N2, P2C><<<ncols, 256, smem, h->stream>>>(Y, nr, c0, ncols, dcols, sqp, D, dscale, eu);
    return cudaGetLastError();
}

// the natural layout (p2 == 0) or the stage-2 split of the length (the only split served)
template <int N1, int N2, int P2F>
static cudaError_t launch_norm_fft(pftcc_handle *h, const float2 *Y, int nr, int c0, int ncols, int dcols,
                                   const float *sqp, float *D, int p2, double dscale, int eu)
{
    if (p2 == 0) return launch_norm_fft_k<N1, N2, 0>(h, Y, nr, c0, ncols, dcols, sqp, D, dscale, eu);
    if (p2 == P2F) return launch_norm_fft_k<N1, N2, P2F>(h, Y, nr, c0, ncols, dcols, sqp, D, dscale, eu);
    return cudaErrorInvalidValue;
}

static cudaError_t launch_norm(pftcc_handle *h, const Geom &g, const float2 *RUf, int nrefs_p, const float2 *CVf,
                               int cols_pad, int r0, int nr, int c0, int ncols, int dcols, const float *sqp, float2 *Y,
                               float *D, int p2, double dscale, int eu)
{
    const int J = g.P / 2 + 1;
    cudaError_t e;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_NORM);
    {
        dim3 grid((ncols + NY2_C - 1) / NY2_C, (nr + NY2_R - 1) / NY2_R, J);
        e = smem_limit((const void *)k_norm_y2, NY2_SMEM);
        if (e != cudaSuccess) return e;
        k_norm_y2<<<grid, 128, NY2_SMEM, h->stream>>>(g.Ks, J, RUf, nrefs_p, CVf, cols_pad, r0, nr, c0, ncols, Y);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    PFTCC_LAUNCH(h);
    switch (g.P) {
    case 64: return launch_norm_fft<8, 4, 8>(h, Y, nr, c0, ncols, dcols, sqp, D, p2, dscale, eu);
    case 180: return launch_norm_fft<10, 9, 15>(h, Y, nr, c0, ncols, dcols, sqp, D, p2, dscale, eu);
    case 300: return launch_norm_fft<15, 10, 20>(h, Y, nr, c0, ncols, dcols, sqp, D, p2, dscale, eu);
    default: break;
    }
    if (eu) return cudaErrorInvalidValue;   // the Euclidean objective needs the transform lengths above
    const size_t smem = ((size_t)NORM_RB * (J | 1) + g.P) * sizeof(double2);
    if (g.P % 4 == 0) {
        if ((e = smem_limit((const void *)k_norm<4>, smem))) return e;
        k_norm<4><<<ncols, 256, smem, h->stream>>>(g, Y, nr, c0, ncols, dcols, sqp, D, p2, dscale);
    } else if (g.P % 2 == 0) {
        if ((e = smem_limit((const void *)k_norm<2>, smem))) return e;
        k_norm<2><<<ncols, 256, smem, h->stream>>>(g, Y, nr, c0, ncols, dcols, sqp, D, p2, dscale);
    } else {
        if ((e = smem_limit((const void *)k_norm<1>, smem))) return e;
        k_norm<1><<<ncols, 256, smem, h->stream>>>(g, Y, nr, c0, ncols, dcols, sqp, D, p2, dscale);
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// stage 2: per (col, row) the length-P FFT of Z(j) = [X(j) + conj X(P-j)] +
// i [X(j) - conj X(P-j)] w_N^{-j} gives z(l) = y(2l) + i y(2l+1), y(rot) =
// sum_{m<N} X(m) w_N^{-m rot}; cc(rot) = (2/N) y / sqrt(D(rot mod P) * sqsum_ptcl).
// One block per particle column; each thread transforms whole rows in its own
// shared-memory slab (element-major, thread-minor: conflict-free), digit-reversed
// on load so the in-place decimation-in-time passes leave natural order.
struct S2Params {
    int N, P, nf, T;
    int f[MAXF];
    int rows;          // rows of the wave (local)
    int xrows, xcols;  // X dims
    int row0;          // global row of local row 0
    int nshifts;
    int r0;            // first reference of the wave's D
    int dcols;         // D column stride
    int col0;          // global column of the wave's first column
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }

__global__ void k_stage2(S2Params sp, const float2 *__restrict__ X, const float *__restrict__ D,
                         const float *__restrict__ sqp, const int *__restrict__ rev, float2 *__restrict__ cand,
                         float *__restrict__ ccall, const int *__restrict__ perm, int nrs_total)
{
    extern __shared__ float4 smem4[];
    const int P = sp.P, N = sp.N, T = sp.T;
    float2 *twP = reinterpret_cast<float2 *>(smem4);   // [P] w_P^{-e}
    float2 *twN = twP + P;                             // [P] w_N^{-j}
    float2 *buf = twN + P;                             // [P][T]
    float *ccs = reinterpret_cast<float *>(buf + (size_t)P * T);   // [rows + 8]
    int *ids = reinterpret_cast<int *>(ccs + sp.rows + 8);         // [rows + 8]
    const int cl = blockIdx.x;           // local column
    const int t = threadIdx.x;
    for (int e = t; e < P; e += T) {
        double sn, cs;
        sincospi(-2.0 * e / P, &sn, &cs);
        twP[e] = make_float2((float)cs, (float)sn);
        sincospi(-2.0 * e / N, &sn, &cs);
        twN[e] = make_float2((float)cs, (float)sn);
    }
    __syncthreads();
    const size_t plane = (size_t)sp.xcols * sp.xrows;
    const float2 *Xc = X + (size_t)cl * sp.xrows;
    // X carries the factor 4 of the half-circle transforms; y/(2N) is the correlation sum
    const float scale = 1.0f / (2.0f * (float)N);
    for (int row = t; row < sp.rows; row += T) {
        // the packed spectrum Z as stage 1 stored it, digit-reversed into the slab
        for (int j = 0; j < P; ++j) buf[(size_t)rev[j] * T + t] = Xc[(size_t)j * plane + row];
        // in-place mixed-radix DIT passes, innermost radix first
        int span = 1;   // m_l of the current level
        for (int l = sp.nf - 1; l >= 0; --l) {
            const int r = sp.f[l];
            const int nl = span * r;
            const int tstep = P / nl, rstep = P / r;
            for (int b0 = 0; b0 < P; b0 += nl) {
                for (int k = 0; k < span; ++k) {
                    float2 y[8];
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        if (q < r) {
                            const float2 v = buf[(size_t)(b0 + q * span + k) * T + t];
                            y[q] = (q == 0 || k == 0) ? v : cmul(v, twP[(q * k * tstep) % P]);
                        }
                    }
#pragma unroll
                    for (int s = 0; s < 8; ++s) {
                        if (s < r) {
                            float2 acc = y[0];
#pragma unroll
                            for (int q = 1; q < 8; ++q)
                                if (q < r) {
                                    const float2 w = twP[((q * s) % r) * rstep];
                                    acc.x += y[q].x * w.x - y[q].y * w.y;
                                    acc.y += y[q].x * w.y + y[q].y * w.x;
                                }
                            buf[(size_t)(b0 + s * span + k) * T + t] = acc;
                        }
                    }
                }
            }
            span = nl;
        }
        // correlations and the argmax over rotations (lowest rotation on ties)
        const int grow = sp.row0 + row;
        const int rl = grow / sp.nshifts - sp.r0;
        const float *Dr = D + ((size_t)rl * sp.dcols + cl) * P;
        float best = -INFINITY;
        int brot = 0;
        float *cc_out = ccall ? ccall + ((size_t)perm[sp.col0 + cl] * nrs_total + grow) * N : nullptr;
        for (int l = 0; l < P; ++l) {
            const float2 z = buf[(size_t)l * T + t];
            const int r0 = 2 * l, r1 = 2 * l + 1;
            const float c0 = scale * z.x * Dr[r0 % P];
            const float c1 = scale * z.y * Dr[r1 % P];
            if (cc_out) { cc_out[r0] = c0; cc_out[r1] = c1; }
            if (c0 > best) { best = c0; brot = r0; }
            if (c1 > best) { best = c1; brot = r1; }
        }
        ccs[row] = best;
        ids[row] = grow * N + brot;
    }
    // merge with the running top-8 of this particle
    float2 *cp = cand + (size_t)(sp.col0 + cl) * 8;
    if (t < 8) {
        const float2 c = cp[t];
        ccs[sp.rows + t] = c.x;
        ids[sp.rows + t] = __float_as_int(c.y);
    }
    __syncthreads();
    if (t < 32) {
        const int n = sp.rows + 8;
        float sel_cc[8];
        int sel_id[8];
        for (int it = 0; it < 8; ++it) {
            float bc = -INFINITY;
            int bi = 0x7fffffff, bpos = -1;
            for (int e = t; e < n; e += 32) {
                const float c = ccs[e];
                const int id = ids[e];
                if (c > bc || (c == bc && id < bi && c != -INFINITY)) { bc = c; bi = id; bpos = e; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const float oc = __shfl_xor_sync(0xffffffffu, bc, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                const int op = __shfl_xor_sync(0xffffffffu, bpos, o);
                if (oc > bc || (oc == bc && oi < bi)) { bc = oc; bi = oi; bpos = op; }
            }
            sel_cc[it] = bc;
            sel_id[it] = bi;
            if (bpos >= 0 && t == (bpos & 31)) ccs[bpos] = -INFINITY;
            __syncwarp();
        }
        if (t < 8) {
            float c = sel_cc[0];
            int id = sel_id[0];
#pragma unroll
            for (int it = 1; it < 8; ++it)
                if (t == it) { c = sel_cc[it]; id = sel_id[it]; }
            cp[t] = make_float2(c, __int_as_float(c == -INFINITY ? -1 : id));
        }
    }
}

// ---------------------------------------------------------------------------
__global__ void k_cand_init(float2 *cand, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n * 8) cand[i] = make_float2(-INFINITY, __int_as_float(-1));
}

// top-1 out of the candidates, or the work list of the exact re-score
__global__ void k_finish(const float2 *__restrict__ cand, const int *__restrict__ perm, int ncols, int N, int nshifts,
                         int has_shifts, int ntop, pftcc_best *__restrict__ out, Work *__restrict__ work,
                         Group *__restrict__ groups)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncols) return;
    const float2 *cp = cand + (size_t)c * 8;
    const int slot = perm[c];
    if (ntop == 0) {
        const int id = __float_as_int(cp[0].y);
        pftcc_best b;
        if (id < 0) { b.iref = 0; b.irot = 0; b.ishift = -1; b.corr = -INFINITY; }
        else {
            const int rs = id / N, rot = id - rs * N;
            b.iref = rs / nshifts + 1;
            b.ishift = has_shifts ? rs % nshifts : -1;
            b.irot = rot + 1;
            b.corr = cp[0].x;
        }
        out[slot] = b;
        return;
    }
    int cnt = 0;
    for (int i = 0; i < ntop; ++i) {
        const int id = __float_as_int(cp[i].y);
        if (id < 0) continue;
        const int rs = id / N;
        work[(size_t)c * ntop + cnt] = Work{rs / nshifts, has_shifts ? rs % nshifts : -1, 0};
        ++cnt;
    }
    groups[c] = Group{slot, c * ntop, cnt, slot};
}

// ---------------------------------------------------------------------------
static int ensure_ws(pftcc_handle *h, void **p, size_t bytes, const char *what)
{
    // workspace buffers grow monotonically; size kept implicitly by the caller's max
    return dev_alloc(h, p, bytes, what);
}

struct WsSizes { size_t UA, UB, RU, CV, D, X, cand, sqp, perm; };

// The Euclidean objective in the particle CTF frame (gencorrs_euclid_1/_2 with the CTF at the
// particle's polar index, as the correlation of this search): for column c (particle slot perm[c])
// the shell weights w_k = pxls(k) / (P sigma2(k)) scale its spectra UB (the correlation term) and
// CV (CTF^2, the reference-energy term), and sqp[c] becomes sum_{k<=kstop} w_k sum_n |ptcl(n,k)|^2,
// so that the search scores sum_k w_k (corr_k - (E_ref,k(rot) + E_ptcl,k) / 2).  One block per column.
__global__ void __launch_bounds__(256) k_euclid_weigh(Geom g, int np, int cols_pad, int M, const int *__restrict__ perm,
                                                      const float *__restrict__ sig2, const float *__restrict__ pxls,
                                                      const float2 *__restrict__ ptcls, float2 *__restrict__ UB,
                                                      double2 *__restrict__ CV, float *__restrict__ sqp)
{
    __shared__ double w[64];
    __shared__ double red[8];
    const int c = blockIdx.x;
    if (c >= np) return;
    const int slot = perm[c], Ks = g.Ks, P = g.P, J = P / 2 + 1;
    for (int k = threadIdx.x; k < Ks; k += blockDim.x)
        w[k] = (double)pxls[k] / ((double)P * (double)sig2[(size_t)slot * g.K + k]);
    __syncthreads();
    for (int e = threadIdx.x; e < M * Ks; e += blockDim.x) {
        const int m = e / Ks, k = e - m * Ks;
        float2 *u = UB + ((size_t)m * cols_pad + c) * Ks + k;
        const float wk = (float)w[k];
        *u = make_float2(u->x * wk, u->y * wk);
    }
    for (int e = threadIdx.x; e < J * Ks; e += blockDim.x) {
        const int k = e % Ks;
        double2 *v = CV + (size_t)c * J * Ks + e;
        *v = make_double2(v->x * w[k], v->y * w[k]);
    }
    double s = 0.0;
    const float2 *q = ptcls + (size_t)slot * g.K * P;
    for (int e = threadIdx.x; e < Ks * P; e += blockDim.x) {
        const float2 v = q[e];
        s += w[e / P] * ((double)v.x * v.x + (double)v.y * v.y);
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < 8; ++i) t += red[i];
        sqp[c] = (float)t;
    }
}

int search_mdomain(pftcc_handle *h, int nshifts_in, const float *shifts_host, int precision, int ntop, pftcc_best *out_dev,
                   float *ccall_dev)
{
    const Geom &g = h->g;
    const int N = g.N, P = g.P, Ks = g.Ks, M = P + 1, J = P / 2 + 1;
    const int eu = h->objfun == PFTCC_OBJFUN_EUCLID;
    if (eu && (h->cfg.ctf_frame != PFTCC_FRAME_PTCL || !stage2_fast_supported(P)))
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "the m-domain Euclidean objective is served in the particle CTF frame "
                                                 "for nrots/2 in {64, 180, 300}; use PFTCC_PREC_EXACT in the reference frame");
    if (Ks > 64) return set_err(h, PFTCC_ERR_UNSUPPORTED, "m-domain search supports at most 64 shells");
    const FFTPlan plan = make_plan(P);
    for (int i = 0; i < plan.nf; ++i)
        if (plan.f[i] > 8) return set_err(h, PFTCC_ERR_UNSUPPORTED, "m-domain search needs nrots/2 with prime factors <= 7");
    const int ns = std::max(1, nshifts_in);
    const long long nrs_ll = (long long)h->nrefs * ns;
    if (nrs_ll * N >= (1LL << 31)) return set_err(h, PFTCC_ERR_ARG, "nrefs * nshifts * nrots too large for candidate ids");
    const int nrs = (int)nrs_ll;
    const int np = h->nptcls;
    SearchWS &ws = h->ws;
    // parity groups: columns ordered even slots first, then odd slots
    std::vector<int> perm;
    perm.reserve(np);
    for (int i = 0; i < np; ++i) if (h->iseven[i]) perm.push_back(i);
    const int n_even = (int)perm.size();
    for (int i = 0; i < np; ++i) if (!h->iseven[i]) perm.push_back(i);
    // columns in tiles of COL_TILE (the tcgen05 M tile): a parity group may start
    // mid-tile, so one spare tile of zero columns
    const int cols_pad = (np + COL_TILE - 1) / COL_TILE * COL_TILE + COL_TILE;
    const int rows_pad = (nrs + S1_TILE - 1) / S1_TILE * S1_TILE;
    // wave sizes: rows x cols per stage-1/stage-2 round; automatic: 4096 x up to 4096 with the
    // stage-1 output X within 8 GiB; a tuning (pftcc_set_tuning / the autotuner) may ask for other
    // sizes, X then within 24 GiB
    int W_rows = std::min(rows_pad, 4096);
    int W_cols = std::min(cols_pad - COL_TILE, 4096);
    size_t x_budget = 8ull << 30;
    if (h->tune.w_rows > 0) { W_rows = std::min(rows_pad, std::max(S1_TILE, h->tune.w_rows / S1_TILE * S1_TILE)); x_budget = 24ull << 30; }
    if (h->tune.w_cols > 0) { W_cols = std::min(cols_pad - COL_TILE, std::max(COL_TILE, h->tune.w_cols / COL_TILE * COL_TILE)); x_budget = 24ull << 30; }
    while ((size_t)M * W_rows * W_cols * sizeof(float2) > x_budget && W_cols > COL_TILE) W_cols /= 2;
    W_cols = std::max(COL_TILE, W_cols / COL_TILE * COL_TILE);
    // compile-time transforms for the common lengths; the generic radix loop otherwise, whose
    // shared memory holds a (cc, id) pair per wave row: its rows are capped to fit 227 KB
    const bool fast_s2 = stage2_fast_supported(P);
    int T = 128;
    while (T > 32 && (size_t)P * T * sizeof(float2) > 180 * 1024) T -= 32;
    auto smem_generic = [&](int rows) {
        return 2 * (size_t)P * sizeof(float2) + (size_t)P * T * sizeof(float2) +
               (size_t)(rows + 8) * (sizeof(float) + sizeof(int));
    };
    if (!fast_s2)
        while (smem_generic(W_rows) > 227 * 1024 && W_rows > S1_TILE) W_rows = std::max(S1_TILE, W_rows / 2 / S1_TILE * S1_TILE);
    const int nr_wave_max = (W_rows + ns - 1) / ns + 2;
    // (re)allocate the workspace when the geometry, the counts or the wave change
    const bool realloc = ws.nrs_pad != rows_pad || ws.np_pad != cols_pad || ws.nshifts != ns || ws.M != M ||
                         ws.W_rows != W_rows || ws.W_cols != W_cols;
    if (realloc) {
        void *bufs[] = {ws.UA, ws.UB, ws.RU, ws.CV, ws.RUf, ws.CVf, ws.D, ws.Yn, ws.X, ws.cand, ws.sqp, ws.shifts,
                        ws.cand_ref, ws.A16, ws.B16, ws.best};
        for (void *b : bufs) dev_free(h, b);
        umma_free(h);
        ws = SearchWS{};
        int st;
        if ((st = ensure_ws(h, (void **)&ws.UA, (size_t)M * rows_pad * Ks * sizeof(float2), "UA")) ||
            (st = ensure_ws(h, (void **)&ws.UB, (size_t)M * cols_pad * Ks * sizeof(float2), "UB")) ||
            (st = ensure_ws(h, (void **)&ws.RU, (size_t)h->nrefs * J * Ks * sizeof(double2), "RU")) ||
            (st = ensure_ws(h, (void **)&ws.CV, (size_t)cols_pad * J * Ks * sizeof(double2), "CV")) ||
            (st = ensure_ws(h, (void **)&ws.D, (size_t)nr_wave_max * W_cols * std::max(2 * P, stage2_fast_dlen(P)) * sizeof(float), "D")) ||
            (st = ensure_ws(h, (void **)&ws.RUf, (size_t)h->nrefs * J * Ks * sizeof(float2), "RUf")) ||
            (st = ensure_ws(h, (void **)&ws.CVf, (size_t)cols_pad * J * Ks * sizeof(float2), "CVf")) ||
            (st = ensure_ws(h, (void **)&ws.Yn, (size_t)nr_wave_max * W_cols * J * sizeof(float2), "Y")) ||
            (st = ensure_ws(h, (void **)&ws.X, (size_t)M * W_rows * W_cols * sizeof(float2), "X")) ||
            (st = ensure_ws(h, (void **)&ws.cand, (size_t)cols_pad * 8 * sizeof(float2), "cand")) ||
            (st = ensure_ws(h, (void **)&ws.sqp, (size_t)cols_pad * sizeof(float), "sqp")) ||
            (st = ensure_ws(h, (void **)&ws.shifts, (size_t)ns * 2 * sizeof(float) + 64, "shifts")) ||
            (st = ensure_ws(h, (void **)&ws.cand_ref, (size_t)cols_pad * sizeof(int) + (size_t)P * sizeof(int), "perm")))
            return st;
        ws.nrs_pad = rows_pad; ws.np_pad = cols_pad; ws.nshifts = ns; ws.M = M; ws.nrs = nrs;
        ws.W_rows = W_rows; ws.W_cols = W_cols;
        ws.X_elems = (size_t)M * W_rows * W_cols;
    }
    int *d_perm = ws.cand_ref;
    int *d_rev = ws.cand_ref + cols_pad;
    // the stage-2 kernel writes input j at slab position digit_rev(j)
    std::vector<int> rev(P);
    for (int j = 0; j < P; ++j) rev[j] = digit_rev(plan, P, j);
    cudaError_t e;
#define CKE(x, w) do { e = (x); if (e != cudaSuccess) return cuda_err(h, e, w); } while (0)
    CKE(cudaMemcpyAsync(d_perm, perm.data(), np * sizeof(int), cudaMemcpyHostToDevice, h->stream), "perm");
    CKE(cudaMemcpyAsync(d_rev, rev.data(), P * sizeof(int), cudaMemcpyHostToDevice, h->stream), "rev");
    std::vector<float> sh(2 * ns, 0.f);
    if (nshifts_in > 0) std::copy(shifts_host, shifts_host + 2 * ns, sh.begin());
    CKE(cudaMemcpyAsync(ws.shifts, sh.data(), sh.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream), "shifts");
    const float *ctf = (h->cfg.with_ctf && h->ctf_ready) ? h->ctfmats : nullptr;
    // particle spectra and CTF^2 spectra
    {
        KTimer kt(h, PFTCC_K_SPEC_PTCL);
        CKE(launch_spec_ptcl(h, g, ctf, d_perm, np, cols_pad, ws.UB, ws.CV, ws.sqp), "spec_ptcl");
        if (eu) {   // shell weights into the particle side, the weighted particle term into sqp
            PFTCC_LAUNCH(h);
            k_euclid_weigh<<<np, 256, 0, h->stream>>>(g, np, cols_pad, M, d_perm, h->d_sig2, h->d_pxls, h->ptcls,
                                                      ws.UB, ws.CV, ws.sqp);
            CKE(cudaGetLastError(), "euclid weights");
        }
        PFTCC_LAUNCH(h);
        k_norm_cvt<<<CVT_BLOCKS, 256, 0, h->stream>>>(np, J, Ks, cols_pad, ws.CV, ws.CVf);
        CKE(cudaGetLastError(), "CV copy");
        PFTCC_LAUNCH(h);
        k_cand_init<<<(cols_pad * 8 + 255) / 256, 256, 0, h->stream>>>(ws.cand, cols_pad);
        CKE(cudaGetLastError(), "cand_init");
    }
    const size_t smem_s1 = 4 * (size_t)Ks * S1_TILE * sizeof(float2);
    CKE(smem_limit((const void *)k_stage1_fp32, smem_s1), "attr");
    const size_t smem_s2 = smem_generic(W_rows);
    if (!fast_s2) CKE(smem_limit((const void *)k_stage2, smem_s2), "attr");
    S2Params sp{};
    sp.N = N; sp.P = P; sp.nf = plan.nf; sp.T = T;
    for (int i = 0; i < plan.nf; ++i) sp.f[i] = plan.f[i];
    sp.nshifts = ns;
    // the top-ntop re-score: FP32 m-domain in the particle frame, the exact kernel in
    // the reference frame
    const bool md_rescore = ntop > 0 && fast_s2 && h->cfg.ctf_frame == PFTCC_FRAME_PTCL;
    if (precision == PFTCC_PREC_BF16X3) {
        const int st = umma_reset(h);
        if (st != PFTCC_OK) return st;
    }
    for (int grp = 0; grp < 2; ++grp) {
        const int gc0 = grp == 0 ? 0 : n_even, gc1 = grp == 0 ? n_even : np;
        if (gc1 <= gc0) continue;
        const float2 *refs = grp == 0 ? h->refs_even : h->refs_odd;
        { KTimer kt(h, PFTCC_K_SPEC_REF);
        CKE(launch_spec_r2(h, g, refs, ws.RU), "spec_r2");
        CKE(launch_spec_ref(h, g, ns, refs, ws.shifts, nrs, rows_pad, ws.UA), "spec_ref");
        if (h->cfg.match_filt)   // the references' shell factors (shellnorm_and_filter_ref) on their spectra
            CKE(launch_shellnorm_apply(h, M, nrs, rows_pad, ns, grp, ws.UA, ws.RU), "shell factors");
        PFTCC_LAUNCH(h);
        k_norm_cvt<<<CVT_BLOCKS, 256, 0, h->stream>>>(h->nrefs, J, Ks, h->nrefs, ws.RU, ws.RUf);
        CKE(cudaGetLastError(), "RU copy"); }
        if (precision == PFTCC_PREC_BF16X3) {
            int st = umma_stage1(h, M, Ks, ws.UA, 0, nrs, rows_pad, ws.UB, gc0, gc1 - gc0, cols_pad, nullptr, 1, grp);
            if (st != PFTCC_OK) return st;
        }
        for (int row0 = 0; row0 < nrs; row0 += W_rows) {
            const int rows = std::min(W_rows, nrs - row0);
            const int rows_t = (rows + S1_TILE - 1) / S1_TILE * S1_TILE;
            const int r_lo = row0 / ns, r_hi = (row0 + rows - 1) / ns;
            for (int c0 = gc0; c0 < gc1; c0 += W_cols) {
                const int cols = std::min(W_cols, gc1 - c0);
                const int cols_t = (cols + COL_TILE - 1) / COL_TILE * COL_TILE;
                if (precision == PFTCC_PREC_BF16X3) {
                    int st = umma_stage1(h, M, Ks, ws.UA, row0, rows_t, rows_pad, ws.UB, c0, cols_t, cols_pad, ws.X, 0, grp);
                    if (st != PFTCC_OK) return st;
                } else {
                    dim3 grid(rows_t / S1_TILE, cols_t / S1_TILE, P / 2 + 1);
                    PFTCC_LAUNCH(h);
                    KTimer kt(h, PFTCC_K_STAGE1);
                    k_stage1_fp32<<<grid, 256, smem_s1, h->stream>>>(Ks, P, ws.UA, rows_pad, row0, ws.UB, cols_pad, c0,
                                                                    ws.X, rows_t, cols_t);
                    CKE(cudaGetLastError(), "stage1");
                }
                // the split-radix stage 2 reads the factor in its visiting order, times 1/(2N)
                CKE(launch_norm(h, g, ws.RUf, h->nrefs, ws.CVf, cols_pad, r_lo, r_hi - r_lo + 1, c0, cols, cols_t,
                                ws.sqp, ws.Yn, ws.D,
                                fast_s2 ? stage2_fast_p2(P) : 0, 1.0 / (2.0 * N), eu), "norm");
                if (fast_s2) {
                    e = launch_stage2_fast(h, P, rows, rows_t, cols_t, row0, ns, r_lo, cols_t, c0, cols, nrs, ws.X, ws.D,
                                           ws.cand, ccall_dev, d_perm, eu);
                    if (e != cudaSuccess)
                        return set_err(h, e == cudaErrorMemoryAllocation ? PFTCC_ERR_OOM : PFTCC_ERR_CUDA,
                                       "stage2 (P " + std::to_string(P) + ", rows " + std::to_string(rows) + ", columns " +
                                           std::to_string(cols) + "): " + cudaGetErrorString(e));
                } else {
                    sp.rows = rows; sp.xrows = rows_t; sp.xcols = cols_t; sp.row0 = row0; sp.r0 = r_lo;
                    sp.dcols = cols_t; sp.col0 = c0;
                    PFTCC_LAUNCH(h);
                    KTimer kt(h, PFTCC_K_STAGE2);
                    k_stage2<<<cols, T, smem_s2, h->stream>>>(sp, ws.X, ws.D, ws.sqp, d_rev, ws.cand, ccall_dev, d_perm, nrs);
                    CKE(cudaGetLastError(), "stage2");
                }
            }
        }
        // particle-frame re-score from this group's FP32 spectra (before the next group
        // overwrites them)
        if (md_rescore && out_dev)
            CKE(launch_rescore_md(h, P, gc1 - gc0, ntop, Ks, ns, nshifts_in > 0, ws.UA, rows_pad, ws.UB, cols_pad,
                                  ws.RU, ws.CV, ws.sqp, ws.cand, d_perm, gc0, out_dev, eu), "rescore");
    }
    if (precision == PFTCC_PREC_BF16X3) {
        int st = umma_check(h);
        if (st != PFTCC_OK) return st;
    }
    // finish: top-1 or the exact re-score of the best ntop (ref, shift) per particle
    if (!out_dev || md_rescore) return PFTCC_OK;
    if (ntop == 0) {
        PFTCC_LAUNCH(h);
        k_finish<<<(np + 127) / 128, 128, 0, h->stream>>>(ws.cand, d_perm, np, N, ns, nshifts_in > 0, 0, out_dev, nullptr,
                                                      nullptr);
        CKE(cudaGetLastError(), "finish");
        return PFTCC_OK;
    }
    if (eu) return set_err(h, PFTCC_ERR_UNSUPPORTED, "the m-domain Euclidean objective re-scores in the m-domain");
    int st = ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>((size_t)np * ntop * sizeof(Work), 4096), "work");
    if (st) return st;
    st = ensure(h, (void **)&h->d_groups, &h->group_cap, std::max<size_t>((size_t)np * sizeof(Group), 256), "groups");
    if (st) return st;
    PFTCC_LAUNCH(h);
    k_finish<<<(np + 127) / 128, 128, 0, h->stream>>>(ws.cand, d_perm, np, N, ns, nshifts_in > 0, ntop, out_dev,
                                                      h->d_work, h->d_groups);
    CKE(cudaGetLastError(), "finish");
    CKE(launch_exact(h, h->d_groups, np, h->d_work, ws.shifts, MODE_BEST, exact_frame(h), 1, nullptr, out_dev),
        "rescore");
#undef CKE
    return PFTCC_OK;
}

}  // namespace pftcc

namespace pftcc {

cudaError_t launch_stage2_waves(pftcc_handle *h, int P, std::vector<S2Wave> &waves, int nshifts, int nrs_total,
                                float2 *cand, float *ccall, const int *perm, int eu);

// every held particle's best out of a searched group starts as "not searched" (reference 0)
__global__ void k_best_clear(pftcc_best *out, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = pftcc_best{0, 0, -1, -INFINITY};
}

// The grouped search: group q searches the particle slots [slot0[q], slot0[q] + nslot[q]) against
// the references [ref0[q], ref0[q] + nref[q]) (0-based), as search_mdomain searches all of them
// against all references.  The columns are ordered by parity, then group; consecutive groups of a
// parity form column batches of at most GB_COLS particles (a larger group is a batch of its own),
// whose spectra, packed operands and candidates are formed per batch, so that the workspace scales
// with the batch and not with the queue.  Each (parity, group) block of columns against its group's
// (reference, shift) rows is one wave, cut into several where its packed spectrum would pass the
// per-wave budget; the waves of a batch run as ONE persistent tcgen05 stage-1 launch over all their
// work items (the device wave table, umma_stage1_waves), the normaliser per wave, and ONE stage-2
// launch over all their columns (launch_stage2_waves).  A wave's stage-1 tiles are aligned (64
// rows, 128 columns) and may take in a neighbouring group's rows or particles, which its stage 2
// then leaves out.
constexpr int GB_COLS = 8192;

int search_mdomain_groups(pftcc_handle *h, int ngroups, const int *ref0, const int *nref, const int *slot0,
                          const int *nslot, int nshifts_in, const float *shifts_host, int precision, int ntop,
                          pftcc_best *out_dev, int check)
{
    const Geom &g = h->g;
    // the tables of this call go through the staging arena of its kind: outside capture the stream
    // drains first (the arena's earlier contents have landed) and the call's staging bytes are
    // recorded, so that the capture arena can be sized for a later capture of the same call
    const bool cap = capturing(h);
    if (cap) {
        h->pin_off[1] = 0;
        if (h->pin_cap[1] < h->pin_need || !h->pin[1])
            return set_err(h, PFTCC_ERR_STATE, "search_groups during graph capture: run the same call once outside capture first");
    } else {
        const cudaError_t e0 = cudaStreamSynchronize(h->stream);
        if (e0 != cudaSuccess) return cuda_err(h, e0, "search_groups");
        h->pin_off[0] = 0;
        h->pin_total = 0;
    }
    const int N = g.P * 2, P = g.P, Ks = g.Ks, M = P + 1, J = P / 2 + 1;
    if (h->objfun == PFTCC_OBJFUN_EUCLID)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "search_groups: the correlation objective only");
    if (!stage2_fast_supported(P))
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "search_groups: nrots/2 in {64, 180, 300}");
    if (Ks > 64) return set_err(h, PFTCC_ERR_UNSUPPORTED, "m-domain search supports at most 64 shells");
    if (precision != PFTCC_PREC_BF16X3 && precision != PFTCC_PREC_FP32)
        return set_err(h, PFTCC_ERR_ARG, "search_groups: precision FP32 or BF16X3");
    const int ns = std::max(1, nshifts_in);
    const long long nrs_ll = (long long)h->nrefs * ns;
    if (nrs_ll * N >= (1LL << 31)) return set_err(h, PFTCC_ERR_ARG, "nrefs * nshifts * nrots too large for candidate ids");
    const int nrs = (int)nrs_ll;
    // the groups: particle ranges disjoint and within the held slots, reference ranges within nrefs
    std::vector<int> owner(h->nptcls, -1);
    for (int q = 0; q < ngroups; ++q) {
        if (nref[q] < 1 || ref0[q] < 0 || ref0[q] + nref[q] > h->nrefs || nslot[q] < 0 || slot0[q] < 0 ||
            slot0[q] + nslot[q] > h->nptcls)
            return set_err(h, PFTCC_ERR_INDEX, "search_groups: group " + std::to_string(q) + " outside the references or slots");
        for (int i = slot0[q]; i < slot0[q] + nslot[q]; ++i) {
            if (owner[i] >= 0) return set_err(h, PFTCC_ERR_ARG, "search_groups: groups share particle slot " + std::to_string(i + 1));
            owner[i] = q;
        }
    }
    // columns: even slots first, then odd, each parity in group order
    std::vector<int> perm;
    std::vector<int> cb(2 * ngroups), ce(2 * ngroups);
    for (int par = 0; par < 2; ++par)
        for (int q = 0; q < ngroups; ++q) {
            cb[2 * q + par] = (int)perm.size();
            for (int i = slot0[q]; i < slot0[q] + nslot[q]; ++i)
                if ((h->iseven[i] != 0) == (par == 0)) perm.push_back(i);
            ce[2 * q + par] = (int)perm.size();
        }
    const int np = (int)perm.size();
    // column batches: (parity, first group, end group, first column, columns)
    struct Batch { int par, q0, q1, c0, n; };
    std::vector<Batch> batches;
    int widest = 0;
    for (int par = 0; par < 2; ++par)
        for (int q = 0; q < ngroups;) {
            int q1 = q, n = 0;
            while (q1 < ngroups) {
                const int w = ce[2 * q1 + par] - cb[2 * q1 + par];
                if (q1 > q && n + w > GB_COLS) break;
                n += w;
                ++q1;
            }
            if (n > 0) {
                batches.push_back(Batch{par, q, q1, cb[2 * q + par], n});
                widest = std::max(widest, n);
            }
            q = q1;
        }
    cudaError_t e;
#define CKG(x, w) do { e = (x); if (e != cudaSuccess) return cuda_err(h, e, w); } while (0)
    PFTCC_LAUNCH(h);
    k_best_clear<<<(h->nptcls + 255) / 256, 256, 0, h->stream>>>(out_dev, h->nptcls);
    CKG(cudaGetLastError(), "clear");
    if (np == 0) return PFTCC_OK;
    const int cols_pad = (widest + COL_TILE - 1) / COL_TILE * COL_TILE + COL_TILE;   // one batch's columns
    const int rows_pad = (nrs + S1_TILE - 1) / S1_TILE * S1_TILE;
    SearchWS &ws = h->ws;
    // the spectra and candidate buffers of one batch (marked as a grouped layout by W_rows = W_cols
    // = 0); the column order, the waves' packed spectra, normalising factors and Y grow as needed
    const bool realloc = ws.nrs_pad != rows_pad || ws.np_pad != cols_pad || ws.nshifts != ns || ws.M != M ||
                         ws.W_rows != 0 || ws.W_cols != 0;
    if (realloc) {
        void *bufs[] = {ws.UA, ws.UB, ws.RU, ws.CV, ws.RUf, ws.CVf, ws.D, ws.Yn, ws.X, ws.cand, ws.sqp, ws.shifts,
                        ws.cand_ref, ws.A16, ws.B16, ws.best};
        for (void *b : bufs) dev_free(h, b);
        umma_free(h);
        ws = SearchWS{};
        int st;
        if ((st = ensure_ws(h, (void **)&ws.UA, (size_t)M * rows_pad * Ks * sizeof(float2), "UA")) ||
            (st = ensure_ws(h, (void **)&ws.UB, (size_t)M * cols_pad * Ks * sizeof(float2), "UB")) ||
            (st = ensure_ws(h, (void **)&ws.RU, (size_t)h->nrefs * J * Ks * sizeof(double2), "RU")) ||
            (st = ensure_ws(h, (void **)&ws.CV, (size_t)cols_pad * J * Ks * sizeof(double2), "CV")) ||
            (st = ensure_ws(h, (void **)&ws.RUf, (size_t)h->nrefs * J * Ks * sizeof(float2), "RUf")) ||
            (st = ensure_ws(h, (void **)&ws.CVf, (size_t)cols_pad * J * Ks * sizeof(float2), "CVf")) ||
            (st = ensure_ws(h, (void **)&ws.cand, (size_t)cols_pad * 8 * sizeof(float2), "cand")) ||
            (st = ensure_ws(h, (void **)&ws.sqp, (size_t)cols_pad * sizeof(float), "sqp")) ||
            (st = ensure_ws(h, (void **)&ws.shifts, (size_t)ns * 2 * sizeof(float) + 64, "shifts")))
            return st;
        ws.nrs_pad = rows_pad; ws.np_pad = cols_pad; ws.nshifts = ns; ws.M = M; ws.nrs = nrs;
        ws.W_rows = 0; ws.W_cols = 0;
        ws.X_elems = 0;
    }
    {
        int st = ensure(h, (void **)&ws.cand_ref, &ws.perm_bytes, (size_t)np * sizeof(int), "column order");
        if (st) return st;
    }
    int *d_perm = ws.cand_ref;
    std::vector<float> sh(2 * ns, 0.f);
    if (nshifts_in > 0) std::copy(shifts_host, shifts_host + 2 * ns, sh.begin());
    {
        int st = stage_upload(h, d_perm, perm.data(), np * sizeof(int), "column order");
        if (st) return st;
        st = stage_upload(h, ws.shifts, sh.data(), sh.size() * sizeof(float), "shifts");
        if (st) return st;
    }
    const float *ctf = (h->cfg.with_ctf && h->ctf_ready) ? h->ctfmats : nullptr;
    const size_t smem_s1 = 4 * (size_t)Ks * S1_TILE * sizeof(float2);
    CKG(smem_limit((const void *)k_stage1_fp32, smem_s1), "attr");
    const int p2 = stage2_fast_p2(P), dlen = stage2_fast_dlen(P);
    const bool md_rescore = ntop > 0 && h->cfg.ctf_frame == PFTCC_FRAME_PTCL;
    {
        const int st = umma_reset(h);    // the device error word of the bounded waits (allocated once)
        if (st != PFTCC_OK) return st;
    }
    // a wave's packed spectrum within 1 GiB; a batch's waves within 2 GiB of Z and 1 GiB of factors
    // at a time
    const size_t z_wave_max = 1ull << 30, z_batch_max = 2ull << 30, d_batch_max = 1ull << 30;
    struct WavePlan { int r_lo, r_hi, a_lo, a_hi, c_lo, c_hi, t_lo, t_hi; };
    int cur_par = -1;
    for (const Batch &bt : batches) {
        const int par = bt.par;
        if (par != cur_par) {   // the reference side of this parity (all references)
            cur_par = par;
            const float2 *refs = par == 0 ? h->refs_even : h->refs_odd;
            KTimer kt(h, PFTCC_K_SPEC_REF);
            CKG(launch_spec_r2(h, g, refs, ws.RU), "spec_r2");
            CKG(launch_spec_ref(h, g, ns, refs, ws.shifts, nrs, rows_pad, ws.UA), "spec_ref");
            if (h->cfg.match_filt)
                CKG(launch_shellnorm_apply(h, M, nrs, rows_pad, ns, par, ws.UA, ws.RU), "shell factors");
            PFTCC_LAUNCH(h);
            k_norm_cvt<<<CVT_BLOCKS, 256, 0, h->stream>>>(h->nrefs, J, Ks, h->nrefs, ws.RU, ws.RUf);
            CKG(cudaGetLastError(), "RU copy");
        }
        // this batch's particles: columns bt.c0 .. bt.c0 + bt.n - 1 of the order, batch-local 0 .. n - 1
        const int *bperm = d_perm + bt.c0;
        {
            KTimer kt(h, PFTCC_K_SPEC_PTCL);
            CKG(launch_spec_ptcl(h, g, ctf, bperm, bt.n, cols_pad, ws.UB, ws.CV, ws.sqp), "spec_ptcl");
            PFTCC_LAUNCH(h);
            k_norm_cvt<<<CVT_BLOCKS, 256, 0, h->stream>>>(bt.n, J, Ks, cols_pad, ws.CV, ws.CVf);
            CKG(cudaGetLastError(), "CV copy");
            PFTCC_LAUNCH(h);
            k_cand_init<<<(cols_pad * 8 + 255) / 256, 256, 0, h->stream>>>(ws.cand, cols_pad);
            CKG(cudaGetLastError(), "cand_init");
        }
        if (precision == PFTCC_PREC_BF16X3) {
            int st = umma_stage1(h, M, Ks, ws.UA, 0, nrs, rows_pad, ws.UB, 0, bt.n, cols_pad, nullptr, 1, par);
            if (st != PFTCC_OK) return st;
        }
        // the batch's waves: per group, rows cut to keep a wave's Z within its budget
        std::vector<WavePlan> plan;
        for (int q = bt.q0; q < bt.q1; ++q) {
            const int c_lo = cb[2 * q + par] - bt.c0, c_hi = ce[2 * q + par] - bt.c0;
            if (c_hi <= c_lo) continue;
            const int t_lo = c_lo / COL_TILE, t_hi = (c_hi + COL_TILE - 1) / COL_TILE;
            const size_t zcol = (size_t)(t_hi - t_lo) * COL_TILE * P * sizeof(float2);   // Z bytes per row
            int rows_max = (int)std::max<size_t>(S1_TILE, z_wave_max / zcol / S1_TILE * S1_TILE);
            for (int r_lo = ref0[q] * ns, r_end = (ref0[q] + nref[q]) * ns; r_lo < r_end;) {
                const int a_lo = r_lo / S1_TILE * S1_TILE;
                const int r_hi = std::min(r_end, a_lo + rows_max);
                const int a_hi = (r_hi + S1_TILE - 1) / S1_TILE * S1_TILE;
                plan.push_back(WavePlan{r_lo, r_hi, a_lo, a_hi, c_lo, c_hi, t_lo, t_hi});
                r_lo = r_hi;
            }
        }
        // sets of waves: one stage-1 launch, the normalisers, one stage-2 launch each
        for (size_t w0 = 0; w0 < plan.size();) {
            size_t zb = 0, db = 0, yb = 0, w1 = w0;
            while (w1 < plan.size()) {
                const WavePlan &p = plan[w1];
                const size_t z = (size_t)P * (p.a_hi - p.a_lo) * (p.t_hi - p.t_lo) * COL_TILE * sizeof(float2);
                const int nrw = (p.r_hi - 1) / ns - p.r_lo / ns + 1;
                const size_t d = (size_t)nrw * (p.c_hi - p.c_lo) * std::max(2 * P, dlen) * sizeof(float);
                const size_t y = (size_t)nrw * (p.c_hi - p.c_lo) * J * sizeof(float2);
                if (w1 > w0 && (zb + z > z_batch_max || db + d > d_batch_max)) break;
                zb += z; db += d; yb = std::max(yb, y); ++w1;
            }
            int st = ensure(h, (void **)&ws.X, &ws.X_elems, zb, "grouped Z");
            if (st) return st;
            st = ensure(h, (void **)&ws.D, &ws.D_bytes, db, "grouped factors");
            if (st) return st;
            st = ensure(h, (void **)&ws.Yn, &ws.Y_bytes, yb, "grouped Y");
            if (st) return st;
            std::vector<S1Wave> s1;
            std::vector<S2Wave> s2;
            size_t zo = 0, dof = 0;
            for (size_t i = w0; i < w1; ++i) {
                const WavePlan &p = plan[i];
                const int xrows = p.a_hi - p.a_lo, xcols = (p.t_hi - p.t_lo) * COL_TILE;
                float2 *Xw = reinterpret_cast<float2 *>(reinterpret_cast<char *>(ws.X) + zo);
                float *Dw = reinterpret_cast<float *>(reinterpret_cast<char *>(ws.D) + dof);
                const int r_lo_ref = p.r_lo / ns, nrw = (p.r_hi - 1) / ns - r_lo_ref + 1;
                const int cols = p.c_hi - p.c_lo;
                if (precision == PFTCC_PREC_BF16X3) {
                    s1.push_back(S1Wave{Xw, p.a_lo / 32, xrows / 32, p.t_lo, p.t_hi - p.t_lo, 0, 0, 0, 0});
                } else {
                    dim3 grid(xrows / S1_TILE, xcols / S1_TILE, P / 2 + 1);
                    PFTCC_LAUNCH(h);
                    KTimer kt(h, PFTCC_K_STAGE1);
                    k_stage1_fp32<<<grid, 256, smem_s1, h->stream>>>(Ks, P, ws.UA, rows_pad, p.a_lo, ws.UB, cols_pad,
                                                                    p.t_lo * COL_TILE, Xw, xrows, xcols);
                    CKG(cudaGetLastError(), "stage1");
                }
                CKG(launch_norm(h, g, ws.RUf, h->nrefs, ws.CVf, cols_pad, r_lo_ref, nrw, p.c_lo, cols, cols, ws.sqp,
                                ws.Yn, Dw, p2, 1.0 / (2.0 * N), 0), "norm");
                s2.push_back(S2Wave{Xw, Dw, p.r_lo, p.r_hi - p.r_lo, p.r_lo - p.a_lo, xrows, xcols, p.c_lo, cols,
                                    p.c_lo - p.t_lo * COL_TILE, r_lo_ref, cols, 0, 0});
                zo += (size_t)P * xrows * xcols * sizeof(float2);
                dof += (size_t)nrw * cols * std::max(2 * P, dlen) * sizeof(float);
            }
            if (precision == PFTCC_PREC_BF16X3) {
                st = umma_stage1_waves(h, M, s1);
                if (st != PFTCC_OK) return st;
            }
            e = launch_stage2_waves(h, P, s2, ns, nrs, ws.cand, nullptr, bperm, 0);
            if (e != cudaSuccess)
                return set_err(h, e == cudaErrorMemoryAllocation ? PFTCC_ERR_OOM : PFTCC_ERR_CUDA,
                               std::string("grouped stage 2: ") + cudaGetErrorString(e));
            w0 = w1;
        }
        // the batch's best: the FP32 m-domain re-score (particle frame), or the exact re-score of the
        // top ntop in the reference frame, or the top 1
        if (md_rescore) {
            CKG(launch_rescore_md(h, P, bt.n, ntop, Ks, ns, nshifts_in > 0, ws.UA, rows_pad, ws.UB, cols_pad, ws.RU,
                                  ws.CV, ws.sqp, ws.cand, bperm, 0, out_dev, 0), "rescore");
        } else if (ntop == 0) {
            PFTCC_LAUNCH(h);
            k_finish<<<(bt.n + 127) / 128, 128, 0, h->stream>>>(ws.cand, bperm, bt.n, N, ns, nshifts_in > 0, 0, out_dev,
                                                                nullptr, nullptr);
            CKG(cudaGetLastError(), "finish");
        } else {
            int st = ensure(h, (void **)&h->d_work, &h->work_cap,
                            std::max<size_t>((size_t)bt.n * ntop * sizeof(Work), 4096), "work");
            if (st) return st;
            st = ensure(h, (void **)&h->d_groups, &h->group_cap, std::max<size_t>((size_t)bt.n * sizeof(Group), 256),
                        "groups");
            if (st) return st;
            PFTCC_LAUNCH(h);
            k_finish<<<(bt.n + 127) / 128, 128, 0, h->stream>>>(ws.cand, bperm, bt.n, N, ns, nshifts_in > 0, ntop,
                                                                out_dev, h->d_work, h->d_groups);
            CKG(cudaGetLastError(), "finish");
            CKG(launch_exact(h, h->d_groups, bt.n, h->d_work, ws.shifts, MODE_BEST, exact_frame(h), 1, nullptr,
                             out_dev),
                "rescore");
        }
    }
    if (!cap) {
        // the capture arena holds a later capture of this call's tables
        h->pin_need = h->pin_total;
        if (h->pin_cap[1] < h->pin_need) {
            if (h->pin[1]) cudaFreeHost(h->pin[1]);
            h->pin[1] = nullptr;
            h->pin_cap[1] = 0;
            CKG(cudaMallocHost(&h->pin[1], h->pin_need), "pinned capture staging");
            h->pin_cap[1] = h->pin_need;
        }
    }
    if (check && !cap) {
        int st = umma_check(h);
        if (st != PFTCC_OK) return st;
    }
#undef CKG
    return PFTCC_OK;
}

}  // namespace pftcc
