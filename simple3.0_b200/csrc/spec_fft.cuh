// spec_fft.cuh -- FP64 transforms of length N = N1 * N2 over the angular samples of a
// batch of shells, for the m-domain spectra of the search (k_search.cu).
//
// The spectra are U(m, k) = sum_{n<P} v_m(n, k) w_N^{-mn}, m = 0..P, N = 2P, with v_m the
// real part of the polar sample a(n, k) for even m and its imaginary part for odd m.  Over
// the full circle the polar samples continue as f(n) = a(n) for n < P and conj(a(n - P))
// for P <= n < N, whose length-N DFT F gives U(m) = F(m) / 2 for even m and
// U(m) = -i F(m) / 2 for odd m (the terms a + conj a = 2 Re a and a - conj a = 2i Im a).
// F is computed by one Cooley-Tukey split, in FP64 with FP64 twiddles:
//   pass 1, task (shell, n1): a length-N2 DFT over n2 of f(n1 + N1 n2), times w_N^{-n1 k2},
//           into buf[shell][k2][n1];
//   pass 2, task (shell, k2): a length-N1 DFT over n1 of buf[shell][k2][.] -> F(k2 + N2 k1).
// buf rows are padded to N1 + 1 entries (conflict-free shared-memory access in both passes).
#pragma once

#include <cuda_runtime.h>

namespace pftcc {
namespace sfft {

__device__ __forceinline__ double2 d_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 d_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 d_mul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}

// forward radix butterflies (the textbook radix-2/3/4/5 DFT formulas), FP64
template <int F> struct DBfly;
template <> struct DBfly<2> {
    __device__ static void run(double2 *v) { const double2 a = v[0], b = v[1]; v[0] = d_add(a, b); v[1] = d_sub(a, b); }
};
template <> struct DBfly<4> {
    __device__ static void run(double2 *v)
    {
        const double2 t0 = d_add(v[0], v[2]), t1 = d_sub(v[0], v[2]);
        const double2 t2 = d_add(v[1], v[3]), d = d_sub(v[1], v[3]);
        v[0] = d_add(t0, t2);
        v[2] = d_sub(t0, t2);
        v[1] = make_double2(t1.x + d.y, t1.y - d.x);   // t1 - i d
        v[3] = make_double2(t1.x - d.y, t1.y + d.x);   // t1 + i d
    }
};
template <> struct DBfly<3> {
    __device__ static void run(double2 *v)
    {
        const double s3 = 0.86602540378443864676;   // sin(2 pi / 3)
        const double2 a = v[0], t1 = d_add(v[1], v[2]), d = d_sub(v[1], v[2]);
        const double2 t2 = make_double2(fma(t1.x, -0.5, a.x), fma(t1.y, -0.5, a.y));
        v[0] = d_add(a, t1);
        v[1] = make_double2(fma(d.y, s3, t2.x), fma(d.x, -s3, t2.y));
        v[2] = make_double2(fma(d.y, -s3, t2.x), fma(d.x, s3, t2.y));
    }
};
template <> struct DBfly<5> {
    __device__ static void run(double2 *v)
    {
        const double c1 = 0.30901699437494742410, c2 = -0.80901699437494742410;   // cos(2pi/5), cos(4pi/5)
        const double s1 = 0.95105651629515357212, s2 = 0.58778525229247312917;    // sin(2pi/5), sin(4pi/5)
        const double2 a = v[0];
        const double2 t1 = d_add(v[1], v[4]), t2 = d_add(v[2], v[3]);
        const double2 t3 = d_sub(v[1], v[4]), t4 = d_sub(v[2], v[3]);
        const double2 m1 = make_double2(fma(c2, t2.x, fma(c1, t1.x, a.x)), fma(c2, t2.y, fma(c1, t1.y, a.y)));
        const double2 m2 = make_double2(fma(c1, t2.x, fma(c2, t1.x, a.x)), fma(c1, t2.y, fma(c2, t1.y, a.y)));
        const double2 n1 = make_double2(fma(s2, t4.x, s1 * t3.x), fma(s2, t4.y, s1 * t3.y));
        const double2 n2 = make_double2(fma(-s1, t4.x, s2 * t3.x), fma(-s1, t4.y, s2 * t3.y));
        v[0] = d_add(d_add(a, t1), t2);
        v[1] = make_double2(m1.x + n1.y, m1.y - n1.x);   // m1 - i n1
        v[4] = make_double2(m1.x - n1.y, m1.y + n1.x);
        v[2] = make_double2(m2.x + n2.y, m2.y - n2.x);
        v[3] = make_double2(m2.x - n2.y, m2.y + n2.x);
    }
};

// length-L forward DFT in registers, natural order in and out; w_L^e = tw[e * STEP], tw the
// w_N^{-e} table of the whole length N = L * STEP (in shared memory)
template <int L, int STEP> struct DFFT {
    static constexpr int F = (L % 4 == 0) ? 4 : (L % 2 == 0) ? 2 : (L % 3 == 0) ? 3 : (L % 5 == 0) ? 5 : 0;
    static_assert(F != 0, "transform length must factor into 2, 3, 5");
    static constexpr int M = L / F;
    __device__ static void run(double2 *x, const double2 *tw)
    {
        double2 s[F][M];
#pragma unroll
        for (int q = 0; q < F; ++q)
#pragma unroll
            for (int j = 0; j < M; ++j) s[q][j] = x[q + F * j];
#pragma unroll
        for (int q = 0; q < F; ++q) DFFT<M, STEP * F>::run(s[q], tw);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            double2 v[F];
#pragma unroll
            for (int q = 0; q < F; ++q) v[q] = (q * k == 0) ? s[q][k] : d_mul(s[q][k], tw[q * k * STEP]);
            DBfly<F>::run(v);
#pragma unroll
            for (int r = 0; r < F; ++r) x[k + M * r] = v[r];
        }
    }
};
template <int STEP> struct DFFT<1, STEP> {
    __device__ static void run(double2 *, const double2 *) {}
};

// the shells per batch and the shared memory of the batch buffer
constexpr int KB = 8;
template <int N1, int N2> __host__ __device__ constexpr int buf_elems() { return KB * N2 * (N1 + 1); }

// F for the nk <= KB shells of a batch: getf(kl, n) returns f(n) of batch shell kl as
// double2, put(kl, m, F) receives F(m) for every m < N (the caller keeps what it needs).  All
// threads of the block take part; buf holds buf_elems<N1, N2>() double2, tw the w_N^{-e} table.
// Starts and ends with the block synchronised (the caller's staging is visible; buf is free again).
template <int N1, int N2, class GetF, class Put>
__device__ __forceinline__ void batch_fft(int nk, const GetF &getf, const Put &put, double2 *buf, const double2 *tw)
{
    __syncthreads();
    // pass 1: tasks (kl, n1), n1 fastest
    for (int t = threadIdx.x; t < nk * N1; t += blockDim.x) {
        const int kl = t / N1, n1 = t - kl * N1;
        double2 x[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) x[n2] = getf(kl, n1 + N1 * n2);
        DFFT<N2, N1>::run(x, tw);
        double2 *row = buf + (size_t)kl * N2 * (N1 + 1) + n1;
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) row[k2 * (N1 + 1)] = (k2 == 0 || n1 == 0) ? x[k2] : d_mul(x[k2], tw[n1 * k2]);
    }
    __syncthreads();
    // pass 2: tasks (kl, k2), kl fastest (consecutive shells store next to each other)
    for (int t = threadIdx.x; t < nk * N2; t += blockDim.x) {
        const int k2 = t / nk, kl = t - k2 * nk;
        const double2 *row = buf + ((size_t)kl * N2 + k2) * (N1 + 1);
        double2 x[N1];
#pragma unroll
        for (int n1 = 0; n1 < N1; ++n1) x[n1] = row[n1];
        DFFT<N1, N2>::run(x, tw);
#pragma unroll
        for (int k1 = 0; k1 < N1; ++k1) put(kl, k2 + N2 * k1, x[k1]);
    }
    __syncthreads();
}

}  // namespace sfft
}  // namespace pftcc
