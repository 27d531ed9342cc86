// k_stage2.cu -- per-(particle, reference x shift) inverse transform of the m-domain
// spectrum, the correlation over all in-plane rotations, its argmax and the
// particle's running top-8; and the FP32 m-domain re-score of the final candidates.
//
// For one triple the spectrum X(m), m = 0..P (Hermitian over the full circle of
// N = 2P rotations) is packed into Z(j) = [X(j) + conj X(P-j)] + i [X(j) - conj X(P-j)]
// w_N^{-j}, j < P, whose length-P forward DFT z(l) = y(2l) + i y(2l+1) gives every
// rotation's correlation sum y(rot) = sum_{m<N} X(m) w_N^{-m rot} (the real-output
// half-length transform; the reference runs the equivalent FFTW c2r per shell in
// calc_corrs_over_k, simple_polarft_corrcalc.f90:1156).  The length-P DFT is one
// Cooley-Tukey split P = P1 * P2 evaluated entirely in registers with compile-time
// unrolled radix-2/3/4/5 butterflies:
//   pass A: for each residue class j1 < P1 a length-P2 DFT over j2 of Z(j1 + P1 j2),
//           times w_P^{-j1 l2}, into a thread-private shared-memory slab;
//   pass B: for each l2 < P2 a length-P1 DFT over j1 -> z(l2 + P2 l1).
// The search (k_stage2_fast) reads Z as stage 1 stored it, P planes of [col][row]; the
// FP32 re-score forms Z from X itself, processing classes j1 and P1 - j1 together so
// that every X element is computed once (Z(j) needs X(j) and X(P - j), which lie in the
// mirror class).
#include "pftcc_internal.cuh"
#include "spec_fft.cuh"

#include <algorithm>
#include <cstdio>
#include <cmath>

namespace pftcc {

constexpr int TW_MAX = 320;
struct TwTables {
    float2 wP[TW_MAX];   // w_P^{-e} = exp(-2 pi i e / P), e < P
    float2 wN[TW_MAX];   // w_N^{-e} = exp(-2 pi i e / N), e < P
    // the same w_P^{-e} = (c, s) as lane pairs for the two-lane transforms: (c, c), (s, s), (-s, -s)
    float2 pc[TW_MAX], ps[TW_MAX], pn[TW_MAX];
};

__device__ __forceinline__ float2 c_mul(float2 a, float2 b) { return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mi(float2 a) { return make_float2(a.y, -a.x); }   // -i * a

// forward radix butterflies (textbook radix-2/3/4/5 DFT formulas)
template <int F> struct Bfly;
template <> struct Bfly<2> {
    __device__ static void run(float2 *v) { const float2 a = v[0], b = v[1]; v[0] = c_add(a, b); v[1] = c_sub(a, b); }
};
template <> struct Bfly<4> {
    __device__ static void run(float2 *v)
    {
        const float2 t0 = c_add(v[0], v[2]), t1 = c_sub(v[0], v[2]);
        const float2 t2 = c_add(v[1], v[3]), t3 = c_mi(c_sub(v[1], v[3]));
        v[0] = c_add(t0, t2);
        v[2] = c_sub(t0, t2);
        v[1] = c_add(t1, t3);
        v[3] = c_sub(t1, t3);
    }
};
template <> struct Bfly<3> {
    __device__ static void run(float2 *v)
    {
        const float s3 = 0.86602540378443865f;   // sin(2 pi / 3)
        const float2 a = v[0], t1 = c_add(v[1], v[2]);
        const float2 t2 = make_float2(a.x - 0.5f * t1.x, a.y - 0.5f * t1.y);
        const float2 d = c_sub(v[1], v[2]);
        const float2 t3 = make_float2(s3 * d.y, -s3 * d.x);   // -i sin(2pi/3) (b - c)
        v[0] = c_add(a, t1);
        v[1] = c_add(t2, t3);
        v[2] = c_sub(t2, t3);
    }
};
template <> struct Bfly<5> {
    __device__ static void run(float2 *v)
    {
        const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;   // cos(2pi/5), cos(4pi/5)
        const float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;    // sin(2pi/5), sin(4pi/5)
        const float2 a = v[0];
        const float2 t1 = c_add(v[1], v[4]), t2 = c_add(v[2], v[3]);
        const float2 t3 = c_sub(v[1], v[4]), t4 = c_sub(v[2], v[3]);
        const float2 m1 = make_float2(a.x + c1 * t1.x + c2 * t2.x, a.y + c1 * t1.y + c2 * t2.y);
        const float2 m2 = make_float2(a.x + c2 * t1.x + c1 * t2.x, a.y + c2 * t1.y + c1 * t2.y);
        const float2 n1 = make_float2(s1 * t3.x + s2 * t4.x, s1 * t3.y + s2 * t4.y);
        const float2 n2 = make_float2(s2 * t3.x - s1 * t4.x, s2 * t3.y - s1 * t4.y);
        v[0] = make_float2(a.x + t1.x + t2.x, a.y + t1.y + t2.y);
        v[1] = c_add(m1, c_mi(n1));
        v[4] = c_sub(m1, c_mi(n1));
        v[2] = c_add(m2, c_mi(n2));
        v[3] = c_sub(m2, c_mi(n2));
    }
};

// length-L forward DFT in registers, natural order in and out; w_L^e = wP[e * STEP]
template <int L, int STEP> struct SFFT {
    static constexpr int F = (L % 4 == 0) ? 4 : (L % 2 == 0) ? 2 : (L % 3 == 0) ? 3 : (L % 5 == 0) ? 5 : 0;
    static_assert(F != 0, "transform length must factor into 2, 3, 5");
    static constexpr int M = L / F;
    __device__ static void run(float2 *x, const TwTables &tw)
    {
        float2 s[F][M];
#pragma unroll
        for (int q = 0; q < F; ++q)
#pragma unroll
            for (int j = 0; j < M; ++j) s[q][j] = x[q + F * j];
#pragma unroll
        for (int q = 0; q < F; ++q) SFFT<M, STEP * F>::run(s[q], tw);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            float2 v[F];
#pragma unroll
            for (int q = 0; q < F; ++q) v[q] = (q * k == 0) ? s[q][k] : c_mul(s[q][k], tw.wP[q * k * STEP]);
            Bfly<F>::run(v);
#pragma unroll
            for (int r = 0; r < F; ++r) x[k + M * r] = v[r];
        }
    }
};
template <int STEP> struct SFFT<1, STEP> {
    __device__ static void run(float2 *, const TwTables &) {}
};

// ---------------------------------------------------------------------------------------
// Two transforms at once with the packed two-lane FP32 instructions of sm_100 (one
// add / mul / fma on a register pair): C2 holds two complex numbers as r = (re_a, re_b),
// i = (im_a, im_b), so a butterfly of two independent transforms costs half the
// instructions of two scalar ones.  Each lane is rounded exactly as the scalar operation.
struct C2 { float2 r, i; };
__device__ __forceinline__ float2 f2_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 f2_sub(float2 a, float2 b)
{
    unsigned long long d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(*reinterpret_cast<unsigned long long *>(&a)),
        "l"(*reinterpret_cast<unsigned long long *>(&b)));
    return *reinterpret_cast<float2 *>(&d);
}
__device__ __forceinline__ float2 f2_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 f2_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 f2_s(float s) { return make_float2(s, s); }
__device__ __forceinline__ C2 p_add(const C2 &a, const C2 &b) { return {f2_add(a.r, b.r), f2_add(a.i, b.i)}; }
__device__ __forceinline__ C2 p_sub(const C2 &a, const C2 &b) { return {f2_sub(a.r, b.r), f2_sub(a.i, b.i)}; }
// a * (c + i s) with c, s and -s given as lane pairs
__device__ __forceinline__ C2 p_twid(const C2 &a, float2 c, float2 s, float2 ns)
{
    return {f2_fma(a.r, c, f2_mul(a.i, ns)), f2_fma(a.r, s, f2_mul(a.i, c))};
}
__device__ __forceinline__ float max3f(float a, float b, float c)
{
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// the radix-2/3/4/5 butterflies above, on lane pairs (-i a = (a.i, -a.r) is folded into
// the adds that follow it)
template <int F> struct PBfly;
template <> struct PBfly<2> {
    __device__ static void run(C2 *v) { const C2 a = v[0], b = v[1]; v[0] = p_add(a, b); v[1] = p_sub(a, b); }
};
template <> struct PBfly<4> {
    __device__ static void run(C2 *v)
    {
        const C2 t0 = p_add(v[0], v[2]), t1 = p_sub(v[0], v[2]);
        const C2 t2 = p_add(v[1], v[3]), d = p_sub(v[1], v[3]);
        v[0] = p_add(t0, t2);
        v[2] = p_sub(t0, t2);
        v[1] = {f2_add(t1.r, d.i), f2_sub(t1.i, d.r)};
        v[3] = {f2_sub(t1.r, d.i), f2_add(t1.i, d.r)};
    }
};
template <> struct PBfly<3> {
    __device__ static void run(C2 *v)
    {
        const float s3 = 0.86602540378443865f;
        const C2 a = v[0], t1 = p_add(v[1], v[2]), d = p_sub(v[1], v[2]);
        const C2 t2 = {f2_fma(t1.r, f2_s(-0.5f), a.r), f2_fma(t1.i, f2_s(-0.5f), a.i)};
        v[0] = p_add(a, t1);
        v[1] = {f2_fma(d.i, f2_s(s3), t2.r), f2_fma(d.r, f2_s(-s3), t2.i)};
        v[2] = {f2_fma(d.i, f2_s(-s3), t2.r), f2_fma(d.r, f2_s(s3), t2.i)};
    }
};
template <> struct PBfly<5> {
    __device__ static void run(C2 *v)
    {
        const float c1 = 0.30901699437494742f, c2 = -0.80901699437494742f;
        const float s1 = 0.95105651629515357f, s2 = 0.58778525229247313f;
        const C2 a = v[0];
        const C2 t1 = p_add(v[1], v[4]), t2 = p_add(v[2], v[3]);
        const C2 t3 = p_sub(v[1], v[4]), t4 = p_sub(v[2], v[3]);
        const C2 m1 = {f2_fma(t2.r, f2_s(c2), f2_fma(t1.r, f2_s(c1), a.r)), f2_fma(t2.i, f2_s(c2), f2_fma(t1.i, f2_s(c1), a.i))};
        const C2 m2 = {f2_fma(t2.r, f2_s(c1), f2_fma(t1.r, f2_s(c2), a.r)), f2_fma(t2.i, f2_s(c1), f2_fma(t1.i, f2_s(c2), a.i))};
        const C2 n1 = {f2_fma(t4.r, f2_s(s2), f2_mul(t3.r, f2_s(s1))), f2_fma(t4.i, f2_s(s2), f2_mul(t3.i, f2_s(s1)))};
        const C2 n2 = {f2_fma(t4.r, f2_s(-s1), f2_mul(t3.r, f2_s(s2))), f2_fma(t4.i, f2_s(-s1), f2_mul(t3.i, f2_s(s2)))};
        v[0] = p_add(p_add(a, t1), t2);
        v[1] = {f2_add(m1.r, n1.i), f2_sub(m1.i, n1.r)};
        v[4] = {f2_sub(m1.r, n1.i), f2_add(m1.i, n1.r)};
        v[2] = {f2_add(m2.r, n2.i), f2_sub(m2.i, n2.r)};
        v[3] = {f2_sub(m2.r, n2.i), f2_add(m2.i, n2.r)};
    }
};

__host__ __device__ constexpr int gcd_c(int a, int b) { return b == 0 ? a : gcd_c(b, a % b); }
// the index o < F M with o = r (mod F) and o = k (mod M), gcd(F, M) = 1
__host__ __device__ constexpr int crt_c(int r, int k, int F, int M)
{
    int o = k;
    while (o % F != r) o += M;
    return o;
}

// two length-L forward DFTs, one per lane, natural order in and out (SFFT's recursion).
// When the radix F and the rest M = L / F are coprime (15 = 3 x 5, 12 = 4 x 3, 20 = 4 x 5)
// the Good-Thomas prime-factor mapping needs no twiddles between the two stages: input
// x((M q + F j) mod L) -> the M-point DFTs over j, the F-point butterflies over q, output
// index o with o = r (mod F) and o = k (mod M); otherwise the Cooley-Tukey split with the
// twiddles w_L^{qk}.
template <int L, int STEP> struct PFFT {
    static constexpr int F = SFFT<L, STEP>::F;
    static constexpr int M = L / F;
    static constexpr bool PFA = M > 1 && gcd_c(F, M) == 1;
    __device__ static void run(C2 *x, const TwTables &tw)
    {
        C2 s[F][M];
#pragma unroll
        for (int q = 0; q < F; ++q)
#pragma unroll
            for (int j = 0; j < M; ++j) s[q][j] = PFA ? x[(M * q + F * j) % L] : x[q + F * j];
#pragma unroll
        for (int q = 0; q < F; ++q) PFFT<M, STEP * F>::run(s[q], tw);
#pragma unroll
        for (int k = 0; k < M; ++k) {
            C2 v[F];
#pragma unroll
            for (int q = 0; q < F; ++q) {
                const int e = q * k * STEP;
                v[q] = (PFA || q * k == 0) ? s[q][k] : p_twid(s[q][k], tw.pc[e], tw.ps[e], tw.pn[e]);
            }
            PBfly<F>::run(v);
#pragma unroll
            for (int r = 0; r < F; ++r) x[PFA ? crt_c(r, k, F, M) : k + M * r] = v[r];
        }
    }
};
template <int STEP> struct PFFT<1, STEP> {
    __device__ static void run(C2 *, const TwTables &) {}
};

// Row slab of the search (two-lane layout): pass-A output (l2, j1) -- re and im as two
// scalars -- sits in lane l2 & 1 of the float2 slots ((l2 >> 1) P1 + j1) 2 + part
// (part 0 = re, 1 = im), element stride T, so that pass B reads the pair of blocks
// (l2, l2 + 1) with one 8-byte load per part.  For odd P2 the last block l2 = P2 - 1 is
// stored in both lanes.

// the loads of class pair (c, cb) of one row: Z(c + P1 j2) and Z(cb + P1 j2)
template <int P1, int P2, class GetZ>
__device__ __forceinline__ void load_pair(int c, int cb, const GetZ &getz, float2 (&na)[P2], float2 (&nb)[P2])
{
#pragma unroll
    for (int j2 = 0; j2 < P2; ++j2) {
        na[j2] = getz(c + P1 * j2);
        nb[j2] = getz(cb + P1 * j2);
    }
}

// pass A of the search over the packed spectrum Z, two classes per step: c and cb = c + 1
// (c again for the last class of an odd range), one per lane -- a length-P2 DFT over j2
// of Z(c + P1 j2), times w_P^{-c l2} (lane-pair twiddles twa / twb, entry c P2 + l2), into
// the slab.  na / nb hold the first pair's loads on entry (issued by the caller during the
// previous row's pass B); the next pair's 2 P2 loads are issued before each transform.
template <int P1, int P2, class GetZ>
__device__ __forceinline__ void passA_pk(int c0, int c1, const GetZ &getz, float2 *slab, int T, const float4 *twa,
                                         const float2 *twb, const TwTables &tw, float2 (&na)[P2], float2 (&nb)[P2])
{
#pragma unroll 1
    for (int c = c0; c < c1; c += 2) {
        const int cb = min(c + 1, c1 - 1);
        C2 z[P2];
#pragma unroll
        for (int j2 = 0; j2 < P2; ++j2) z[j2] = {make_float2(na[j2].x, nb[j2].x), make_float2(na[j2].y, nb[j2].y)};
        if (c + 2 < c1) load_pair<P1, P2>(c + 2, min(c + 3, c1 - 1), getz, na, nb);
        PFFT<P2, P1>::run(z, tw);
        float2 *sa = slab + (size_t)c * 2 * T, *sb = slab + (size_t)cb * 2 * T;
#pragma unroll
        for (int l2 = 0; l2 < P2; ++l2) {
            C2 o = z[l2];
            if (l2 > 0) {
                const float4 w = twa[c * P2 + l2];
                o = p_twid(o, make_float2(w.x, w.y), make_float2(w.z, w.w), twb[c * P2 + l2]);
            }
            const int q = (l2 >> 1) * P1 * 2;
#pragma unroll
            for (int ln = 0; ln < 2; ++ln) {
                if (ln != (l2 & 1) && !((P2 & 1) && l2 == P2 - 1)) continue;
                reinterpret_cast<float *>(sa + q * T)[ln] = o.r.x;
                reinterpret_cast<float *>(sa + (q + 1) * T)[ln] = o.i.x;
                reinterpret_cast<float *>(sb + q * T)[ln] = o.r.y;
                reinterpret_cast<float *>(sb + (q + 1) * T)[ln] = o.i.y;
            }
        }
    }
}

// Pass A, split into the pieces the two halves of a row's transform take: class 0 (its
// own mirror, X(P) closes it), the class pairs (c, P1 - c) for C0 <= c < C1, and for even
// P1 the self-mirrored class P1/2.  Outputs, times w_P^{-j1 l2}, go to the row's slab
// (element stride T).
template <int P1, int P2, class GetX>
__device__ __forceinline__ void passA_class0(const GetX &getx, float2 *slab, int T, const TwTables &tw)
{
    constexpr int P = P1 * P2;
    float2 xa[P2 + 1];
#pragma unroll
    for (int j2 = 0; j2 < P2; ++j2) xa[j2] = getx(P1 * j2);
    xa[P2] = getx(P);
    xa[0].y = 0.f;       // X(0) and X(P) are real
    xa[P2].y = 0.f;
    float2 z[P2];
#pragma unroll
    for (int j2 = 0; j2 < P2; ++j2) z[j2] = make_z(xa[j2], xa[P2 - j2], tw.wN[P1 * j2]);
    SFFT<P2, P1>::run(z, tw);
#pragma unroll
    for (int l2 = 0; l2 < P2; ++l2) slab[(l2 * P1) * T] = z[l2];
}

// the class-pair loop runs over a runtime range (one copy of its code for both halves of
// a row's transform); c * l2 < P1 * P2 for every class and pass-B index, so the twiddle
// indices need no reduction
template <int P1, int P2, class GetX>
__device__ __forceinline__ void passA_pairs(int c0, int c1, const GetX &getx, float2 *slab, int T, const TwTables &tw)
{
#pragma unroll 1
    for (int c = c0; c < c1; ++c) {
        float2 xa[P2], xb[P2];
#pragma unroll
        for (int j2 = 0; j2 < P2; ++j2) {
            xa[j2] = getx(c + P1 * j2);
            xb[j2] = getx(P1 - c + P1 * j2);
        }
        float2 za[P2], zb[P2];
#pragma unroll
        for (int j2 = 0; j2 < P2; ++j2) {
            za[j2] = make_z(xa[j2], xb[P2 - 1 - j2], tw.wN[c + P1 * j2]);
            zb[j2] = make_z(xb[j2], xa[P2 - 1 - j2], tw.wN[P1 - c + P1 * j2]);
        }
        SFFT<P2, P1>::run(za, tw);
        SFFT<P2, P1>::run(zb, tw);
#pragma unroll
        for (int l2 = 0; l2 < P2; ++l2) {
            slab[(l2 * P1 + c) * T] = l2 == 0 ? za[l2] : c_mul(za[l2], tw.wP[c * l2]);
            slab[(l2 * P1 + P1 - c) * T] = l2 == 0 ? zb[l2] : c_mul(zb[l2], tw.wP[(P1 - c) * l2]);
        }
    }
}

template <int P1, int P2, class GetX>
__device__ __forceinline__ void passA_mid(const GetX &getx, float2 *slab, int T, const TwTables &tw)
{
    constexpr int P = P1 * P2;
    if constexpr ((P1 & 1) == 0) {
        constexpr int c = P1 / 2;
        float2 xa[P2];
#pragma unroll
        for (int j2 = 0; j2 < P2; ++j2) xa[j2] = getx(c + P1 * j2);
        float2 z[P2];
#pragma unroll
        for (int j2 = 0; j2 < P2; ++j2) z[j2] = make_z(xa[j2], xa[P2 - 1 - j2], tw.wN[c + P1 * j2]);
        SFFT<P2, P1>::run(z, tw);
#pragma unroll
        for (int l2 = 0; l2 < P2; ++l2) slab[(l2 * P1 + c) * T] = l2 == 0 ? z[l2] : c_mul(z[l2], tw.wP[(c * l2) % P]);
    }
}

// pass B for l2 in [L0, L1): length-P1 DFTs, correlations, argmax (lowest rotation on ties).
// EU (the Euclidean objective): dinv(rho) is the additive term, the value scale * v + dinv(rho)
template <int P1, int P2, class Dinv, bool EU = false>
__device__ __forceinline__ void passB(int L0, int L1, const float2 *slab, int T, const TwTables &tw, const Dinv &dinv,
                                      float scale, float *cc_out, float &best, int &brot)
{
    constexpr int P = P1 * P2;
#pragma unroll 1
    for (int l2 = L0; l2 < L1; ++l2) {
        float2 v[P1];
#pragma unroll
        for (int j1 = 0; j1 < P1; ++j1) v[j1] = slab[(l2 * P1 + j1) * T];
        SFFT<P1, P2>::run(v, tw);
#pragma unroll
        for (int l1 = 0; l1 < P1; ++l1) {
            const int l = l2 + P2 * l1;
            const int r0 = 2 * l, r1 = 2 * l + 1;
            const float c0 = EU ? fmaf(scale, v[l1].x, dinv(r0 < P ? r0 : r0 - P))
                                : scale * v[l1].x * dinv(r0 < P ? r0 : r0 - P);
            const float c1 = EU ? fmaf(scale, v[l1].y, dinv(r1 < P ? r1 : r1 - P))
                                : scale * v[l1].y * dinv(r1 < P ? r1 : r1 - P);
            if (cc_out) { cc_out[r0] = c0; cc_out[r1] = c1; }
            if (c0 > best || (c0 == best && r0 < brot)) { best = c0; brot = r0; }
            if (c1 > best || (c1 == best && r1 < brot)) { best = c1; brot = r1; }
        }
    }
}

// pass B on the block pair (l, l + 1), l even: two length-P1 DFTs (one per lane) of the
// slab blocks, times the normalising factors -- stored in pair order, four per l1:
// (l, re), (l + 1, re), (l, im), (l + 1, im), already carrying the 1/(2N) scale -- leaving
// the correlation of rot = 2 (l + lane + P2 l1) + part in lane `lane` of v[l1].r / v[l1].i.
// EU: the factors are the Euclidean objective's additive terms, the value escale * v + d
template <int P1, int P2, bool EU>
__device__ __forceinline__ void passB_pair(int l, const float2 *slab, int T, const TwTables &tw, const float4 *Dp,
                                           float escale, C2 (&v)[P1])
{
    const float4 *dq = Dp + (size_t)(l >> 1) * P1;
    float4 d[P1];
#pragma unroll
    for (int l1 = 0; l1 < P1; ++l1) d[l1] = __ldg(dq + l1);   // issued ahead of the transform
    const float2 *sq = slab + (size_t)(l >> 1) * P1 * 2 * T;
#pragma unroll
    for (int j1 = 0; j1 < P1; ++j1) v[j1] = {sq[(2 * j1) * T], sq[(2 * j1 + 1) * T]};
    PFFT<P1, P2>::run(v, tw);
    if constexpr (EU) {
        const float2 sc = f2_s(escale);
#pragma unroll
        for (int l1 = 0; l1 < P1; ++l1) {
            v[l1].r = f2_fma(v[l1].r, sc, make_float2(d[l1].x, d[l1].y));
            v[l1].i = f2_fma(v[l1].i, sc, make_float2(d[l1].z, d[l1].w));
        }
    } else {
#pragma unroll
        for (int l1 = 0; l1 < P1; ++l1) {
            v[l1].r = f2_mul(v[l1].r, make_float2(d[l1].x, d[l1].y));
            v[l1].i = f2_mul(v[l1].i, make_float2(d[l1].z, d[l1].w));
        }
    }
}

// pass B of the search for the block pairs (l, l + 1), l = L0, L0 + 2, ... < L1 (L0 even;
// for odd P2 the pair (P2 - 1, P2) holds block P2 - 1 twice): the maximum correlation and
// its rotation (lowest rotation among equal maxima).  Each pair's 4 P1 values are reduced
// with max; afterwards the winning pair -- every pair when another one reached the same
// maximum -- is evaluated again by the same code (identical values) and scanned for the
// lowest rotation holding the maximum.
template <int P1, int P2, bool EU>
__device__ __forceinline__ void passB_search(int L0, int L1, const float2 *slab, int T, const TwTables &tw,
                                             const float4 *Dp, float escale, float &best, int &brot)
{
    float bv = -INFINITY;
    int bl = -1, l = L0, lend = L1, stage = 0, rmin = 0x7fffffff;
    bool tie = false;
#pragma unroll 1
    while (true) {
        C2 v[P1];
        passB_pair<P1, P2, EU>(l, slab, T, tw, Dp, escale, v);
        if (stage == 0) {
            float m = fmaxf(v[0].r.x, v[0].r.y);
            m = max3f(m, v[0].i.x, v[0].i.y);
#pragma unroll
            for (int l1 = 1; l1 < P1; ++l1) {
                m = max3f(m, v[l1].r.x, v[l1].r.y);
                m = max3f(m, v[l1].i.x, v[l1].i.y);
            }
            if (m > bv) { bv = m; bl = l; tie = false; }
            else if (m == bv) tie = true;
            l += 2;
            if (l < L1) continue;
            if (bl < 0) break;
            stage = 1;
            l = tie ? L0 : bl;
            lend = tie ? L1 : bl + 2;
        } else {
            const int lb = min(l + 1, P2 - 1);
#pragma unroll
            for (int l1 = 0; l1 < P1; ++l1) {
                const int ra = 2 * (l + P2 * l1), rb = 2 * (lb + P2 * l1);
                if (v[l1].r.x == bv) rmin = min(rmin, ra);
                if (v[l1].i.x == bv) rmin = min(rmin, ra + 1);
                if (v[l1].r.y == bv) rmin = min(rmin, rb);
                if (v[l1].i.y == bv) rmin = min(rmin, rb + 1);
            }
            l += 2;
            if (l >= lend) break;
        }
    }
    best = bv;
    brot = bl < 0 ? 0 : rmin;
}

// pass B writing every correlation (corr_all), with the per-rotation argmax
template <int P1, int P2, bool EU>
__device__ __forceinline__ void passB_all(int L0, int L1, const float2 *slab, int T, const TwTables &tw,
                                          const float4 *Dp, float escale, float *cc_out, float &best, int &brot)
{
#pragma unroll 1
    for (int l = L0; l < L1; l += 2) {
        C2 v[P1];
        passB_pair<P1, P2, EU>(l, slab, T, tw, Dp, escale, v);
        const bool two = l + 1 < P2;
#pragma unroll
        for (int l1 = 0; l1 < P1; ++l1) {
            const float cv[4] = {v[l1].r.x, v[l1].i.x, v[l1].r.y, v[l1].i.y};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                if (e >= 2 && !two) continue;
                const int r = 2 * (l + (e >> 1) + P2 * l1) + (e & 1);
                cc_out[r] = cv[e];
                if (cv[e] > best || (cv[e] == best && r < brot)) { best = cv[e]; brot = r; }
            }
        }
    }
}

// how a row's transform is split between its NT threads: thread (role) r takes the class
// pairs [r n / NT, (r + 1) n / NT) of the n = ceil(P1 / 2) pairs (2k, 2k + 1) of pass A and the
// block pairs likewise of the ceil(P2 / 2) pairs (2q, 2q + 1) of pass B
__host__ __device__ constexpr int role_part(int n, int r, int nt) { return r * n / nt; }

// the whole per-triple transform in one thread; getx(j) returns X(j) for j = 0..P;
// dinv(rot) the normalising factor; slab is this thread's shared-memory slab with
// element stride T
template <int P1, int P2, class GetX, class Dinv>
__device__ __forceinline__ void triple_corr(const GetX &getx, const Dinv &dinv, float2 *slab, int T, const TwTables &tw,
                                            float scale, float *cc_out, float &best, int &brot)
{
    passA_class0<P1, P2>(getx, slab, T, tw);
    passA_pairs<P1, P2>(1, (P1 + 1) / 2, getx, slab, T, tw);
    passA_mid<P1, P2>(getx, slab, T, tw);
    passB<P1, P2>(0, P2, slab, T, tw, dinv, scale, cc_out, best, brot);
}

// ---------------------------------------------------------------------------------------
struct S2Fast {
    int nshifts, N, nrs_total, nwaves;
    float escale;   // the Euclidean objective: the transform's scale 1/(2N) (the factors are additive)
};

// the normalising factors per (reference, particle) in the order the search's pass B
// reads them: 4 P1 values per block pair, ceil(P2 / 2) pairs (the last pair of an odd P2
// repeats block P2 - 1)
template <int P1, int P2> __host__ __device__ constexpr int s2_dlen() { return 4 * P1 * ((P2 + 1) / 2); }

// threads per row of the search's stage 2
constexpr int S2_THREADS_PER_ROW = 2;

// (c, id) ranks above (c2, id2): larger correlation, then lower id
__device__ __forceinline__ bool ranks_above(float c, int id, float c2, int id2) { return c > c2 || (c == c2 && id < id2); }

// ROWS rows in flight per block, NT threads per row: warps w + r ROWS/32 (role r) share the
// rows' slabs and meet at named barrier 1 + w twice per row (after pass A; after pass B, when
// roles 1.. hand their argmax over).  Role 0 keeps its rows' running top-8 in registers; at
// the end the block merges those lists with the particle's running top-8.
// X here is the packed spectrum Z, P planes of [col][row].
template <int P1, int P2, int ROWS, int NT, bool WRITE, bool EU>
__global__ void __launch_bounds__(NT * ROWS, 1) k_stage2_fast(S2Fast sp, const TwTables tw, const S2Wave *__restrict__ waves,
                                                            float2 *__restrict__ cand, float *__restrict__ ccall,
                                                            const int *__restrict__ perm)
{
    constexpr int Q2 = (P2 + 1) / 2, DLEN = s2_dlen<P1, P2>(), NPA = (P1 + 1) / 2;
    // this block's wave (the last one starting at or before it) and column within it
    int lo = 0, hi = sp.nwaves - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (__ldg(&waves[mid].blk0) <= (int)blockIdx.x) lo = mid; else hi = mid - 1;
    }
    const S2Wave *W = waves + lo;
    const int cl = (int)blockIdx.x - __ldg(&W->blk0);
    const float2 *X = reinterpret_cast<const float2 *>(__ldg(reinterpret_cast<const unsigned long long *>(&W->X)));
    const float *Dinv = reinterpret_cast<const float *>(__ldg(reinterpret_cast<const unsigned long long *>(&W->D)));
    const int w_rows = __ldg(&W->rows), w_row0 = __ldg(&W->row0), w_rofs = __ldg(&W->rofs);
    const int w_xrows = __ldg(&W->xrows), w_xcols = __ldg(&W->xcols), w_col0 = __ldg(&W->col0);
    const int w_zc0 = __ldg(&W->zc0), w_r0 = __ldg(&W->r0), w_dcols = __ldg(&W->dcols);
    extern __shared__ float4 smem4[];
    const int t = threadIdx.x;
    const int role = t / ROWS, lr = t - role * ROWS;
    const int bar = 1 + (lr >> 5);
    float2 *slab = reinterpret_cast<float2 *>(smem4) + lr;                                      // [Q2 P1 2][ROWS]
    float4 *twa = smem4 + (size_t)Q2 * P1 * ROWS;                                               // [P1 P2]
    float2 *twb = reinterpret_cast<float2 *>(twa + P1 * P2);                                    // [P1 P2]
    float *xfer_c = reinterpret_cast<float *>(twb + P1 * P2);                                   // [NT - 1][ROWS]
    int *xfer_r = reinterpret_cast<int *>(xfer_c + (NT - 1) * ROWS);                            // [NT - 1][ROWS]
    // lane-pair twiddles of pass A: lane a class c, lane b class min(c + 1, P1 - 1) (pairs
    // start at even classes in every role's range)
    for (int e = t; e < P1 * P2; e += blockDim.x) {
        const int c = e / P2, l2 = e - c * P2;
        const int cb = min(c + 1, P1 - 1);
        const float2 wa = tw.wP[c * l2], wb = tw.wP[cb * l2];
        twa[e] = make_float4(wa.x, wb.x, wa.y, wb.y);
        twb[e] = make_float2(-wa.y, -wb.y);
    }
    __syncthreads();
    // Z offsets in float2 units fit 32 bits (the launcher checks P xcols xrows < 2^32); the wave's
    // rows start at Z row w_rofs
    const uint32_t plane = (uint32_t)w_xcols * (uint32_t)w_xrows;
    const float2 *Xc = X + (size_t)(w_zc0 + cl) * w_xrows + w_rofs;
    float kc[8];
    int ki[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) { kc[k] = -INFINITY; ki[k] = 0x7fffffff; }
    // this role's classes [ca, ce) of Z and pass-B blocks [lb0, lb1)
    const int ca = 2 * role_part(NPA, role, NT), ce = min(P1, 2 * role_part(NPA, role + 1, NT));
    const int lb0 = 2 * role_part(Q2, role, NT), lb1 = min(P2, 2 * role_part(Q2, role + 1, NT));
    auto zload = [&](int row) {
        const float2 *xr = Xc + row;
        return [=](int j) {
            float2 v;
            asm volatile("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];"
                         : "=f"(v.x), "=f"(v.y)
                         : "l"(xr + (uint32_t)j * plane));
            return v;
        };
    };
    float2 na[P2], nb[P2];   // the first class pair of this thread's next row
    if (lr < w_rows && ca < ce) load_pair<P1, P2>(ca, min(ca + 1, ce - 1), zload(lr), na, nb);
    for (int base = 0; base < w_rows; base += ROWS) {
        const int row = base + lr;
        const bool active = row < w_rows;
        const int grow = w_row0 + row;
        // this row's reference: its factors in pass-B order
        const float4 *Dr = reinterpret_cast<const float4 *>(
            Dinv + ((size_t)(grow / sp.nshifts - w_r0) * w_dcols + cl) * DLEN);
        if (active) passA_pk<P1, P2>(ca, ce, zload(row), slab, ROWS, twa, twb, tw, na, nb);
        asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(32 * NT) : "memory");
        if (row + ROWS < w_rows && ca < ce) load_pair<P1, P2>(ca, min(ca + 1, ce - 1), zload(row + ROWS), na, nb);
        float best = -INFINITY;
        int brot = 0;
        if (active) {
            if constexpr (WRITE) {
                float *cc_out = ccall + ((size_t)perm[w_col0 + cl] * sp.nrs_total + grow) * sp.N;
                passB_all<P1, P2, EU>(lb0, lb1, slab, ROWS, tw, Dr, sp.escale, cc_out, best, brot);
            } else {
                passB_search<P1, P2, EU>(lb0, lb1, slab, ROWS, tw, Dr, sp.escale, best, brot);
            }
            if (role > 0) { xfer_c[(role - 1) * ROWS + lr] = best; xfer_r[(role - 1) * ROWS + lr] = brot; }
        }
        asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(32 * NT) : "memory");
        if (active && role == 0) {
#pragma unroll
            for (int r = 1; r < NT; ++r) {
                const float oc = xfer_c[(r - 1) * ROWS + lr];
                const int orot = xfer_r[(r - 1) * ROWS + lr];
                if (oc > best || (oc == best && orot < brot)) { best = oc; brot = orot; }
            }
            if (best != -INFINITY) {
                // insert into the running top-8 (kept sorted)
                float c = best;
                int id = grow * sp.N + brot;
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    if (ranks_above(c, id, kc[k], ki[k])) {
                        const float tc = kc[k];
                        const int ti = ki[k];
                        kc[k] = c; ki[k] = id; c = tc; id = ti;
                    }
                }
            }
        }
    }
    // merge the role-0 lists with the particle's running top-8 (lowest id among equal
    // correlations); the slab space holds the candidates now
    __syncthreads();
    float *ccs = reinterpret_cast<float *>(smem4);                 // [8 ROWS + 8]
    int *ids = reinterpret_cast<int *>(ccs + 8 * ROWS + 8);
    if (role == 0) {
#pragma unroll
        for (int k = 0; k < 8; ++k) { ccs[8 * lr + k] = kc[k]; ids[8 * lr + k] = ki[k]; }
    }
    float2 *cp = cand + (size_t)(w_col0 + cl) * 8;
    if (t < 8) {
        const float2 c = cp[t];
        ccs[8 * ROWS + t] = c.x;
        ids[8 * ROWS + t] = __float_as_int(c.y);
    }
    __syncthreads();
    if (t < 32) {
        const int n = 8 * ROWS + 8;
        float keep_c = -INFINITY;
        int keep_i = -1;
        for (int it = 0; it < 8; ++it) {
            float bc = -INFINITY;
            int bi = 0x7fffffff, bpos = -1;
            for (int e = t; e < n; e += 32) {
                const float c = ccs[e];
                const int id = ids[e];
                if (c != -INFINITY && ranks_above(c, id, bc, bi)) { bc = c; bi = id; bpos = e; }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const float oc = __shfl_xor_sync(0xffffffffu, bc, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                const int op = __shfl_xor_sync(0xffffffffu, bpos, o);
                if (ranks_above(oc, oi, bc, bi)) { bc = oc; bi = oi; bpos = op; }
            }
            if (t == it) { keep_c = bc; keep_i = bc == -INFINITY ? -1 : bi; }
            if (bpos >= 0 && t == (bpos & 31)) ccs[bpos] = -INFINITY;
            __syncwarp();
        }
        if (t < 8) cp[t] = make_float2(keep_c, __int_as_float(keep_i));
    }
}

// ---------------------------------------------------------------------------------------
// FP32 m-domain re-score of the top-ntop candidates of each particle (particle frame):
// X(m) = 4 sum_k UA[m][rs][k] conj(UB[m][col][k]) from the FP32 spectra, the FP64
// normaliser from the |ref|^2 and CTF^2 spectra, the same transform and argmax.  One block
// per particle, its ntop <= 8 candidates in four phases:
//   A  Y(c, j) = (wgt_j / P) sum_k conj(RU[r_c][j][k]) CV[col][j][k] in FP64, a thread per (c, j);
//   B  D(c, rho) from Y by the length-P/2 FP64 transform of the packed half spectrum (the
//      normaliser's k_norm_fft, split H1 x H2 = P/2), stored as 1/sqrt(D * sqsum_ptcl);
//   C  X(c, m) in FP32, a thread per (c, m);
//   D  the per-triple transform and argmax of each candidate (two threads each, the halves of
//      triple_corr), then the particle's best (lowest id among equal correlations).
template <int P> struct HalfSplit;
template <> struct HalfSplit<64> { static constexpr int H1 = 8, H2 = 4; };
template <> struct HalfSplit<180> { static constexpr int H1 = 10, H2 = 9; };
template <> struct HalfSplit<300> { static constexpr int H1 = 15, H2 = 10; };
constexpr int RS_MAX = 8;     // candidates per particle
constexpr int RS_THREADS = 256;

template <int P1, int P2> __host__ __device__ constexpr size_t rescore_smem_bytes()
{
    constexpr int P = P1 * P2, J = P / 2 + 1, H = P / 2;
    constexpr int H1 = HalfSplit<P>::H1, H2 = HalfSplit<P>::H2;
    return sizeof(double2) * ((size_t)2 * H + (size_t)RS_MAX * J + (size_t)RS_MAX * H2 * (H1 + 1)) +
           sizeof(float2) * ((size_t)RS_MAX * (P + 1) + (size_t)P * RS_MAX) + sizeof(float) * (size_t)RS_MAX * P;
}

template <int P1, int P2, bool EU>
__global__ void __launch_bounds__(RS_THREADS) k_rescore_md(int ncols, int ntop, int Ks, int N, int nshifts,
                                                           int has_shifts, const TwTables tw,
                                                           const float2 *__restrict__ UA, int rows_pad,
                                                           const float2 *__restrict__ UB, int cols_pad,
                                                           const double2 *__restrict__ RU,
                                                           const double2 *__restrict__ CV, const float *__restrict__ sqp,
                                                           const float2 *__restrict__ cand, const int *__restrict__ perm,
                                                           int c0, pftcc_best *__restrict__ out)
{
    constexpr int P = P1 * P2, J = P / 2 + 1, H = P / 2, M = P + 1;
    constexpr int H1 = HalfSplit<P>::H1, H2 = HalfSplit<P>::H2;
    extern __shared__ float4 smem4[];
    double2 *tw_h = reinterpret_cast<double2 *>(smem4);            // [H] w_{P/2}^{-e}
    double2 *wp = tw_h + H;                                         // [H] w_P^{+e}
    double2 *Ys = wp + H;                                           // [RS_MAX][J]
    double2 *buf = Ys + RS_MAX * J;                                 // [RS_MAX][H2][H1 + 1]
    float2 *Xs = reinterpret_cast<float2 *>(buf + RS_MAX * H2 * (H1 + 1));   // [RS_MAX][M]
    float2 *slab = Xs + RS_MAX * M;                                 // [P][RS_MAX]
    float *Ds = reinterpret_cast<float *>(slab + P * RS_MAX);       // [RS_MAX][P]
    __shared__ int rs_s[RS_MAX];
    __shared__ float bc_s[RS_MAX];
    __shared__ int bi_s[RS_MAX];
    const int cl = c0 + blockIdx.x;
    if (cl >= c0 + ncols) return;
    const int t = threadIdx.x;
    const int nc = min(ntop, RS_MAX);
    if (t < nc) {
        const int id = __float_as_int(cand[(size_t)cl * 8 + t].y);
        rs_s[t] = id >= 0 ? id / N : -1;
    }
    for (int e = t; e < H; e += blockDim.x) {
        double sn, cs;
        sincospi(-2.0 * e / H, &sn, &cs);
        tw_h[e] = make_double2(cs, sn);
        sincospi(2.0 * e / P, &sn, &cs);
        wp[e] = make_double2(cs, sn);
    }
    __syncthreads();
    // A: Y, eight lanes per (candidate, j) over the shells (coalesced reads), summed by shuffles;
    // the loop runs the same trips in every warp so that the shuffles see all lanes
    const int l8 = t & 7, grp = t >> 3;
    constexpr int NGRP = RS_THREADS / 8;
    for (int base = 0; base < nc * J; base += NGRP) {
        const int e = base + grp;
        const int c = e / J, j = e - c * J;
        const int rs = e < nc * J ? rs_s[c] : -1;
        double yr = 0.0, yi = 0.0;
        if (rs >= 0) {
            const double2 *ru = RU + ((size_t)(rs / nshifts) * J + j) * Ks;
            const double2 *cv = CV + ((size_t)cl * J + j) * Ks;
            for (int k = l8; k < Ks; k += 8) {
                const double2 u = ru[k], v = cv[k];
                yr += u.x * v.x + u.y * v.y;
                yi += u.x * v.y - u.y * v.x;
            }
        }
#pragma unroll
        for (int o = 4; o; o >>= 1) {
            yr += __shfl_xor_sync(0xffffffffu, yr, o);
            yi += __shfl_xor_sync(0xffffffffu, yi, o);
        }
        if (e < nc * J && l8 == 0) {
            const double wgt = ((j == 0 || 2 * j == P) ? 1.0 : 2.0) / P;
            Ys[c * J + j] = make_double2(wgt * yr, wgt * yi);
        }
    }
    __syncthreads();
    // B: D, pass 1 (c, n1) then pass 2 (c, k2)
    for (int e = t; e < nc * H1; e += blockDim.x) {
        const int c = e / H1, n1 = e - c * H1;
        const double2 *y = Ys + c * J;
        double2 x[H2];
#pragma unroll
        for (int n2 = 0; n2 < H2; ++n2) {
            const int j = n1 + H1 * n2;
            double2 hj, hh;
            if (j == 0) {
                hj = make_double2(y[0].x, 0.0);
                hh = make_double2(y[H].x, 0.0);
            } else {
                const double2 a = y[j], b = y[H - j];
                hj = make_double2(0.5 * a.x, 0.5 * a.y);
                hh = make_double2(0.5 * b.x, -0.5 * b.y);
            }
            const double2 ev = sfft::d_add(hj, hh), od = sfft::d_mul(sfft::d_sub(hj, hh), wp[j]);
            x[n2] = make_double2(ev.x - od.y, -(ev.y + od.x));   // conj(ev + i od)
        }
        sfft::DFFT<H2, H1>::run(x, tw_h);
        double2 *row = buf + (size_t)c * H2 * (H1 + 1) + n1;
#pragma unroll
        for (int k2 = 0; k2 < H2; ++k2)
            row[k2 * (H1 + 1)] = (k2 == 0 || n1 == 0) ? x[k2] : sfft::d_mul(x[k2], tw_h[n1 * k2]);
    }
    __syncthreads();
    const double sq = (double)sqp[cl];
    for (int e = t; e < nc * H2; e += blockDim.x) {
        const int c = e / H2, k2 = e - c * H2;
        const double2 *row = buf + ((size_t)c * H2 + k2) * (H1 + 1);
        double2 x[H1];
#pragma unroll
        for (int n1 = 0; n1 < H1; ++n1) x[n1] = row[n1];
        sfft::DFFT<H1, H2>::run(x, tw_h);
#pragma unroll
        for (int k1 = 0; k1 < H1; ++k1) {
            const int l = k2 + H2 * k1;
            if constexpr (EU) {   // -(D + sum_k w_k |ptcl_k|^2) / 2
                Ds[c * P + 2 * l] = (float)(-0.5 * (x[k1].x + sq));
                Ds[c * P + 2 * l + 1] = (float)(-0.5 * (-x[k1].y + sq));
            } else {
                Ds[c * P + 2 * l] = (float)(1.0 / sqrt(x[k1].x * sq));
                Ds[c * P + 2 * l + 1] = (float)(1.0 / sqrt(-x[k1].y * sq));
            }
        }
    }
    // C: X, eight lanes per (candidate, m) over the shells as in A
    const size_t pa = (size_t)rows_pad * Ks, pb = (size_t)cols_pad * Ks;
    for (int base = 0; base < nc * M; base += NGRP) {
        const int e = base + grp;
        const int c = e / M, m = e - c * M;
        const int rs = e < nc * M ? rs_s[c] : -1;
        float xr = 0.f, xi = 0.f;
        if (rs >= 0) {
            const float2 *a = UA + (size_t)rs * Ks + (size_t)m * pa, *b = UB + (size_t)cl * Ks + (size_t)m * pb;
            for (int k = l8; k < Ks; k += 8) {
                const float2 av = a[k], bv = b[k];
                xr = fmaf(av.x, bv.x, fmaf(av.y, bv.y, xr));
                xi = fmaf(av.y, bv.x, fmaf(-av.x, bv.y, xi));
            }
        }
#pragma unroll
        for (int o = 4; o; o >>= 1) {
            xr += __shfl_xor_sync(0xffffffffu, xr, o);
            xi += __shfl_xor_sync(0xffffffffu, xi, o);
        }
        if (e < nc * M && l8 == 0) Xs[c * M + m] = make_float2(4.f * xr, 4.f * xi);
    }
    __syncthreads();
    // D: transform and argmax per candidate, two lanes of warp 0 per candidate (lanes 2c, 2c + 1):
    // pass A by classes (class 0 and the first half of the mirror pairs; the rest and the
    // middle class), pass B by blocks [0, LB) and [LB, P2); the halves' maxima are combined
    // with the lowest rotation among equal maxima
    if (t < 32) {
        constexpr int NPAIR = (P1 + 1) / 2, PM = 1 + (NPAIR - 1) / 2, LB = (P2 + 1) / 2;
        const int c = t >> 1, half = t & 1;
        const bool act = c < nc;
        const int rs = act ? rs_s[c] : -1;
        float best = -INFINITY;
        int brot = 0;
        float2 *sl = slab + (act ? c : 0);
        auto getx = [&](int j) { return Xs[c * M + j]; };
        auto dinv = [&](int rho) { return Ds[c * P + rho]; };
        if (rs >= 0) {
            if (half == 0) {
                passA_class0<P1, P2>(getx, sl, RS_MAX, tw);
                passA_pairs<P1, P2>(1, PM, getx, sl, RS_MAX, tw);
            } else {
                passA_pairs<P1, P2>(PM, NPAIR, getx, sl, RS_MAX, tw);
                passA_mid<P1, P2>(getx, sl, RS_MAX, tw);
            }
        }
        __syncwarp();
        if (rs >= 0)
            passB<P1, P2, decltype(dinv), EU>(half ? LB : 0, half ? P2 : LB, sl, RS_MAX, tw, dinv,
                                              1.0f / (2.0f * (float)N), nullptr, best, brot);
        const float ob = __shfl_xor_sync(0xffffffffu, best, 1);
        const int orot = __shfl_xor_sync(0xffffffffu, brot, 1);
        if (ob > best || (ob == best && orot < brot)) { best = ob; brot = orot; }
        if (act && half == 0) {
            bc_s[c] = best;
            bi_s[c] = rs < 0 ? 0x7fffffff : rs * N + brot;
        }
    }
    __syncthreads();
    if (t == 0) {
        float b = -INFINITY;
        int bid = 0x7fffffff;
        for (int i = 0; i < nc; ++i) {
            const float c = bc_s[i];
            const int id = bi_s[i];
            if (id != 0x7fffffff && (c > b || (c == b && id < bid))) { b = c; bid = id; }
        }
        pftcc_best o;
        if (bid == 0x7fffffff) { o.iref = 0; o.irot = 0; o.ishift = -1; o.corr = -INFINITY; }
        else {
            const int rs2 = bid / N, rot = bid - rs2 * N;
            o.iref = rs2 / nshifts + 1;
            o.ishift = has_shifts ? rs2 % nshifts : -1;
            o.irot = rot + 1;
            o.corr = b;
        }
        out[perm[cl]] = o;
    }
}

// ---------------------------------------------------------------------------------------
static void fill_tw(TwTables &tw, int P)
{
    for (int e = 0; e < P; ++e) {
        const double a = -2.0 * M_PI * e / P, b = -2.0 * M_PI * e / (2.0 * P);
        tw.wP[e] = make_float2((float)cos(a), (float)sin(a));
        tw.wN[e] = make_float2((float)cos(b), (float)sin(b));
        tw.pc[e] = make_float2(tw.wP[e].x, tw.wP[e].x);
        tw.ps[e] = make_float2(tw.wP[e].y, tw.wP[e].y);
        tw.pn[e] = make_float2(-tw.wP[e].y, -tw.wP[e].y);
    }
}

bool stage2_fast_supported(int P) { return P == 64 || P == 180 || P == 300; }

// the inner factor P2 of the split P = P1 x P2 used for each supported length
int stage2_fast_p2(int P) { return P == 64 ? 8 : P == 180 ? 15 : P == 300 ? 20 : 0; }

// floats of normalising factors per (reference, particle) the search's pass B reads
int stage2_fast_dlen(int P)
{
    switch (P) {
    case 64: return s2_dlen<8, 8>();
    case 180: return s2_dlen<12, 15>();
    case 300: return s2_dlen<15, 20>();
    default: return P;
    }
}

template <int P1, int P2>
static cudaError_t launch_s2(pftcc_handle *h, const S2Fast &sp, int blocks, const S2Wave *waves_dev, float2 *cand,
                             float *ccall, const int *perm, bool eu)
{
    TwTables tw;
    fill_tw(tw, P1 * P2);
    // row slabs of P complex (the two-lane layout): 128 rows in flight up to P = 200, 64
    // beyond; NT threads per row
    constexpr int ROWS = P1 * P2 <= 200 ? 128 : 64;
    constexpr int NT = S2_THREADS_PER_ROW;
    const size_t smem = (size_t)((P2 + 1) / 2) * P1 * 2 * ROWS * sizeof(float2) +
                        (size_t)P1 * P2 * (sizeof(float4) + sizeof(float2)) +
                        (size_t)(NT - 1) * ROWS * (sizeof(float) + sizeof(int));
    auto kern = ccall ? (eu ? k_stage2_fast<P1, P2, ROWS, NT, true, true> : k_stage2_fast<P1, P2, ROWS, NT, true, false>)
                      : (eu ? k_stage2_fast<P1, P2, ROWS, NT, false, true> : k_stage2_fast<P1, P2, ROWS, NT, false, false>);
    cudaError_t e = smem_limit((const void *)kern, smem);
    if (e != cudaSuccess) return e;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_STAGE2);
    kern<<<blocks, NT * ROWS, smem, h->stream>>>(sp, tw, waves_dev, cand, ccall, perm);
    return cudaGetLastError();
}

// every wave of the list in one launch, one block per column (blk0 filled in)
cudaError_t launch_stage2_waves(pftcc_handle *h, int P, std::vector<S2Wave> &waves, int nshifts, int nrs_total,
                                float2 *cand, float *ccall, const int *perm, int eu)
{
    UmmaState &us = h->ws.umma;
    const int nw = (int)waves.size();
    if (nw == 0) return cudaSuccess;
    long long blocks = 0;
    for (S2Wave &w : waves) {
        if ((unsigned long long)P * w.xcols * w.xrows >= (1ull << 32) || w.cols <= 0 || w.rows <= 0 ||
            w.zc0 + w.cols > w.xcols || w.rofs + w.rows > w.xrows)
            return cudaErrorInvalidValue;
        w.blk0 = (int)blocks;
        blocks += w.cols;
    }
    if (blocks >= (1LL << 31)) return cudaErrorInvalidValue;
    if (us.s2waves_cap < nw) {
        dev_free(h, us.d_s2waves);
        us.d_s2waves = nullptr;
        us.s2waves_cap = 0;
        const int cap = std::max(nw, 16);
        if (dev_alloc(h, (void **)&us.d_s2waves, (size_t)cap * sizeof(S2Wave), "stage-2 waves") != PFTCC_OK)
            return cudaErrorMemoryAllocation;
        us.s2waves_cap = cap;
    }
    if (stage_upload(h, us.d_s2waves, waves.data(), (size_t)nw * sizeof(S2Wave), "stage-2 waves") != PFTCC_OK)
        return cudaErrorInvalidValue;
    S2Fast sp{nshifts, 2 * P, nrs_total, nw, 1.0f / (2.0f * (float)(2 * P))};
    switch (P) {
    case 64: return launch_s2<8, 8>(h, sp, (int)blocks, us.d_s2waves, cand, ccall, perm, eu != 0);
    case 180: return launch_s2<12, 15>(h, sp, (int)blocks, us.d_s2waves, cand, ccall, perm, eu != 0);
    case 300: return launch_s2<15, 20>(h, sp, (int)blocks, us.d_s2waves, cand, ccall, perm, eu != 0);
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_stage2_fast(pftcc_handle *h, int P, int rows, int xrows, int xcols, int row0, int nshifts, int r0,
                               int dcols, int col0, int cols, int nrs_total, const float2 *X, const float *Dinv,
                               float2 *cand, float *ccall, const int *perm, int eu)
{
    std::vector<S2Wave> w(1);
    w[0] = S2Wave{X, Dinv, row0, rows, 0, xrows, xcols, col0, cols, 0, r0, dcols, 0, 0};
    return launch_stage2_waves(h, P, w, nshifts, nrs_total, cand, ccall, perm, eu);
}

template <int P1, int P2, bool EU>
static cudaError_t launch_rs(pftcc_handle *h, int ncols, int ntop, int Ks, int nshifts, int has_shifts,
                             const float2 *UA, int rows_pad, const float2 *UB, int cols_pad, const double2 *RU,
                             const double2 *CV, const float *sqp, const float2 *cand, const int *perm, int c0,
                             pftcc_best *out)
{
    constexpr int P = P1 * P2;
    TwTables tw;
    fill_tw(tw, P);
    if (ntop < 1 || ntop > RS_MAX) return cudaErrorInvalidValue;
    const size_t smem = rescore_smem_bytes<P1, P2>();
    cudaError_t e = smem_limit((const void *)k_rescore_md<P1, P2, EU>, smem);
    if (e != cudaSuccess) return e;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_EXACT);
    k_rescore_md<P1, P2, EU><<<ncols, RS_THREADS, smem, h->stream>>>(
        ncols, ntop, Ks, 2 * P, nshifts, has_shifts, tw, UA, rows_pad, UB, cols_pad, RU, CV, sqp, cand, perm, c0, out);
    return cudaGetLastError();
}

template <int P1, int P2>
static cudaError_t launch_rs_eu(pftcc_handle *h, int eu, int ncols, int ntop, int Ks, int nshifts, int has_shifts,
                                const float2 *UA, int rows_pad, const float2 *UB, int cols_pad, const double2 *RU,
                                const double2 *CV, const float *sqp, const float2 *cand, const int *perm, int c0,
                                pftcc_best *out)
{
    if (eu)
        return launch_rs<P1, P2, true>(h, ncols, ntop, Ks, nshifts, has_shifts, UA, rows_pad, UB, cols_pad, RU, CV,
                                       sqp, cand, perm, c0, out);
    return launch_rs<P1, P2, false>(h, ncols, ntop, Ks, nshifts, has_shifts, UA, rows_pad, UB, cols_pad, RU, CV, sqp,
                                    cand, perm, c0, out);
}

cudaError_t launch_rescore_md(pftcc_handle *h, int P, int ncols, int ntop, int Ks, int nshifts, int has_shifts,
                              const float2 *UA, int rows_pad, const float2 *UB, int cols_pad, const double2 *RU,
                              const double2 *CV, const float *sqp, const float2 *cand, const int *perm, int c0,
                              pftcc_best *out, int eu)
{
    switch (P) {
    case 64: return launch_rs_eu<8, 8>(h, eu, ncols, ntop, Ks, nshifts, has_shifts, UA, rows_pad, UB, cols_pad, RU, CV, sqp, cand, perm, c0, out);
    case 180: return launch_rs_eu<12, 15>(h, eu, ncols, ntop, Ks, nshifts, has_shifts, UA, rows_pad, UB, cols_pad, RU, CV, sqp, cand, perm, c0, out);
    case 300: return launch_rs_eu<15, 20>(h, eu, ncols, ntop, Ks, nshifts, has_shifts, UA, rows_pad, UB, cols_pad, RU, CV, sqp, cand, perm, c0, out);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace pftcc
