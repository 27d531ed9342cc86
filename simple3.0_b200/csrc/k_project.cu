// k_project.cu -- polar projection of a volume's Fourier transform: the references of a
// refine3D round (simple_projector.f90: expand_cmat :66-132, fproject_polar :218-239,
// interp_fcomp_norm / interp_fcomp_grid :269-307; simple_ori.f90 euler2m :1275-1284).
//
//   k_expand_cmat    the cube cmat_exp(h, k, m), h, k, m in [-E, E], E = box/2 + 2, of the
//                    volume's half FT: each logical address wrapped cyclically into
//                    [-box/2, box/2] x [-box/2, box/2 - 1]^2 and read with Friedel symmetry
//                    (negative h: conjugate of (-h, -k, -m)), times factor; one thread per
//                    cube element, [m][k][h] order;
//   k_fproject_polar one thread per (reference, shell, rotation) sample: loc = (x, y, 0) R
//                    with (x, y) the sample's polar coordinates and R the orientation's
//                    rotation matrix, the 3x3x3 Kaiser-Bessel window around nint(loc)
//                    (Whalf = 1.5: W = 3, beta = 7.4), weights the product of the axes'
//                    apodisations, the sum normalised by the weights' sum unless griddev;
//                    written into the reference set as the polar FT [ref][K][P].
#include "pftcc_internal.cuh"

#include <algorithm>

namespace pftcc {

// I0 by the Abramowitz & Stegun 9.8.1 / 9.8.2 polynomial approximations (the reference's
// bessi0, simple_kbinterpol.f90:229-252), in FP64
__device__ double kb_i0(double x)
{
    if (x < 3.75) {
        double y = x / 3.75;
        y = y * y;
        return 1.0 + y * (3.5156229 + y * (3.0899424 + y * (1.2067492 + y * (0.2659732 + y * (0.0360768 + y * 0.0045813)))));
    }
    const double y = 3.75 / x;
    return (0.39894228 + y * (0.01328592 + y * (0.00225319 + y * (-0.00157565 + y * (0.00916281 +
            y * (-0.02057706 + y * (0.02635537 + y * (-0.01647633 + y * 0.00392377)))))))) * exp(x) / sqrt(x);
}

// apod (simple_kbinterpol.f90:130-141), Whalf = 1.5
__device__ double kb_apod(double x)
{
    const double whalf = 1.5, W = 3.0, beta = 7.4;
    if (fabs(x) > whalf) return 0.0;
    double a = (2.0 / W) * x;
    a = 1.0 - a * a;
    if (a < 0.0) a = 0.0;
    return (1.0 / W) * kb_i0(beta * sqrt(a));
}

// cyci_1d (simple_math.f90:746-757)
__device__ __forceinline__ int cyc1(int lo, int hi, int i)
{
    if (i > hi) return lo + (i - hi) - 1;
    if (i < lo) return hi - (lo - i) + 1;
    return i;
}

__global__ void k_expand_cmat(int box, const float2 *__restrict__ half, float factor, float2 *__restrict__ cube)
{
    const int E = box / 2 + 2, S = 2 * E + 1, ld = box / 2 + 1;
    const long long n = (long long)S * S * S;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int hh = (int)(e % S), kk = (int)((e / S) % S), mm = (int)(e / ((long long)S * S));
        int h = cyc1(-box / 2, box / 2, hh - E), k = cyc1(-box / 2, box / 2 - 1, kk - E),
            m = cyc1(-box / 2, box / 2 - 1, mm - E);
        float sgn = 1.f;
        if (h < 0) { h = -h; k = -k; m = -m; sgn = -1.f; }
        const int p2 = k + (k < 0 ? box : 0), p3 = m + (m < 0 ? box : 0);
        const float2 v = half[((size_t)p3 * box + p2) * ld + h];
        cube[e] = make_float2(factor * v.x, factor * sgn * v.y);
    }
}

// R: 9 doubles per reference, row-major r(i, j) of euler2m; mask: K ints or null.  loc is formed
// in FP64 so that the window's nint follows the exact rotated coordinate.
__global__ void __launch_bounds__(256) k_fproject_polar(Geom g, int box, const float2 *__restrict__ cube,
                                                        const float *__restrict__ polar, const double *__restrict__ R,
                                                        const int *__restrict__ mask, int n, int griddev,
                                                        float2 *__restrict__ out)
{
    const int E = box / 2 + 2, S = 2 * E + 1;
    const int N = g.N, P = g.P, K = g.K;
    const long long total = (long long)n * K * P;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % P), ik = (int)((e / P) % K), r = (int)(e / ((long long)K * P));
        double accr = 0.0, acci = 0.0;
        if (!mask || mask[ik]) {
            const double *rm = R + (size_t)r * 9;
            const double vx = polar[(size_t)ik * 2 * N + i], vy = polar[(size_t)ik * 2 * N + N + i];
            double loc[3];
#pragma unroll
            for (int j = 0; j < 3; ++j) loc[j] = vx * rm[j] + vy * rm[3 + j];
            int w0[3];
            double wa[3][3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                w0[d] = (int)round(loc[d]) - 1;   // nint: half away from zero
#pragma unroll
                for (int l = 0; l < 3; ++l) wa[d][l] = kb_apod((double)(w0[d] + l) - loc[d]);
            }
            double wsum = 0.0;
#pragma unroll
            for (int c = 0; c < 3; ++c)
#pragma unroll
                for (int b = 0; b < 3; ++b) {
                    const float2 *row = cube + ((size_t)(w0[2] + c + E) * S + (w0[1] + b + E)) * S + (w0[0] + E);
#pragma unroll
                    for (int a = 0; a < 3; ++a) {
                        const double w = wa[0][a] * wa[1][b] * wa[2][c];
                        const float2 v = __ldg(row + a);
                        accr += w * v.x;
                        acci += w * v.y;
                        wsum += w;
                    }
                }
            if (!griddev) { accr /= wsum; acci /= wsum; }
        }
        out[e] = make_float2((float)accr, (float)acci);
    }
}

// I1 by the Abramowitz & Stegun 9.8.3 / 9.8.4 polynomial approximations (the reference's
// bessi1, simple_kbinterpol.f90:282-308), x >= 0, in FP64
__device__ double kb_i1(double x)
{
    if (x < 3.75) {
        double y = x / 3.75;
        y = y * y;
        return x * (0.5 + y * (0.87890594 + y * (0.51498869 + y * (0.15084934 + y * (0.2658733e-1 +
                    y * (0.301532e-2 + y * 0.32411e-3))))));
    }
    const double y = 3.75 / x;
    return (0.39894228 + y * (-0.3988024e-1 + y * (-0.362018e-2 + y * (0.163801e-2 + y * (-0.1031555e-1 +
            y * (0.2282967e-1 + y * (-0.2895312e-1 + y * (0.1787654e-1 + y * (-0.420059e-2))))))))) *
           exp(x) / sqrt(x);
}

// dapod (simple_kbinterpol.f90:179-192): d apod / dx = -4 beta x I1(beta s) / (s W^3),
// s = sqrt(1 - (2x/W)^2), 0 where s^2 <= 0
__device__ double kb_dapod(double x)
{
    const double W = 3.0, beta = 7.4;
    double a = (2.0 / W) * x;
    a = 1.0 - a * a;
    if (a <= 0.0) return 0.0;
    const double s = sqrt(a);
    return -4.0 * beta * x * kb_i1(beta * s) / s / (W * W * W);
}

// fdf_project_polar (simple_projector.f90:245-267) with fdf_interp_fcomp (:338-400), one
// thread per (reference, shell, rotation) sample: the normalised interpolation N / D of
// interp_fcomp_norm and its derivatives with respect to the three Euler angles (per radian).
// d loc / d e_j = vec dR_j (euler2dm); each tap's weight derivative is the sum over the axes of
// -dapod(win - loc) d loc / d e_j times the other two axes' apod, and
// dfcomp_j = (sum wd_j c * D - N sum wd_j) / D^2.  FP64 throughout, FP32 out as set_ref_fcomp /
// set_dref_fcomp store it.  RD: 36 doubles per reference, R then dR/de1..3, row-major.
__global__ void __launch_bounds__(256) k_fdf_project_polar(Geom g, int box, const float2 *__restrict__ cube,
                                                           const float *__restrict__ polar,
                                                           const double *__restrict__ RD, int n,
                                                           float2 *__restrict__ out, float2 *__restrict__ dout)
{
    const int E = box / 2 + 2, S = 2 * E + 1;
    const int N = g.N, P = g.P, K = g.K;
    const long long total = (long long)n * K * P;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(e % P), ik = (int)((e / P) % K), r = (int)(e / ((long long)K * P));
        const double *rm = RD + (size_t)r * 36, *dm = rm + 9;
        const double vx = polar[(size_t)ik * 2 * N + i], vy = polar[(size_t)ik * 2 * N + N + i];
        double loc[3], dl[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            loc[d] = vx * rm[d] + vy * rm[3 + d];
#pragma unroll
            for (int j = 0; j < 3; ++j) dl[j][d] = vx * dm[9 * j + d] + vy * dm[9 * j + 3 + d];
        }
        int w0[3];
        double wa[3][3], da[3][3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            w0[d] = (int)round(loc[d]) - 1;
#pragma unroll
            for (int l = 0; l < 3; ++l) {
                wa[d][l] = kb_apod((double)(w0[d] + l) - loc[d]);
                da[d][l] = kb_dapod((double)(w0[d] + l) - loc[d]);
            }
        }
        double nr = 0.0, ni = 0.0, D = 0.0, njr[3] = {0.0, 0.0, 0.0}, nji[3] = {0.0, 0.0, 0.0},
               dj[3] = {0.0, 0.0, 0.0};
#pragma unroll
        for (int c = 0; c < 3; ++c)
#pragma unroll
            for (int b = 0; b < 3; ++b) {
                const float2 *row = cube + ((size_t)(w0[2] + c + E) * S + (w0[1] + b + E)) * S + (w0[0] + E);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const float2 v = __ldg(row + a);
                    const double w = wa[0][a] * wa[1][b] * wa[2][c];
                    nr += w * v.x;
                    ni += w * v.y;
                    D += w;
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const double wd = -da[0][a] * dl[j][0] * wa[1][b] * wa[2][c] -
                                          wa[0][a] * da[1][b] * dl[j][1] * wa[2][c] -
                                          wa[0][a] * wa[1][b] * da[2][c] * dl[j][2];
                        njr[j] += wd * v.x;
                        nji[j] += wd * v.y;
                        dj[j] += wd;
                    }
                }
            }
        out[e] = make_float2((float)(nr / D), (float)(ni / D));
        const double d2 = D * D;
#pragma unroll
        for (int j = 0; j < 3; ++j)
            dout[((size_t)r * 3 + j) * K * P + (size_t)ik * P + i] =
                make_float2((float)((njr[j] * D - nr * dj[j]) / d2), (float)((nji[j] * D - ni * dj[j]) / d2));
    }
}

cudaError_t launch_fdf_project_polar(pftcc_handle *h, int box, const float2 *cube, const double *RD, int n,
                                     float2 *out, float2 *dout)
{
    const long long total = (long long)n * h->g.K * h->g.P;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_POLARIZE);
    k_fdf_project_polar<<<(int)std::min<long long>((total + 255) / 256, 8192), 256, 0, h->stream>>>(
        h->g, box, cube, h->polar, RD, n, out, dout);
    return cudaGetLastError();
}

cudaError_t launch_expand_cmat(pftcc_handle *h, int box, const float2 *half, float factor, float2 *cube)
{
    const long long S = box + 5, n = S * S * S;
    PFTCC_LAUNCH(h);
    k_expand_cmat<<<(int)std::min<long long>((n + 255) / 256, 4096), 256, 0, h->stream>>>(box, half, factor, cube);
    return cudaGetLastError();
}

cudaError_t launch_fproject_polar(pftcc_handle *h, int box, const float2 *cube, const double *R, const int *mask, int n,
                                  int griddev, float2 *out)
{
    const long long total = (long long)n * h->g.K * h->g.P;
    PFTCC_LAUNCH(h);
    KTimer kt(h, PFTCC_K_POLARIZE);
    k_fproject_polar<<<(int)std::min<long long>((total + 255) / 256, 8192), 256, 0, h->stream>>>(
        h->g, box, cube, h->polar, R, mask, n, griddev, out);
    return cudaGetLastError();
}

}  // namespace pftcc
