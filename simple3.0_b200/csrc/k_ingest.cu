// k_ingest.cu -- particle ingestion: prepimg4align (simple_strategy2D3D_common.f90:316-366) for a
// batch of real-space particle images, ending in the half-plane FTs that polarize grids.
//
// The reference's chain for one particle image of side B (rmat(x, y), x fastest):
//   noise_norm (simple_image.f90:6623-6640) against the background outside the disc of radius
//     msk; fft (fwd_ft :5773-5782: shift_phorig, r2c, / B^2); shift2Dserial([-x, -y]) (:6149-6174)
//     when |x| or |y| > SHTHRESH = 0.001; the CTF phase flip (simple_ctf.f90 apply_serial 'flip'
//     :312-403) for CTFFLAG_YES; ifft (bwd_ft :5784-5791: c2r, shift_phorig); clip to the centred
//     boxmatch window (:6471-6516); mask 'soft' (:6208-6300): zero_background (:5176-5203) and the
//     cosine edge cosedge (simple_math.f90:1089-1103); fft and the factor boxmatch^2 / B^2.
// Here:
//   k_ingest_norm   one block per image: FP64 background mean and (n-1) deviation, the image
//                   normalised into the FFT input;
//   cuFFT R2C       B x B, batched;
//   k_ingest_freq   one thread per half-plane component: times the shift phase (its angle in
//                   FP64, the phasor rounded to FP32 as the reference's cmplx(..., sp)) and the
//                   sign of the CTF (evaluated in FP64) over B^2.  The phase-origin swaps before
//                   the forward and after the inverse transform multiply the spectrum by
//                   (-1)^(h+k) twice and cancel.  The columns h = 0 and h = B/2 are replaced by
//                   their Hermitian parts -- what a c2r transform keeps of them -- so that the
//                   C2R input is a valid half spectrum;
//   cuFFT C2R       B x B, batched, unnormalised;
//   k_ingest_mask   one block per image: the centred boxmatch window, the lower medians of its
//                   four border lines (rank selection in shared memory), the cosine edge (of the
//                   inner mask, the focus mask or msk, :349-358), the division by the gridding's
//                   instrument function for griddev 'yes' (:360-362), and the quadrant swap of the
//                   final fft's phase origin folded into the store, with the factor 1 / B^2
//                   (= 1 / boxmatch^2 of fwd_ft times boxmatch^2 / B^2);
//   cuFFT R2C       boxmatch x boxmatch, batched: the half-plane cmat(h, k), k at its physical index.
#include "pftcc_internal.cuh"

#include <cufft.h>

#include <algorithm>
#include <string>

#define CK(expr, what)                                       \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return cuda_err(h, e_, what); \
    } while (0)
#define ST(expr)                       \
    do {                               \
        int s_ = (expr);               \
        if (s_ != PFTCC_OK) return s_; \
    } while (0)

namespace pftcc {

struct IngestState {
    int B = 0, Bm = 0, batch = 0;
    cufftHandle fwd = 0, inv = 0, fwdm = 0;
    bool have_fwd = false, have_inv = false, have_fwdm = false;
    float *R = nullptr;     // [batch][B][B]
    float2 *Z = nullptr;    // [batch][B][B/2+1]
    float *Rm = nullptr;    // [batch][Bm][Bm]
};

constexpr int IN_THREADS = 256;

__device__ __forceinline__ double in_block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < IN_THREADS / 32; ++w) t += red[w];
    return t;
}

// noise_norm with lmsk = disc of radius msk about (B/2 + 1, B/2 + 1), 1-based (disc_2 :506-523,
// cendist :2719-2748); background = outside the disc
__global__ void __launch_bounds__(IN_THREADS) k_ingest_norm(const float *__restrict__ imgs, int B, float msk,
                                                            float *__restrict__ out)
{
    __shared__ double red[IN_THREADS / 32];
    const float *src = imgs + (size_t)blockIdx.x * B * B;
    float *dst = out + (size_t)blockIdx.x * B * B;
    const int c = B / 2 + 1;
    const double m = (double)msk;
    double s = 0.0, n = 0.0;
    for (int e = threadIdx.x; e < B * B; e += blockDim.x) {
        const int i = e % B + 1, j = e / B + 1;
        const double di = i - c, dj = j - c;
        if (!(sqrt(di * di + dj * dj) <= m)) { s += src[e]; n += 1.0; }
    }
    s = in_block_sum(s, red);
    n = in_block_sum(n, red);
    double ave = s / n;
    if (!(fabs(ave) > 1e-10)) ave = 0.0;
    double ep = 0.0, vs = 0.0;
    for (int e = threadIdx.x; e < B * B; e += blockDim.x) {
        const int i = e % B + 1, j = e / B + 1;
        const double di = i - c, dj = j - c;
        if (!(sqrt(di * di + dj * dj) <= m)) {
            const double v = (double)src[e] - ave;
            ep += v;
            vs += v * v;
        }
    }
    ep = in_block_sum(ep, red);
    vs = in_block_sum(vs, red);
    const double var = (vs - ep * ep / n) / (n - 1.0);
    const double inv = (var == var && var > 0.0) ? 1.0 / sqrt(var) : 1.0;
    for (int e = threadIdx.x; e < B * B; e += blockDim.x) dst[e] = (float)(((double)src[e] - ave) * inv);
}

// sign(1, tval) of apply_serial 'flip': tval = sin(pi wl s2 (df - wl^2 s2 Cs / 2) + phshift + ampc),
// constructor :54-70, init :73-81, evalPhSh :88-98, eval_df :185-189 (phshift always added, as
// apply_serial passes ctfparms%phshift), in FP64
__device__ float ctf_flip_sign(const pftcc_ctfparams &c, double s2, double ang)
{
    const double kv = 1000.0 * (double)c.kv;
    const double wl = (12.26 / sqrt(kv + (0.9784 * kv * kv) / 1.0e6)) / (double)c.smpd;
    const double cs = ((double)c.cs * 1.0e7) / (double)c.smpd;
    const double ampc = atan((double)c.fraca / sqrt(1.0 - (double)c.fraca * c.fraca));
    const double sc = 1.0e4 / (double)c.smpd;
    const double dfx = (double)c.dfx * sc, dfy = (double)c.dfy * sc;
    const double angast = (double)c.angast / 180.0 * 3.141592653589793;
    const double df = 0.5 * (dfx + dfy + cos(2.0 * (ang - angast)) * (dfx - dfy));
    const double chi = 3.141592653589793 * wl * s2 * (df - 0.5 * wl * wl * s2 * cs) + (double)c.phshift + ampc;
    return sin(chi) >= 0.0 ? 1.f : -1.f;
}

__device__ __forceinline__ float2 in_factor(int B, int h, int k, bool shift, float sh1, float sh2, bool flip,
                                            const pftcc_ctfparams &cp, float scale)
{
    float fr = scale, fi = 0.f;
    if (shift) {
        const double a = (double)h * (double)sh1 + (double)k * (double)sh2;
        double sa, ca;
        sincos(a, &sa, &ca);
        fr = (float)ca * scale;
        fi = (float)sa * scale;
    }
    if (flip) {
        const double hinv = (double)h / B, kinv = (double)k / B;
        const float sg = ctf_flip_sign(cp, hinv * hinv + kinv * kinv, atan2((double)k, (double)h));
        fr *= sg;
        fi *= sg;
    }
    return make_float2(fr, fi);
}

__device__ __forceinline__ float2 cmulf(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// xy [n][2], flag [n] (CTFFLAG_NO 0, YES 1, FLIP 2), ctf [n] (read for flag 1 only)
__global__ void __launch_bounds__(IN_THREADS) k_ingest_freq(float2 *__restrict__ Z, int n, int B,
                                                            const float *__restrict__ xy, const int *__restrict__ flag,
                                                            const pftcc_ctfparams *__restrict__ ctf)
{
    const int H = B / 2 + 1;
    const long long total = (long long)n * B * H;
    const float shconst = 3.14159265358979f / (float)(B / 2);   // PI / real(ldim / 2.) in single precision
    const float scale = 1.f / ((float)B * (float)B);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const int h = (int)(e % H), kp = (int)((e / H) % B), im = (int)(e / ((long long)B * H));
        const float x = xy[2 * im], y = xy[2 * im + 1];
        const bool shift = fabsf(x) > 0.001f || fabsf(y) > 0.001f;
        const float sh1 = -x * shconst, sh2 = -y * shconst;
        const bool flip = flag[im] == 1;
        pftcc_ctfparams cp;
        if (flip) cp = ctf[im];
        const int k = kp < B / 2 ? kp : kp - B;
        float2 *img = Z + (size_t)im * B * H;
        if (h != 0 && h != B / 2) {
            img[(size_t)kp * H + h] = cmulf(img[(size_t)kp * H + h], in_factor(B, h, k, shift, sh1, sh2, flip, cp, scale));
        } else if (kp <= B / 2) {
            // the pair (h, k), (h, -k) of a self-Friedel column: both become the Hermitian part
            const int kpm = (B - kp) % B, km = -k == B / 2 ? -B / 2 : -k;
            const float2 a = cmulf(img[(size_t)kp * H + h], in_factor(B, h, k, shift, sh1, sh2, flip, cp, scale));
            const float2 b = cmulf(img[(size_t)kpm * H + h], in_factor(B, h, km, shift, sh1, sh2, flip, cp, scale));
            const float2 s = make_float2(0.5f * (a.x + b.x), 0.5f * (a.y - b.y));
            img[(size_t)kp * H + h] = s;
            if (kpm != kp) img[(size_t)kpm * H + h] = make_float2(s.x, -s.y);
        }
    }
}

// the centred Bm window of the inverse transform, zero_background, cosine edge, quadrant swap and
// 1 / B^2 into the final transform's input.  Shared memory: 4 border lines of Bm floats.
// the gridding's instrument function (gen_instrfun_img, simple_gridding.f90:18-55, with
// kbinterpol%instr, simple_kbinterpol.f90:211-225): w(i) = sinh(y) / y with
// y = sqrt(beta^2 - (pi W x)^2), x = (i - (Bm/2 + 1)) / Bm for the 1-based index i, W = 3 and
// beta = 7.4 (the window of half-width 1.5, :97-103); |x| <= 1/2 always lies below the threshold
// beta / (pi W), so every sample takes the sinh branch
__device__ __forceinline__ double instrfun(int i, int Bm)
{
    const double piW = (double)(3.14159265f * 3.0f), betasq = (double)(7.4f * 7.4f);
    const double x = (double)(float)((float)(i - (Bm / 2 + 1)) / (float)Bm);
    const double y = sqrt(betasq - (piW * x) * (piW * x));
    return y < 1e-10 ? 1.0 : sinh(y) / y;
}

__global__ void __launch_bounds__(IN_THREADS) k_ingest_mask(const float *__restrict__ R, int B, int Bm, float msk,
                                                            float inner, float iwidth, int griddev,
                                                            float *__restrict__ out)
{
    extern __shared__ float lines[];   // [4][Bm]
    __shared__ float med4[4];
    const float *src = R + (size_t)blockIdx.x * B * B;
    float *dst = out + (size_t)blockIdx.x * Bm * Bm;
    const int st = (B - Bm) / 2;
    // border lines of the window: rmat(1, :), rmat(Bm, :), rmat(:, 1), rmat(:, Bm)
    for (int t = threadIdx.x; t < Bm; t += blockDim.x) {
        lines[t] = src[(size_t)(st + t) * B + st];
        lines[Bm + t] = src[(size_t)(st + t) * B + st + Bm - 1];
        lines[2 * Bm + t] = src[(size_t)st * B + st + t];
        lines[3 * Bm + t] = src[(size_t)(st + Bm - 1) * B + st + t];
    }
    __syncthreads();
    // selec(k = Bm/2): the value v_t with #(v < v_t) < k <= #(v <= v_t)
    const int kth = Bm / 2;
    for (int e = threadIdx.x; e < 4 * Bm; e += blockDim.x) {
        const int l = e / Bm;
        const float v = lines[e];
        int lt = 0, le = 0;
        for (int u = 0; u < Bm; ++u) {
            const float w = lines[l * Bm + u];
            lt += w < v;
            le += w <= v;
        }
        if (lt < kth && kth <= le) med4[l] = v;   // equal values for every such t
    }
    __syncthreads();
    double med = ((double)med4[0] + (double)med4[1] + (double)med4[2] + (double)med4[3]) / 4.0;
    if (!(fabs(med) > 1e-10)) med = 0.0;
    int minlen = (int)floor(2.0 * ((double)msk + 6.0) + 0.5);
    if (minlen > Bm) minlen = Bm;
    const double maxrad = (double)(minlen / 2), width = 2.0 * (maxrad - (double)msk);
    const double scale = 1.0 / ((double)B * (double)B);
    for (int e = threadIdx.x; e < Bm * Bm; e += blockDim.x) {
        const int i = e % Bm + 1, j = e / Bm + 1;   // 1-based x, y
        const int iq = i <= Bm / 2 ? i : Bm + 1 - i, jq = j <= Bm / 2 ? j : Bm + 1 - j;
        const double cx = -Bm / 2.0 + (iq - 1), cy = -Bm / 2.0 + (jq - 1);
        const double rad = sqrt(cx * cx + cy * cy);
        double w = 1.0;
        if (rad >= maxrad) w = 0.0;
        else if (rad >= maxrad - width) w = (cos(((rad - (maxrad - width)) / width) * 3.141592653589793) + 1.0) / 2.0;
        if (inner > 0.f) {   // cosedge_inner (simple_math.f90:1128-1140): zero inside inner - width
            const double mi = (double)inner, wi = (double)iwidth;
            if (rad < mi - wi) w = 0.0;
            else if (rad <= mi) w *= (1.0 + cos(3.141592653589793 * (mi - rad) / wi)) / 2.0;
        }
        if (w > 0.9999) w = 1.0;
        double v = ((double)src[(size_t)(st + j - 1) * B + st + i - 1] - med) * w;
        if (griddev) v /= instrfun(i, Bm) * instrfun(j, Bm);   // div_by_instrfun (simple_polarizer.f90:111-116)
        const int io = (i - 1 + Bm / 2) % Bm, jo = (j - 1 + Bm / 2) % Bm;   // shift_phorig
        dst[(size_t)jo * Bm + io] = (float)(v * scale);
    }
}

static int plan2d(pftcc_handle *h, cufftHandle *p, int B, cufftType t, int batch)
{
    int dims[2] = {B, B};
    cufftResult r = cufftPlanMany(p, 2, dims, nullptr, 1, 0, nullptr, 1, 0, t, batch);
    if (r != CUFFT_SUCCESS) return set_err(h, PFTCC_ERR_CUDA, "cuFFT plan (" + std::to_string((int)r) + ")");
    r = cufftSetStream(*p, h->stream);
    if (r != CUFFT_SUCCESS) return set_err(h, PFTCC_ERR_CUDA, "cuFFT stream (" + std::to_string((int)r) + ")");
    return PFTCC_OK;
}

void ingest_free(pftcc_handle *h)
{
    IngestState *s = static_cast<IngestState *>(h->ingest);
    if (!s) return;
    if (s->have_fwd) cufftDestroy(s->fwd);
    if (s->have_inv) cufftDestroy(s->inv);
    if (s->have_fwdm) cufftDestroy(s->fwdm);
    dev_free(h, s->R);
    dev_free(h, s->Z);
    dev_free(h, s->Rm);
    delete s;
    h->ingest = nullptr;
}

int ingest_batch_max(int B)
{
    // scratch per image: R, Z, Rm (<= B^2 floats each, Z (B/2+1) B complex): ~1 GiB per batch
    const size_t per = (size_t)B * B * 4 * 4;
    return (int)std::max<size_t>(1, std::min<size_t>(4096, (1ull << 30) / per));
}

// n <= cap images; the cuFFT plans and scratch serve cap images per call (a shorter batch is
// transformed at the full count, the surplus slots holding stale data that nothing reads), so a
// tail batch needs no new plans; cm_out holds cap half-plane images
int ingest_images(pftcc_handle *h, const float *imgs_dev, int n, int cap, int B, const float *xy_dev,
                  const int *flag_dev, const pftcc_ctfparams *ctf_dev, const pftcc_prep_opts &o, float2 *cm_out)
{
    const float msk = o.msk;
    // the final soft mask: inner mask, else focus mask, else msk (prepimg4align :349-358)
    const float fmsk = o.inner > 0.f ? msk : (o.focusmsk > 0.f ? o.focusmsk : msk);
    const float iwidth = o.width > 0.f ? o.width : 10.f;
    const int Bm = h->g.box;
    IngestState *s = static_cast<IngestState *>(h->ingest);
    if (s && (s->B != B || s->Bm != Bm || s->batch != cap)) {
        CK(cudaStreamSynchronize(h->stream), "ingest");
        ingest_free(h);
        s = nullptr;
    }
    if (!s) {
        s = new IngestState();
        h->ingest = s;
        s->B = B;
        s->Bm = Bm;
        s->batch = cap;
        ST(dev_alloc(h, (void **)&s->R, (size_t)cap * B * B * sizeof(float), "ingest real"));
        ST(dev_alloc(h, (void **)&s->Z, (size_t)cap * B * (B / 2 + 1) * sizeof(float2), "ingest spectra"));
        ST(dev_alloc(h, (void **)&s->Rm, (size_t)cap * Bm * Bm * sizeof(float), "ingest masked"));
        CK(cudaMemsetAsync(s->R, 0, (size_t)cap * B * B * sizeof(float), h->stream), "ingest");
        CK(cudaMemsetAsync(s->Rm, 0, (size_t)cap * Bm * Bm * sizeof(float), h->stream), "ingest");
        ST(plan2d(h, &s->fwd, B, CUFFT_R2C, cap));
        s->have_fwd = true;
        ST(plan2d(h, &s->inv, B, CUFFT_C2R, cap));
        s->have_inv = true;
        ST(plan2d(h, &s->fwdm, Bm, CUFFT_R2C, cap));
        s->have_fwdm = true;
    }
    if (n <= 0) return PFTCC_OK;
    PFTCC_LAUNCH(h);
    {
        KTimer kt(h, PFTCC_K_POLARIZE);
        k_ingest_norm<<<n, IN_THREADS, 0, h->stream>>>(imgs_dev, B, msk, s->R);
    }
    CK(cudaGetLastError(), "ingest norm");
    if (cufftExecR2C(s->fwd, s->R, reinterpret_cast<cufftComplex *>(s->Z)) != CUFFT_SUCCESS)
        return set_err(h, PFTCC_ERR_CUDA, "cuFFT forward");
    const long long total = (long long)n * B * (B / 2 + 1);
    PFTCC_LAUNCH(h);
    {
        KTimer kt(h, PFTCC_K_POLARIZE);
        k_ingest_freq<<<(int)std::min<long long>((total + IN_THREADS - 1) / IN_THREADS, 8192), IN_THREADS, 0,
                        h->stream>>>(s->Z, n, B, xy_dev, flag_dev, ctf_dev);
    }
    CK(cudaGetLastError(), "ingest spectra");
    if (cufftExecC2R(s->inv, reinterpret_cast<cufftComplex *>(s->Z), s->R) != CUFFT_SUCCESS)
        return set_err(h, PFTCC_ERR_CUDA, "cuFFT inverse");
    PFTCC_LAUNCH(h);
    {
        KTimer kt(h, PFTCC_K_POLARIZE);
        k_ingest_mask<<<n, IN_THREADS, 4 * Bm * sizeof(float), h->stream>>>(s->R, B, Bm, fmsk, o.inner, iwidth,
                                                                           o.griddev, s->Rm);
    }
    CK(cudaGetLastError(), "ingest mask");
    if (cufftExecR2C(s->fwdm, s->Rm, reinterpret_cast<cufftComplex *>(cm_out)) != CUFFT_SUCCESS)
        return set_err(h, PFTCC_ERR_CUDA, "cuFFT forward (boxmatch)");
    return PFTCC_OK;
}

}  // namespace pftcc
