// pftcc_capi.cu -- the C ABI of libpftcc_b200.so (declared in include/pftcc_b200.h):
// handle life cycle, host-side tables (polar grid, shift constants, gridding taps),
// setters/getters and the per-pair and batched correlation entry points.
#include "pftcc_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

using namespace pftcc;

namespace pftcc {

int set_err(pftcc_handle *h, int code, const std::string &msg)
{
    if (h) h->last_err = msg;
    return code;
}

cudaError_t smem_limit(const void *kernel, size_t bytes)
{
    struct Limit { int dev; const void *fn; size_t max; };
    static std::mutex mu;
    static std::vector<Limit> known;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(mu);
    for (const Limit &l : known)
        if (l.dev == dev && l.fn == kernel) return bytes <= l.max ? cudaSuccess : cudaErrorInvalidValue;
    int optin = 0;
    if ((e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess) return e;
    cudaFuncAttributes fa;
    if ((e = cudaFuncGetAttributes(&fa, kernel)) != cudaSuccess) return e;
    const int max = optin - (int)fa.sharedSizeBytes;
    if ((e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max)) != cudaSuccess) return e;
    known.push_back(Limit{dev, kernel, (size_t)max});
    return bytes <= (size_t)max ? cudaSuccess : cudaErrorInvalidValue;
}

int cuda_err(pftcc_handle *h, cudaError_t e, const char *what)
{
    if (e == cudaSuccess) return PFTCC_OK;
    const int code = (e == cudaErrorMemoryAllocation) ? PFTCC_ERR_OOM : PFTCC_ERR_CUDA;
    return set_err(h, code, std::string(what) + ": " + cudaGetErrorString(e));
}

// Device memory comes from the device's stream-ordered pool, which keeps up to 32 GB of freed
// memory for reuse: handles created and killed one after another (a queue of chunks) reuse
// the same memory instead of returning to the driver for every buffer.
static cudaError_t pool_ready(int dev)
{
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(mu);
    for (int d : done)
        if (d == dev) return cudaSuccess;
    cudaMemPool_t pool;
    cudaError_t e = cudaDeviceGetDefaultMemPool(&pool, dev);
    if (e != cudaSuccess) return e;
    unsigned long long keep = 32ull << 30;   // bytes of freed memory the pool holds on to
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) return e;
    done.push_back(dev);
    return cudaSuccess;
}

bool capturing(const pftcc_handle *h)
{
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    return cudaStreamIsCapturing(h->stream, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone;
}

int stage_upload(pftcc_handle *h, void *dst_dev, const void *src, size_t bytes, const char *what)
{
    if (bytes == 0) return PFTCC_OK;
    const int a = capturing(h) ? 1 : 0;
    const size_t need = (bytes + 63) / 64 * 64;
    if (h->pin_off[a] + need > h->pin_cap[a]) {
        if (a) return set_err(h, PFTCC_ERR_STATE, std::string("staging of ") + what +
                                                      " during graph capture: run the same call once outside capture first");
        // the arena's earlier contents may still be on their way: drain the stream, then reuse or grow
        cudaError_t e = cudaStreamSynchronize(h->stream);
        if (e != cudaSuccess) return cuda_err(h, e, "staging");
        h->pin_off[0] = 0;
        if (need > h->pin_cap[0]) {
            if (h->pin[0]) cudaFreeHost(h->pin[0]);
            h->pin[0] = nullptr;
            h->pin_cap[0] = 0;
            const size_t cap = std::max<size_t>(need, 1 << 20);
            if ((e = cudaMallocHost(&h->pin[0], cap)) != cudaSuccess) return cuda_err(h, e, "pinned staging");
            h->pin_cap[0] = cap;
        }
    }
    char *stg = static_cast<char *>(h->pin[a]) + h->pin_off[a];
    std::memcpy(stg, src, bytes);
    h->pin_off[a] += need;
    if (!a) h->pin_total += need;
    const cudaError_t e = cudaMemcpyAsync(dst_dev, stg, bytes, cudaMemcpyHostToDevice, h->stream);
    return e == cudaSuccess ? PFTCC_OK : cuda_err(h, e, what);
}

int dev_alloc(pftcc_handle *h, void **p, size_t bytes, const char *what)
{
    *p = nullptr;
    if (bytes == 0) return PFTCC_OK;
    if (capturing(h))
        return set_err(h, PFTCC_ERR_STATE, std::string("device allocation of ") + what +
                                               " during graph capture: run the same call once outside capture first");
    cudaError_t e = pool_ready(h->dev);
    if (e == cudaSuccess) e = cudaMallocAsync(p, bytes, h->stream);
    // the buffer may next be used on another stream (pftcc_set_stream): complete the allocation
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return set_err(h, PFTCC_ERR_OOM, std::string("device allocation failed for ") + what + " (" +
                                              std::to_string(bytes) + " bytes): " + cudaGetErrorString(e));
    }
    return PFTCC_OK;
}

// returns a buffer to the pool in the order of the handle's stream (after its last use there)
void dev_free(pftcc_handle *h, void *p)
{
    if (p) cudaFreeAsync(p, h->stream);
}

int ensure(pftcc_handle *h, void **p, size_t *cap, size_t bytes, const char *what)
{
    if (*cap >= bytes && *p) return PFTCC_OK;
    if (*p) dev_free(h, *p);
    *p = nullptr;
    *cap = 0;
    int st = dev_alloc(h, p, bytes, what);
    if (st == PFTCC_OK) *cap = bytes;
    return st;
}

KTimer::KTimer(pftcc_handle *h_, int cls_) : h(h_), cls(cls_)
{
    if (!h->prof) return;
    for (cudaEvent_t *e : {&a, &b}) {
        if (!h->prof_pool.empty()) { *e = h->prof_pool.back(); h->prof_pool.pop_back(); }
        else if (cudaEventCreate(e) != cudaSuccess) { *e = nullptr; }
    }
    if (a) cudaEventRecord(a, h->stream);
}

KTimer::~KTimer()
{
    if (!a || !b) return;
    cudaEventRecord(b, h->stream);
    h->prof_pending.push_back(pftcc_handle::ProfEv{cls, a, b});
}

}  // namespace pftcc

#define CK(expr, what)                                             \
    do {                                                           \
        cudaError_t e_ = (expr);                                   \
        if (e_ != cudaSuccess) return cuda_err(h, e_, what);       \
    } while (0)
#define ST(expr)                     \
    do {                             \
        int s_ = (expr);             \
        if (s_ != PFTCC_OK) return s_; \
    } while (0)

static int slot_of(const pftcc_handle *h, int iptcl)
{
    if (iptcl < h->pfrom || iptcl > h->pto) return -1;
    return h->pinds[iptcl - h->pfrom] - 1;
}

#define SLOT_OR_FAIL(slot, iptcl)                                                                  \
    const int slot = slot_of(h, iptcl);                                                            \
    if (slot < 0)                                                                                  \
        return set_err(h, PFTCC_ERR_INDEX, "particle index " + std::to_string(iptcl) +             \
                                               " is not held (pfromto/pinds)");

#define REF_OR_FAIL(iref)                                                                            \
    if ((iref) < 1 || (iref) > h->nrefs)                                                             \
        return set_err(h, PFTCC_ERR_INDEX, "reference index " + std::to_string(iref) + " out of range");

// ---------------------------------------------------------------------------------------
// host tables: polar grid and shift constants (new :261-317), single precision where the
// reference is single precision
static void build_tables(pftcc_handle *h)
{
    const Geom &g = h->g;
    const int N = g.N, P = g.P, K = g.K;
    h->h_polar.assign((size_t)K * 2 * N, 0.f);
    h->h_argtransf.assign((size_t)K * N, 0.0);
    h->h_argtransf1.assign(N, 0.0);
    h->angtab.assign(N, 0.f);
    const float twopi = 2.0f * acosf(-1.0f);
    const float ang = twopi / (float)N;
    const float pif = acosf(-1.0f);
    const double A = acos(-1.0) / (double)(g.box / 2);
    for (int irot = 0; irot < N; ++irot) {
        const float a = (float)irot * ang;
        for (int ik = 0; ik < K; ++ik) {
            const int k = g.kfrom + ik;
            h->h_polar[(size_t)ik * 2 * N + irot] = sinf(a) * (float)k;
            h->h_polar[(size_t)ik * 2 * N + N + irot] = -cosf(a) * (float)k;
        }
        h->angtab[irot] = (a / pif) * 180.0f;   // rad2deg
    }
    for (int ik = 0; ik < K; ++ik)
        for (int irot = 0; irot < P; ++irot) {
            h->h_argtransf[(size_t)ik * N + irot] = (double)h->h_polar[(size_t)ik * 2 * N + irot] * A;
            h->h_argtransf[(size_t)ik * N + P + irot] = (double)h->h_polar[(size_t)ik * 2 * N + N + irot] * A;
        }
    for (int irot = 0; irot < P; ++irot) {
        const float a = (float)irot * ang;
        h->h_argtransf1[irot] = (double)sinf(a) * A;
        h->h_argtransf1[P + irot] = (double)(-cosf(a)) * A;
    }
}

// Kaiser-Bessel window with Whalf = KBWINSZ = 1.5 and alpha = KBALPHA = sqrt(2)
// (simple_defs.f90:131-132): W = 3, beta = 7.4 (simple_kbinterpol.f90:92-109), apod
// in single precision around the double precision I0 of :229-252 (Abramowitz &
// Stegun 9.8.1 / 9.8.2).
static double kb_bessi0(double x)
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

static float kb_apod(float x)
{
    const float whalf = 1.5f, W = 3.0f, beta = 7.4f;
    const float twooW = 2.0f / W, oneoW = 1.0f / W;
    if (fabsf(x) > whalf) return 0.f;
    float arg = twooW * x;
    arg = 1.0f - arg * arg;
    return (float)((double)oneoW * kb_bessi0((double)(beta * sqrtf(arg))));
}

static int f_nint(float x) { return (int)(x >= 0.f ? floorf(x + 0.5f) : -floorf(-x + 0.5f)); }

static int cyci(int lo, int hi, int i)
{
    if (i > hi) return lo + (i - hi) - 1;
    if (i < lo) return hi - (lo - i) + 1;
    return i;
}

// init_polarizer (simple_polarizer.f90:41-92): taps [K][P][9] in the order of
// reshape(w, wlen) (window index in x fastest), offsets into cmat(box/2+1, box) with
// the conjugation of get_fcomp2D (simple_image.f90:1894-1907) as a bitwise complement.
static int build_polarizer(pftcc_handle *h, int griddev)
{
    if (h->pol_griddev == griddev && h->pol_off) return PFTCC_OK;
    const Geom &g = h->g;
    const int N = g.N, P = g.P, K = g.K, box = g.box, ld = box / 2 + 1;
    std::vector<int> off((size_t)K * P * 9);
    std::vector<float> wt((size_t)K * P * 9);
    for (int ik = 0; ik < K; ++ik)
        for (int i = 0; i < P; ++i) {
            const float lx = h->h_polar[(size_t)ik * 2 * N + i], ly = h->h_polar[(size_t)ik * 2 * N + N + i];
            const int w1 = f_nint(lx) - 1, w2 = f_nint(ly) - 1;
            float ax[3], ay[3], w[3][3], wsum = 0.f;
            for (int l = 0; l < 3; ++l) {
                ax[l] = kb_apod((float)(w1 + l) - lx);
                ay[l] = kb_apod((float)(w2 + l) - ly);
            }
            for (int m = 0; m < 3; ++m)
                for (int l = 0; l < 3; ++l) {
                    w[l][m] = ax[l] * ay[m];
                    wsum += w[l][m];   // column-major sum(w)
                }
            for (int m = 0; m < 3; ++m)
                for (int l = 0; l < 3; ++l) {
                    const int t = m * 3 + l;
                    const int hh = cyci(-box / 2, box / 2, w1 + l);
                    const int kk = cyci(-box / 2, box / 2 - 1, w2 + m);
                    int p1, p2, conj = 0;
                    if (hh >= 0) { p1 = hh; p2 = kk + (kk < 0 ? box : 0); }
                    else { p1 = -hh; p2 = -kk + (-kk < 0 ? box : 0); conj = 1; }
                    const int o = p2 * ld + p1;
                    off[((size_t)ik * P + i) * 9 + t] = conj ? ~o : o;
                    wt[((size_t)ik * P + i) * 9 + t] = griddev ? w[l][m] : w[l][m] / wsum;
                }
        }
    if (!h->pol_off) {
        ST(dev_alloc(h, (void **)&h->pol_off, off.size() * sizeof(int), "gridding offsets"));
        ST(dev_alloc(h, (void **)&h->pol_w, wt.size() * sizeof(float), "gridding weights"));
    }
    CK(cudaMemcpyAsync(h->pol_off, off.data(), off.size() * sizeof(int), cudaMemcpyHostToDevice, h->stream), "taps");
    CK(cudaMemcpyAsync(h->pol_w, wt.data(), wt.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream), "taps");
    CK(cudaStreamSynchronize(h->stream), "taps");
    h->pol_griddev = griddev;
    return PFTCC_OK;
}

static void free_all(pftcc_handle *h)
{
    void *ptrs[] = {h->refs_even, h->refs_odd, h->ptcls, h->sqsums, h->ctfmats, h->d_iseven, h->d_ctfp, h->polar,
                    h->argtransf, h->argtransf1, h->pol_off, h->pol_w, h->pol_stage, h->d_work, h->d_groups,
                    h->d_out, h->d_shifts, h->d_dout, h->d_best, h->ws.UA, h->ws.UB, h->ws.RU, h->ws.CV,
                    h->ws.RUf, h->ws.CVf, h->ws.D, h->ws.Yn, h->ws.X, h->ws.cand, h->ws.sqp, h->ws.A16, h->ws.B16, h->ws.shifts, h->ws.best,
                    h->ws.cand_ref, h->vol_cube, h->d_sig2, h->d_pxls, h->drefs_even, h->drefs_odd, h->d_optlp,
                    h->d_snorm};
    for (void *p : ptrs) dev_free(h, p);
    umma_free(h);
    ingest_free(h);
    for (auto &p : h->prof_pending) { cudaEventDestroy(p.a); cudaEventDestroy(p.b); }
    for (cudaEvent_t e : h->prof_pool) cudaEventDestroy(e);
    cudaStream_t own = h->own_stream ? h->own_stream : h->stream;
    if (own) cudaStreamDestroy(own);
    for (void *&p : h->pin) { if (p) cudaFreeHost(p); p = nullptr; }
}

static int alloc_ptcl_arrays(pftcc_handle *h)
{
    const size_t KP = (size_t)h->g.K * h->g.P;
    const size_t n = std::max(1, h->nptcls);
    ST(dev_alloc(h, (void **)&h->ptcls, n * KP * sizeof(float2), "particle pfts"));
    ST(dev_alloc(h, (void **)&h->sqsums, n * sizeof(float), "particle square sums"));
    ST(dev_alloc(h, (void **)&h->d_iseven, n, "particle eo flags"));
    ST(dev_alloc(h, (void **)&h->d_ctfp, n * sizeof(pftcc_ctfparams), "ctf parameters"));
    CK(cudaMemsetAsync(h->ptcls, 0, n * KP * sizeof(float2), h->stream), "zero ptcls");
    CK(cudaMemsetAsync(h->sqsums, 0, n * sizeof(float), h->stream), "zero sqsums");
    h->iseven.assign(n, 1);
    CK(cudaMemcpyAsync(h->d_iseven, h->iseven.data(), n, cudaMemcpyHostToDevice, h->stream), "eo");
    h->h_ctfp.assign(n, pftcc_ctfparams{});
    return PFTCC_OK;
}

static int push_iseven(pftcc_handle *h)
{
    CK(cudaMemcpyAsync(h->d_iseven, h->iseven.data(), h->iseven.size(), cudaMemcpyHostToDevice, h->stream), "eo");
    CK(cudaStreamSynchronize(h->stream), "eo");
    return PFTCC_OK;
}

extern "C" {

const char *pftcc_strerror(int s)
{
    switch (s) {
    case PFTCC_OK: return "ok";
    case PFTCC_ERR_ARG: return "invalid argument";
    case PFTCC_ERR_INDEX: return "index out of range";
    case PFTCC_ERR_STATE: return "call out of order";
    case PFTCC_ERR_CUDA: return "CUDA error";
    case PFTCC_ERR_OOM: return "device out of memory";
    case PFTCC_ERR_TIMEOUT: return "device wait timed out";
    case PFTCC_ERR_NODEV: return "no usable sm_100 device";
    case PFTCC_ERR_UNSUPPORTED: return "unsupported mode";
    default: return "unknown status";
    }
}

const char *pftcc_last_error(const pftcc_handle *h) { return h ? h->last_err.c_str() : "null handle"; }
long long pftcc_kernel_launches(const pftcc_handle *h) { return h ? h->launches : 0; }

int pftcc_new(const pftcc_config *cfg, const int *ptcl_mask, const int *eoarr, pftcc_handle **out)
{
    if (!cfg || !out) return PFTCC_ERR_ARG;
    *out = nullptr;
    pftcc_handle *h = new (std::nothrow) pftcc_handle();
    if (!h) return PFTCC_ERR_OOM;
    auto fail = [&](int code, const std::string &msg) {
        fprintf(stderr, "pftcc_new: %s\n", msg.c_str());
        free_all(h);
        delete h;
        return code;
    };
    const pftcc_config c = *cfg;
    // error checks of new :227-243
    if (c.pfromto[1] - c.pfromto[0] + 1 < 1) return fail(PFTCC_ERR_ARG, "nptcls (# of particles) must be > 0");
    if (c.nrefs < 1) return fail(PFTCC_ERR_ARG, "nrefs (# of reference sections) must be > 0");
    if (c.box < 2 || (c.box & 1)) return fail(PFTCC_ERR_ARG, "only even logical dims supported");
    if (c.nrots < 4 || (c.nrots & 1) || c.nrots > 768) return fail(PFTCC_ERR_ARG, "nrots must be even, in [4, 768]");
    if (c.kfromto[0] < 1 || c.kfromto[1] < c.kfromto[0] || c.kstop < c.kfromto[0] || c.kstop > c.kfromto[1])
        return fail(PFTCC_ERR_ARG, "need 1 <= kfromto(1) <= kstop <= kfromto(2)");
    if (c.kfromto[1] + 2 > c.box / 2) return fail(PFTCC_ERR_ARG, "kfromto(2) beyond the gridding window of the box");
    if (c.ctf_frame != PFTCC_FRAME_REF && c.ctf_frame != PFTCC_FRAME_PTCL) return fail(PFTCC_ERR_ARG, "bad ctf_frame");
    h->cfg = c;
    h->g.N = c.nrots;
    h->g.P = c.nrots / 2;
    h->g.kfrom = c.kfromto[0];
    h->g.kto = c.kfromto[1];
    h->g.kstop = c.kstop;
    h->g.K = c.kfromto[1] - c.kfromto[0] + 1;
    h->g.Ks = c.kstop - c.kfromto[0] + 1;
    h->g.box = c.box;
    h->nrefs = c.nrefs;
    h->pfrom = c.pfromto[0];
    h->pto = c.pfromto[1];
    const int span = h->pto - h->pfrom + 1;
    h->pinds.assign(span, 0);
    int cnt = 0;
    for (int i = 0; i < span; ++i)
        if (!ptcl_mask || ptcl_mask[i]) h->pinds[i] = ++cnt;   // :278-288
    if (cnt < 1) return fail(PFTCC_ERR_ARG, "the particle mask selects no particle");
    h->nptcls = cnt;
    // device: sm_100 only, no fallback
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        cudaGetLastError();
        return fail(PFTCC_ERR_NODEV, "no CUDA device visible");
    }
    if (c.device < 0 || c.device >= ndev) return fail(PFTCC_ERR_NODEV, "device ordinal out of range");
    // one attribute, not the whole property record (which takes milliseconds to gather)
    int major = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, c.device) != cudaSuccess || major != 10)
        return fail(PFTCC_ERR_NODEV, "device is not sm_100 (B200)");
    h->dev = c.device;
    if (cudaSetDevice(h->dev) != cudaSuccess) return fail(PFTCC_ERR_NODEV, "cudaSetDevice failed");
    if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(PFTCC_ERR_CUDA, "stream creation failed");
    build_tables(h);
    const size_t KP = (size_t)h->g.K * h->g.P;
    int st = PFTCC_OK;
    if ((st = dev_alloc(h, (void **)&h->refs_even, (size_t)h->nrefs * KP * sizeof(float2), "refs even")) ||
        (st = dev_alloc(h, (void **)&h->refs_odd, (size_t)h->nrefs * KP * sizeof(float2), "refs odd")) ||
        (st = dev_alloc(h, (void **)&h->polar, h->h_polar.size() * sizeof(float), "polar")) ||
        (st = dev_alloc(h, (void **)&h->argtransf, h->h_argtransf.size() * sizeof(double), "argtransf")) ||
        (st = dev_alloc(h, (void **)&h->argtransf1, h->h_argtransf1.size() * sizeof(double), "argtransf1")) ||
        (st = alloc_ptcl_arrays(h)))
        return fail(st, h->last_err);
    if (cudaMemsetAsync(h->refs_even, 0, (size_t)h->nrefs * KP * sizeof(float2), h->stream) ||
        cudaMemsetAsync(h->refs_odd, 0, (size_t)h->nrefs * KP * sizeof(float2), h->stream) ||
        cudaMemcpyAsync(h->polar, h->h_polar.data(), h->h_polar.size() * sizeof(float), cudaMemcpyHostToDevice,
                        h->stream) ||
        cudaMemcpyAsync(h->argtransf, h->h_argtransf.data(), h->h_argtransf.size() * sizeof(double),
                        cudaMemcpyHostToDevice, h->stream) ||
        cudaMemcpyAsync(h->argtransf1, h->h_argtransf1.data(), h->h_argtransf1.size() * sizeof(double),
                        cudaMemcpyHostToDevice, h->stream))
        return fail(PFTCC_ERR_CUDA, "initial uploads failed");
    // eo assignment :289-306
    if (eoarr) {
        bool all_m1 = true;
        for (int i = 0; i < span; ++i)
            if (eoarr[i] != -1) all_m1 = false;
        if (!all_m1)
            for (int i = 0; i < span; ++i)
                if (h->pinds[i] > 0) h->iseven[h->pinds[i] - 1] = eoarr[i] == 0;
    }
    if (push_iseven(h) != PFTCC_OK) return fail(PFTCC_ERR_CUDA, h->last_err);
    if (h->cfg.match_filt) {
        // matched-filter mode: ref_optlp = 1 (allocated with source = 1., :255) and the shell factors
        const size_t nf = (size_t)std::max(1, h->nrefs) * h->g.Ks;
        std::vector<float> ones(nf, 1.f);
        if ((st = dev_alloc(h, (void **)&h->d_optlp, nf * sizeof(float), "ref_optlp")) ||
            (st = dev_alloc(h, (void **)&h->d_snorm, 2 * nf * sizeof(float), "shell factors")))
            return fail(st, h->last_err);
        if (cudaMemcpyAsync(h->d_optlp, ones.data(), nf * sizeof(float), cudaMemcpyHostToDevice, h->stream) ||
            cudaStreamSynchronize(h->stream))
            return fail(PFTCC_ERR_CUDA, "ref_optlp upload failed");
    }
    *out = h;
    return PFTCC_OK;
}

int pftcc_kill(pftcc_handle *h)
{
    if (!h) return PFTCC_OK;
    cudaSetDevice(h->dev);
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_all(h);
    delete h;
    return PFTCC_OK;
}

}  // extern "C"

// ---- the Euclidean objective's per-particle noise ---------------------------------------
namespace pftcc {
// sigma2_noise columns in slot order on the device -- NaN for a held particle outside the
// assigned fromp:top range, counted in sig_uncovered -- and the pixels per shell
// (setup_pxls_p_shell :879-893: the pixels h, k = 1..kto of the positive quadrant whose
// rounded radius nint(sqrt(h^2 + k^2)) is a shell kfrom..kto)
static int sigma2_build(pftcc_handle *h)
{
    const int K = h->g.K;
    std::vector<float> px(K, 0.f);
    const int kfrom = h->cfg.kfromto[0], kto = h->cfg.kfromto[1];
    for (int a = 1; a <= kto; ++a)
        for (int b = 1; b <= kto; ++b) {
            const int sh = (int)std::lround(std::sqrt((double)(a * a + b * b)));
            if (sh >= kfrom && sh <= kto) px[sh - kfrom] += 1.f;
        }
    const int slots = std::max(1, h->nptcls);
    std::vector<float> col((size_t)slots * K, NAN);
    int uncovered = 0;
    for (size_t gi = 0; gi < h->pinds.size(); ++gi) {
        const int slot = h->pinds[gi] - 1;
        if (slot < 0) continue;
        const int iptcl = h->pfrom + (int)gi;
        if (iptcl < h->sig_from || iptcl > h->sig_to) {
            ++uncovered;
            continue;
        }
        std::memcpy(&col[(size_t)slot * K], &h->h_sig2[(size_t)(iptcl - h->sig_from) * K], K * sizeof(float));
    }
    dev_free(h, h->d_sig2);
    h->d_sig2 = nullptr;
    ST(dev_alloc(h, (void **)&h->d_sig2, col.size() * sizeof(float), "sigma2_noise"));
    if (!h->d_pxls) ST(dev_alloc(h, (void **)&h->d_pxls, K * sizeof(float), "pixels per shell"));
    CK(cudaMemcpyAsync(h->d_sig2, col.data(), col.size() * sizeof(float), cudaMemcpyHostToDevice, h->stream), "sigma2");
    CK(cudaMemcpyAsync(h->d_pxls, px.data(), K * sizeof(float), cudaMemcpyHostToDevice, h->stream), "pxls_p_shell");
    CK(cudaStreamSynchronize(h->stream), "sigma2");
    h->sig_uncovered = uncovered;
    h->sig_dirty = 0;
    return PFTCC_OK;
}

int snorm_ready(pftcc_handle *h, int r0, int n)
{
    if (!h->cfg.match_filt || n <= 0) return PFTCC_OK;
    if (!h->d_snorm || !h->d_optlp) return set_err(h, PFTCC_ERR_STATE, "matched-filter arrays missing");
    CK(launch_shellnorm(h, r0, n), "shell factors");
    return PFTCC_OK;
}

int exact_objfun_ok(pftcc_handle *h)
{
    if (h->objfun == PFTCC_OBJFUN_EUCLID && h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "in the particle CTF frame the Euclidean objective is served by the "
                                                 "m-domain search (PFTCC_PREC_FP32 / PFTCC_PREC_BF16X3)");
    return PFTCC_OK;
}

int euclid_ready(pftcc_handle *h, int may_alloc)
{
    if (h->h_sig2.empty())
        return set_err(h, PFTCC_ERR_STATE, "the Euclidean objective needs sigma2_noise: call pftcc_assign_sigma2_noise");
    if (h->sig_dirty || !h->d_sig2) {
        if (!may_alloc)
            return set_err(h, PFTCC_ERR_STATE, "sigma2_noise is not on the device for the current particles: assign it "
                                               "again (pftcc_assign_sigma2_noise) before this call");
        ST(sigma2_build(h));
    }
    if (h->sig_uncovered)
        return set_err(h, PFTCC_ERR_STATE, std::to_string(h->sig_uncovered) +
                                               " held particles lie outside the assigned sigma2_noise range");
    return PFTCC_OK;
}
}  // namespace pftcc

extern "C" {

int pftcc_set_objfun(pftcc_handle *h, int objfun)
{
    if (!h) return PFTCC_ERR_ARG;
    if (objfun != PFTCC_OBJFUN_CC && objfun != PFTCC_OBJFUN_EUCLID)
        return set_err(h, PFTCC_ERR_ARG, "objfun must be PFTCC_OBJFUN_CC or PFTCC_OBJFUN_EUCLID");
    std::lock_guard<std::mutex> lk(h->mtx);
    h->objfun = objfun;
    return PFTCC_OK;
}

int pftcc_set_pssnr(pftcc_handle *h, int on)
{
    if (!h) return PFTCC_ERR_ARG;
    if (on && !h->cfg.match_filt)
        return set_err(h, PFTCC_ERR_STATE, "set_pssnr: l_pssnr needs the matched-filter mode (cfg.match_filt)");
    std::lock_guard<std::mutex> lk(h->mtx);
    h->pssnr = on ? 1 : 0;
    h->ws.ptcl_spectra_valid = 0;
    return PFTCC_OK;
}

int pftcc_set_ref_optlp(pftcc_handle *h, int iref, const float *optlp)
{
    if (!h || !optlp) return set_err(h, PFTCC_ERR_ARG, "set_ref_optlp: bad arguments");
    REF_OR_FAIL(iref);
    if (!h->cfg.match_filt || !h->d_optlp)
        return set_err(h, PFTCC_ERR_STATE, "set_ref_optlp: the handle was created without match_filt");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    CK(cudaMemcpyAsync(h->d_optlp + (size_t)(iref - 1) * h->g.Ks, optlp, h->g.Ks * sizeof(float),
                       cudaMemcpyHostToDevice, h->stream), "set_ref_optlp");
    CK(cudaStreamSynchronize(h->stream), "set_ref_optlp");
    return PFTCC_OK;
}

int pftcc_prep_matchfilt_batch(pftcc_handle *h, int n, const int *iptcl, const int *iref, const int *irot)
{
    if (!h || n < 0 || (n > 0 && (!iptcl || !iref || !irot))) return set_err(h, PFTCC_ERR_ARG, "prep_matchfilt: bad arguments");
    if (n == 0 || !h->cfg.match_filt) return PFTCC_OK;   // memoize_fft only: nothing to hold (:997-1001)
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    if (h->cfg.with_ctf && !h->ctf_ready)
        return set_err(h, PFTCC_ERR_STATE, "CTF is on but create_polar_absctfmats has not been called");
    struct Req { int iref, slot, irot, pad; };
    std::vector<Req> rq;
    rq.reserve(n);
    std::vector<char> seen(std::max(1, h->nptcls), 0);
    for (int i = 0; i < n; ++i) {
        const int sl = slot_of(h, iptcl[i]);
        if (sl < 0) return set_err(h, PFTCC_ERR_INDEX, "prep_matchfilt: particle not held");
        if (iref[i] < 0 || iref[i] > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "prep_matchfilt: iref out of range");
        if (irot[i] < 1 || irot[i] > h->g.N) return set_err(h, PFTCC_ERR_INDEX, "prep_matchfilt: irot out of range");
        if (seen[sl]) return set_err(h, PFTCC_ERR_ARG, "prep_matchfilt: a particle appears twice in one batch");
        seen[sl] = 1;
        if (iref[i] == 0) continue;   // iref 0: memoization only (:997)
        rq.push_back(Req{iref[i] - 1, sl, irot[i], 0});
    }
    if (rq.empty()) return PFTCC_OK;
    ST(ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>(rq.size() * sizeof(Req), 4096), "matchfilt requests"));
    CK(cudaMemcpyAsync(h->d_work, rq.data(), rq.size() * sizeof(Req), cudaMemcpyHostToDevice, h->stream), "matchfilt");
    CK(launch_prep_matchfilt(h, h->d_work, (int)rq.size()), "prep_matchfilt kernel");
    CK(cudaStreamSynchronize(h->stream), "prep_matchfilt");
    h->ws.ptcl_spectra_valid = 0;
    return PFTCC_OK;
}

int pftcc_prep_matchfilt(pftcc_handle *h, int iptcl, int iref, int irot)
{
    return pftcc_prep_matchfilt_batch(h, 1, &iptcl, &iref, &irot);
}

int pftcc_assign_sigma2_noise(pftcc_handle *h, int fromp, int top, const float *sigma2)
{
    if (!h || !sigma2 || top < fromp) return set_err(h, PFTCC_ERR_ARG, "assign_sigma2_noise: bad arguments");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    h->h_sig2.assign(sigma2, sigma2 + (size_t)(top - fromp + 1) * h->g.K);
    h->sig_from = fromp;
    h->sig_to = top;
    h->sig_dirty = 1;
    return sigma2_build(h);
}

int pftcc_reallocate_ptcls(pftcc_handle *h, int nptcls, const int *pinds)
{
    if (!h || nptcls < 1 || !pinds) return set_err(h, PFTCC_ERR_ARG, "reallocate_ptcls: bad arguments");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    int lo = pinds[0], hi = pinds[0];
    for (int i = 0; i < nptcls; ++i) { lo = std::min(lo, pinds[i]); hi = std::max(hi, pinds[i]); }
    h->pfrom = lo;
    h->pto = hi;
    h->pinds.assign(hi - lo + 1, 0);
    for (int i = 0; i < nptcls; ++i) h->pinds[pinds[i] - lo] = i + 1;   // :551-554
    if (nptcls != h->nptcls) {
        CK(cudaStreamSynchronize(h->stream), "sync");
        void *old[] = {h->ptcls, h->sqsums, h->d_iseven, h->d_ctfp, h->ctfmats};
        for (void *p : old) dev_free(h, p);
        h->ptcls = nullptr; h->sqsums = nullptr; h->d_iseven = nullptr; h->d_ctfp = nullptr; h->ctfmats = nullptr;
        h->nptcls = nptcls;
        ST(alloc_ptcl_arrays(h));
    } else {
        const size_t KP = (size_t)h->g.K * h->g.P;
        CK(cudaMemsetAsync(h->ptcls, 0, (size_t)nptcls * KP * sizeof(float2), h->stream), "zero ptcls");
        CK(cudaMemsetAsync(h->sqsums, 0, (size_t)nptcls * sizeof(float), h->stream), "zero sqsums");
        h->iseven.assign(nptcls, 1);
    }
    h->ctf_ready = 0;
    h->ws.ptcl_spectra_valid = 0;
    h->sig_dirty = 1;
    if (!h->h_sig2.empty()) ST(sigma2_build(h));
    return push_iseven(h);
}

// ---- setters ---------------------------------------------------------------------------
int pftcc_set_refs(pftcc_handle *h, int first_iref, int n, const float *pfts, int iseven)
{
    if (!h || !pfts || n < 0) return set_err(h, PFTCC_ERR_ARG, "set_refs: bad arguments");
    if (first_iref < 1 || first_iref + n - 1 > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "set_refs: range");
    cudaSetDevice(h->dev);
    const size_t KP = (size_t)h->g.K * h->g.P;
    float2 *dst = (iseven ? h->refs_even : h->refs_odd) + (size_t)(first_iref - 1) * KP;
    CK(cudaMemcpyAsync(dst, pfts, (size_t)n * KP * sizeof(float2), cudaMemcpyHostToDevice, h->stream), "set_refs");
    CK(cudaStreamSynchronize(h->stream), "set_refs");
    return PFTCC_OK;
}

int pftcc_set_ref_pft(pftcc_handle *h, int iref, const float *pft, int iseven)
{
    return pftcc_set_refs(h, iref, 1, pft, iseven);
}

int pftcc_set_ptcls(pftcc_handle *h, int first_slot, int n, const float *pfts)
{
    if (!h || !pfts || n < 0) return set_err(h, PFTCC_ERR_ARG, "set_ptcls: bad arguments");
    if (first_slot < 0 || first_slot + n > h->nptcls) return set_err(h, PFTCC_ERR_INDEX, "set_ptcls: range");
    cudaSetDevice(h->dev);
    const size_t KP = (size_t)h->g.K * h->g.P;
    CK(cudaMemcpyAsync(h->ptcls + (size_t)first_slot * KP, pfts, (size_t)n * KP * sizeof(float2),
                       cudaMemcpyHostToDevice, h->stream), "set_ptcls");
    CK(launch_sqsums(h, first_slot, n), "sqsums");
    CK(cudaStreamSynchronize(h->stream), "set_ptcls");
    h->ws.ptcl_spectra_valid = 0;
    return PFTCC_OK;
}

int pftcc_set_ptcl_pft(pftcc_handle *h, int iptcl, const float *pft)
{
    if (!h) return PFTCC_ERR_ARG;
    SLOT_OR_FAIL(slot, iptcl);
    return pftcc_set_ptcls(h, slot, 1, pft);
}

int pftcc_set_ref_fcomp(pftcc_handle *h, int iref, int irot, int k, const float *comp, int iseven)
{
    if (!h || !comp) return PFTCC_ERR_ARG;
    REF_OR_FAIL(iref);
    if (irot < 1 || irot > h->g.P || k < h->g.kfrom || k > h->g.kto)
        return set_err(h, PFTCC_ERR_INDEX, "set_ref_fcomp: (irot, k) out of range");
    cudaSetDevice(h->dev);
    const size_t KP = (size_t)h->g.K * h->g.P;
    float2 *dst = (iseven ? h->refs_even : h->refs_odd) + (size_t)(iref - 1) * KP +
                  (size_t)(k - h->g.kfrom) * h->g.P + (irot - 1);
    CK(cudaMemcpyAsync(dst, comp, sizeof(float2), cudaMemcpyHostToDevice, h->stream), "set_ref_fcomp");
    CK(cudaStreamSynchronize(h->stream), "set_ref_fcomp");
    return PFTCC_OK;
}

int pftcc_cp_even2odd_ref(pftcc_handle *h, int iref)
{
    if (!h) return PFTCC_ERR_ARG;
    REF_OR_FAIL(iref);
    cudaSetDevice(h->dev);
    const size_t KP = (size_t)h->g.K * h->g.P;
    CK(cudaMemcpyAsync(h->refs_odd + (iref - 1) * KP, h->refs_even + (iref - 1) * KP, KP * sizeof(float2),
                       cudaMemcpyDeviceToDevice, h->stream), "cp_even2odd_ref");
    CK(cudaStreamSynchronize(h->stream), "cp_even2odd_ref");
    return PFTCC_OK;
}

int pftcc_cp_even_ref2ptcl(pftcc_handle *h, int iref, int iptcl)
{
    if (!h) return PFTCC_ERR_ARG;
    REF_OR_FAIL(iref);
    SLOT_OR_FAIL(slot, iptcl);
    cudaSetDevice(h->dev);
    const size_t KP = (size_t)h->g.K * h->g.P;
    CK(cudaMemcpyAsync(h->ptcls + slot * KP, h->refs_even + (iref - 1) * KP, KP * sizeof(float2),
                       cudaMemcpyDeviceToDevice, h->stream), "cp_even_ref2ptcl");
    CK(launch_sqsums(h, slot, 1), "sqsums");
    CK(cudaStreamSynchronize(h->stream), "cp_even_ref2ptcl");
    h->ws.ptcl_spectra_valid = 0;
    return PFTCC_OK;
}

int pftcc_swap_ptclsevenodd(pftcc_handle *h)
{
    if (!h) return PFTCC_ERR_ARG;
    for (auto &e : h->iseven) e = !e;
    return push_iseven(h);
}

int pftcc_set_eo(pftcc_handle *h, int iptcl, int is_even)
{
    if (!h) return PFTCC_ERR_ARG;
    SLOT_OR_FAIL(slot, iptcl);
    h->iseven[slot] = is_even ? 1 : 0;
    return push_iseven(h);
}

int pftcc_set_eos(pftcc_handle *h, const int *eoarr)
{
    if (!h || !eoarr) return PFTCC_ERR_ARG;
    bool all_m1 = true;
    for (int i = 0; i < h->nptcls; ++i)
        if (eoarr[i] != -1) all_m1 = false;
    for (int i = 0; i < h->nptcls; ++i) h->iseven[i] = all_m1 ? 1 : (eoarr[i] == 0);
    return push_iseven(h);
}

int pftcc_zero_refs_beyond_kstop(pftcc_handle *h)
{
    if (!h) return PFTCC_ERR_ARG;
    cudaSetDevice(h->dev);
    CK(launch_zero_beyond_kstop(h), "zero_refs_beyond_kstop");
    CK(cudaStreamSynchronize(h->stream), "zero_refs_beyond_kstop");
    return PFTCC_OK;
}

// ---- CTF ---------------------------------------------------------------------------------
int pftcc_create_polar_absctfmats(pftcc_handle *h, const pftcc_ctfparams *params)
{
    if (!h || !params) return set_err(h, PFTCC_ERR_ARG, "create_polar_absctfmats: bad arguments");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    for (int i = 0; i < h->nptcls; ++i) {
        const pftcc_ctfparams &p = params[i];
        if (!(p.smpd > 0.f) || !(p.kv > 0.f) || !(p.fraca >= 0.f && p.fraca < 1.f))
            return set_err(h, PFTCC_ERR_ARG, "create_polar_absctfmats: bad ctf parameters for slot " +
                                                 std::to_string(i));
    }
    h->h_ctfp.assign(params, params + h->nptcls);
    if (!h->ctfmats)
        ST(dev_alloc(h, (void **)&h->ctfmats, (size_t)h->nptcls * h->g.K * h->g.P * sizeof(float), "ctfmats"));
    CK(cudaMemcpyAsync(h->d_ctfp, params, (size_t)h->nptcls * sizeof(pftcc_ctfparams), cudaMemcpyHostToDevice,
                       h->stream), "ctf params");
    for (int c0 = 0; c0 < h->nptcls; c0 += 65535) {
        const int n = std::min(65535, h->nptcls - c0);
        CK(launch_ctfmat(h, h->d_ctfp + c0, n, h->ctfmats + (size_t)c0 * h->g.K * h->g.P, 0.f, 0), "ctfmat");
    }
    CK(cudaStreamSynchronize(h->stream), "ctfmat");
    h->ctf_ready = 1;
    h->ws.ptcl_spectra_valid = 0;
    return PFTCC_OK;
}

// ---- polarizer -----------------------------------------------------------------------------
static int polarize_dev(pftcc_handle *h, int first_slot, int n, const float2 *src_dev, int griddev)
{
    ST(build_polarizer(h, griddev));
    for (int c0 = 0; c0 < n; c0 += 65535) {
        const int m = std::min(65535, n - c0);
        const size_t img = (size_t)h->g.box * (h->g.box / 2 + 1);
        CK(launch_polarize(h, src_dev + (size_t)c0 * img, m, first_slot + c0), "polarize");
    }
    h->ws.ptcl_spectra_valid = 0;
    return PFTCC_OK;
}

int pftcc_polarize_ptcls_dev(pftcc_handle *h, int first_slot, int n, const void *cmats_dev, int griddev)
{
    if (!h || !cmats_dev || n < 0) return set_err(h, PFTCC_ERR_ARG, "polarize_ptcls_dev: bad arguments");
    if (first_slot < 0 || first_slot + n > h->nptcls) return set_err(h, PFTCC_ERR_INDEX, "polarize: slot range");
    if (((uintptr_t)cmats_dev & 15) != 0) return set_err(h, PFTCC_ERR_ARG, "polarize: images must be 16-byte aligned");
    cudaSetDevice(h->dev);
    ST(polarize_dev(h, first_slot, n, (const float2 *)cmats_dev, griddev));
    CK(cudaStreamSynchronize(h->stream), "polarize");
    return PFTCC_OK;
}

int pftcc_polarize_ptcls(pftcc_handle *h, int first_slot, int n, const float *cmats, int griddev)
{
    if (!h || !cmats || n < 0) return set_err(h, PFTCC_ERR_ARG, "polarize_ptcls: bad arguments");
    if (first_slot < 0 || first_slot + n > h->nptcls) return set_err(h, PFTCC_ERR_INDEX, "polarize: slot range");
    cudaSetDevice(h->dev);
    const size_t img = (size_t)h->g.box * (h->g.box / 2 + 1) * sizeof(float2);
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>((size_t)n, (256u << 20) / img));
    ST(ensure(h, &h->pol_stage, &h->pol_stage_bytes, (size_t)chunk * img, "polarize staging"));
    for (int c0 = 0; c0 < n; c0 += chunk) {
        const int m = std::min(chunk, n - c0);
        CK(cudaMemcpyAsync(h->pol_stage, (const char *)cmats + (size_t)c0 * img, (size_t)m * img,
                           cudaMemcpyHostToDevice, h->stream), "polarize upload");
        ST(polarize_dev(h, first_slot + c0, m, (const float2 *)h->pol_stage, griddev));
    }
    CK(cudaStreamSynchronize(h->stream), "polarize");
    return PFTCC_OK;
}

// ---- particle ingestion (prepimg4align) ------------------------------------------------
static int prep_ptcls_common(pftcc_handle *h, int first_slot, int n, const float *imgs, int imgs_on_device,
                             int box_in, const float *xy, const int *ctfflag, const pftcc_ctfparams *ctf,
                             const pftcc_prep_opts &o)
{
    if (!h || !imgs || !xy || !ctfflag || n < 0) return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: bad arguments");
    if (first_slot < 0 || first_slot + n > h->nptcls) return set_err(h, PFTCC_ERR_INDEX, "prep_ptcls: slot range");
    const int Bm = h->g.box;
    const float msk = o.msk;
    if (box_in < Bm || (box_in & 1)) return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: box must be even and >= boxmatch");
    if (!(msk > 0.f) || !(msk < 0.5f * Bm)) return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: msk must lie in (0, boxmatch/2)");
    if (!std::isfinite(o.inner) || !std::isfinite(o.width) || !std::isfinite(o.focusmsk) ||
        (o.focusmsk > 0.f && !(o.focusmsk < 0.5f * Bm)) || (o.inner > 0.f && !(o.inner < msk)) ||
        (o.griddev != 0 && o.griddev != 1))
        return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: inner must lie below msk, focusmsk below boxmatch/2, griddev 0 or 1");
    for (int i = 0; i < n; ++i) {
        if (ctfflag[i] < 0 || ctfflag[i] > 2) return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: unsupported CTF flag");
        if (ctfflag[i] == 1 && !ctf) return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: CTFFLAG_YES needs CTF parameters");
        if (!std::isfinite(xy[2 * i]) || !std::isfinite(xy[2 * i + 1]))
            return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: shift not finite");
    }
    if (n == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    const int cap = std::min(n, ingest_batch_max(box_in));
    const size_t img_in = (size_t)box_in * box_in * sizeof(float);
    const size_t img_out = (size_t)Bm * (Bm / 2 + 1) * sizeof(float2);
    // staging: input images (host path), the cap half-plane outputs, per-image descriptors
    const size_t in_bytes = imgs_on_device ? 0 : (size_t)cap * img_in;
    const size_t desc_bytes = (size_t)cap * (2 * sizeof(float) + sizeof(int) + sizeof(pftcc_ctfparams));
    ST(ensure(h, &h->pol_stage, &h->pol_stage_bytes, in_bytes + (size_t)cap * img_out + desc_bytes + 256, "ingest staging"));
    char *base = static_cast<char *>(h->pol_stage);
    float2 *cm = reinterpret_cast<float2 *>(base);
    float *in = reinterpret_cast<float *>(base + (size_t)cap * img_out);
    char *desc = base + (size_t)cap * img_out + in_bytes;
    float *dxy = reinterpret_cast<float *>(desc);
    int *dflag = reinterpret_cast<int *>(desc + (size_t)cap * 2 * sizeof(float));
    pftcc_ctfparams *dctf = reinterpret_cast<pftcc_ctfparams *>(
        (reinterpret_cast<uintptr_t>(dflag + cap) + 15) & ~uintptr_t(15));
    for (int c0 = 0; c0 < n; c0 += cap) {
        const int m = std::min(cap, n - c0);
        const float *src = imgs_on_device ? imgs + (size_t)c0 * box_in * box_in : in;
        if (!imgs_on_device)
            CK(cudaMemcpyAsync(in, imgs + (size_t)c0 * box_in * box_in, (size_t)m * img_in, cudaMemcpyHostToDevice,
                               h->stream), "prep_ptcls upload");
        CK(cudaMemcpyAsync(dxy, xy + 2 * (size_t)c0, (size_t)m * 2 * sizeof(float), cudaMemcpyHostToDevice, h->stream),
           "prep_ptcls shifts");
        CK(cudaMemcpyAsync(dflag, ctfflag + c0, (size_t)m * sizeof(int), cudaMemcpyHostToDevice, h->stream),
           "prep_ptcls flags");
        if (ctf)
            CK(cudaMemcpyAsync(dctf, ctf + c0, (size_t)m * sizeof(pftcc_ctfparams), cudaMemcpyHostToDevice, h->stream),
               "prep_ptcls ctf");
        ST(ingest_images(h, src, m, cap, box_in, dxy, dflag, dctf, o, cm));
        ST(polarize_dev(h, first_slot + c0, m, cm, o.griddev));
        // the staging is reused by the next chunk's uploads
        CK(cudaStreamSynchronize(h->stream), "prep_ptcls");
    }
    return PFTCC_OK;
}

int pftcc_prep_ptcls(pftcc_handle *h, int first_slot, int n, const float *imgs, int box_in, const float *xy,
                     const int *ctfflag, const pftcc_ctfparams *ctf, float msk)
{
    const pftcc_prep_opts o{msk, 0.f, 0.f, 0.f, 0};
    return prep_ptcls_common(h, first_slot, n, imgs, 0, box_in, xy, ctfflag, ctf, o);
}

int pftcc_prep_ptcls_dev(pftcc_handle *h, int first_slot, int n, const void *imgs_dev, int box_in, const float *xy,
                         const int *ctfflag, const pftcc_ctfparams *ctf, float msk)
{
    const pftcc_prep_opts o{msk, 0.f, 0.f, 0.f, 0};
    return prep_ptcls_common(h, first_slot, n, static_cast<const float *>(imgs_dev), 1, box_in, xy, ctfflag, ctf, o);
}

int pftcc_prep_ptcls_opts(pftcc_handle *h, int first_slot, int n, const float *imgs, int box_in, const float *xy,
                          const int *ctfflag, const pftcc_ctfparams *ctf, const pftcc_prep_opts *opts)
{
    if (!opts) return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: no options");
    return prep_ptcls_common(h, first_slot, n, imgs, 0, box_in, xy, ctfflag, ctf, *opts);
}

int pftcc_prep_ptcls_opts_dev(pftcc_handle *h, int first_slot, int n, const void *imgs_dev, int box_in, const float *xy,
                              const int *ctfflag, const pftcc_ctfparams *ctf, const pftcc_prep_opts *opts)
{
    if (!opts) return set_err(h, PFTCC_ERR_ARG, "prep_ptcls: no options");
    return prep_ptcls_common(h, first_slot, n, static_cast<const float *>(imgs_dev), 1, box_in, xy, ctfflag, ctf, *opts);
}

// ---- polar projection of a volume (simple_projector.f90) --------------------------------
}  // extern "C"

// euler2m (simple_ori.f90:1275-1284, rotmat :1350-1390): R = R3(e3) R2(e2) R1(e1), angles in
// degrees, row-major; with dR, euler2dm (simple_ori_light.f90:87-147): dR/de1 = R3 R2 dR1,
// dR/de2 = R3 dR2 R1, dR/de3 = dR3 R2 R1, the derivatives per radian (drotmat :107-146)
void pftcc::host_euler2m(const double e[3], double *R, double *dR)
{
    double m[3][9], d[3][9];
    for (int a = 0; a < 3; ++a) {
        const double t = e[a] * 3.14159265358979323846 / 180.0, c = std::cos(t), sn = std::sin(t);
        double *x = m[a], *y = d[a];
        for (int i = 0; i < 9; ++i) x[i] = y[i] = 0.0;
        if (a == 1) {   // about y (tilt)
            x[0] = c; x[2] = -sn; x[4] = 1.0; x[6] = sn; x[8] = c;
            y[0] = -sn; y[2] = -c; y[6] = c; y[8] = -sn;
        } else {        // about z
            x[0] = c; x[1] = sn; x[3] = -sn; x[4] = c; x[8] = 1.0;
            y[0] = -sn; y[1] = c; y[3] = -c; y[4] = -sn;
        }
    }
    auto mul3 = [](const double *a, const double *b, const double *c, double *out) {
        double t[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double v = 0.0;
                for (int l = 0; l < 3; ++l) v += a[3 * i + l] * b[3 * l + j];
                t[3 * i + j] = v;
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double v = 0.0;
                for (int l = 0; l < 3; ++l) v += t[3 * i + l] * c[3 * l + j];
                out[3 * i + j] = v;
            }
    };
    mul3(m[2], m[1], m[0], R);
    if (dR) {
        mul3(m[2], m[1], d[0], dR);
        mul3(m[2], d[1], m[0], dR + 9);
        mul3(d[2], m[1], m[0], dR + 18);
    }
}

extern "C" {

int pftcc_set_volume_ft(pftcc_handle *h, const float *cmat_half, int box, float factor)
{
    if (!h || !cmat_half || box < 2 || (box & 1)) return set_err(h, PFTCC_ERR_ARG, "set_volume_ft: bad arguments");
    if (h->g.kto > box / 2) return set_err(h, PFTCC_ERR_ARG, "set_volume_ft: kfromto(2) beyond the volume's Nyquist");
    if (!std::isfinite(factor)) return set_err(h, PFTCC_ERR_ARG, "set_volume_ft: factor not finite");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    const size_t half = (size_t)box * box * (box / 2 + 1), S = (size_t)box + 5;
    if (h->vol_box != box) {
        dev_free(h, h->vol_cube);
        h->vol_cube = nullptr;
        h->vol_box = 0;
        ST(dev_alloc(h, (void **)&h->vol_cube, S * S * S * sizeof(float2), "expanded volume FT"));
    }
    float2 *stage = nullptr;
    ST(dev_alloc(h, (void **)&stage, half * sizeof(float2), "volume FT upload"));
    cudaError_t e = cudaMemcpyAsync(stage, cmat_half, half * sizeof(float2), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = launch_expand_cmat(h, box, stage, factor, h->vol_cube);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    dev_free(h, stage);
    if (e != cudaSuccess) return cuda_err(h, e, "set_volume_ft");
    h->vol_box = box;
    return PFTCC_OK;
}

int pftcc_fproject_polar(pftcc_handle *h, int first_iref, int n, const float *euls, const int *mask, int iseven,
                         int griddev)
{
    if (!h || !euls || n < 0) return set_err(h, PFTCC_ERR_ARG, "fproject_polar: bad arguments");
    if (first_iref < 1 || first_iref + n - 1 > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "fproject_polar: range");
    if (!h->vol_cube) return set_err(h, PFTCC_ERR_STATE, "fproject_polar: no volume (set_volume_ft first)");
    if (n == 0) return PFTCC_OK;
    std::vector<double> R((size_t)n * 9);
    for (int r = 0; r < n; ++r) {
        const double e[3] = {(double)euls[3 * r], (double)euls[3 * r + 1], (double)euls[3 * r + 2]};
        if (!std::isfinite(e[0]) || !std::isfinite(e[1]) || !std::isfinite(e[2]))
            return set_err(h, PFTCC_ERR_ARG, "fproject_polar: Euler angle not finite");
        host_euler2m(e, &R[(size_t)r * 9], nullptr);
    }
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    double *dR = nullptr;
    int *dmask = nullptr;
    ST(dev_alloc(h, (void **)&dR, R.size() * sizeof(double), "rotation matrices"));
    if (mask) {
        int st = dev_alloc(h, (void **)&dmask, (size_t)h->g.K * sizeof(int), "projection shell mask");
        if (st) { dev_free(h, dR); return st; }
    }
    const size_t KP = (size_t)h->g.K * h->g.P;
    float2 *dst = (iseven ? h->refs_even : h->refs_odd) + (size_t)(first_iref - 1) * KP;
    cudaError_t e = cudaMemcpyAsync(dR, R.data(), R.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && mask)
        e = cudaMemcpyAsync(dmask, mask, (size_t)h->g.K * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = launch_fproject_polar(h, h->vol_box, h->vol_cube, dR, dmask, n, griddev ? 1 : 0, dst);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    dev_free(h, dR);
    dev_free(h, dmask);
    if (e != cudaSuccess) return cuda_err(h, e, "fproject_polar");
    return PFTCC_OK;
}

static int ensure_drefs(pftcc_handle *h)
{
    if (h->drefs_even && h->drefs_odd) return PFTCC_OK;
    const size_t bytes = (size_t)h->nrefs * 3 * h->g.K * h->g.P * sizeof(float2);
    ST(dev_alloc(h, (void **)&h->drefs_even, bytes, "derivative references (even)"));
    ST(dev_alloc(h, (void **)&h->drefs_odd, bytes, "derivative references (odd)"));
    CK(cudaMemsetAsync(h->drefs_even, 0, bytes, h->stream), "zero drefs");
    CK(cudaMemsetAsync(h->drefs_odd, 0, bytes, h->stream), "zero drefs");
    return PFTCC_OK;
}

int pftcc_fdf_project_polar(pftcc_handle *h, int first_iref, int n, const double *euls, int iseven)
{
    if (!h || !euls || n < 0) return set_err(h, PFTCC_ERR_ARG, "fdf_project_polar: bad arguments");
    if (first_iref < 1 || first_iref + n - 1 > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "fdf_project_polar: range");
    if (!h->vol_cube) return set_err(h, PFTCC_ERR_STATE, "fdf_project_polar: no volume (set_volume_ft first)");
    if (n == 0) return PFTCC_OK;
    std::vector<double> RD((size_t)n * 36);
    for (int r = 0; r < n; ++r) {
        const double *e = euls + 3 * r;
        if (!std::isfinite(e[0]) || !std::isfinite(e[1]) || !std::isfinite(e[2]))
            return set_err(h, PFTCC_ERR_ARG, "fdf_project_polar: Euler angle not finite");
        host_euler2m(e, &RD[(size_t)r * 36], &RD[(size_t)r * 36 + 9]);
    }
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(ensure_drefs(h));
    double *dRD = nullptr;
    ST(dev_alloc(h, (void **)&dRD, RD.size() * sizeof(double), "rotation matrices and derivatives"));
    const size_t KP = (size_t)h->g.K * h->g.P;
    float2 *dst = (iseven ? h->refs_even : h->refs_odd) + (size_t)(first_iref - 1) * KP;
    float2 *ddst = (iseven ? h->drefs_even : h->drefs_odd) + (size_t)(first_iref - 1) * 3 * KP;
    cudaError_t e = cudaMemcpyAsync(dRD, RD.data(), RD.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = launch_fdf_project_polar(h, h->vol_box, h->vol_cube, dRD, n, dst, ddst);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    dev_free(h, dRD);
    if (e != cudaSuccess) return cuda_err(h, e, "fdf_project_polar");
    return PFTCC_OK;
}

int pftcc_get_dref_pft(pftcc_handle *h, int iref, int iseven, float *dpft)
{
    if (!h || !dpft) return PFTCC_ERR_ARG;
    REF_OR_FAIL(iref);
    if (!h->drefs_even) return set_err(h, PFTCC_ERR_STATE, "no derivative references (fdf_project_polar first)");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    const size_t n3 = (size_t)3 * h->g.K * h->g.P;
    const float2 *src = (iseven ? h->drefs_even : h->drefs_odd) + (size_t)(iref - 1) * n3;
    CK(cudaMemcpyAsync(dpft, src, n3 * sizeof(float2), cudaMemcpyDeviceToHost, h->stream), "get_dref_pft");
    CK(cudaStreamSynchronize(h->stream), "get_dref_pft");
    return PFTCC_OK;
}

int pftcc_cont_shift_grad_batch(pftcc_handle *h, int n, const pftcc_grad_req *req, double *f, double *grad5)
{
    if (!h || n < 0 || (n > 0 && (!req || !f || !grad5)))
        return set_err(h, PFTCC_ERR_ARG, "cont_shift_grad: bad arguments");
    if (n == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    if (h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "the orientation gradient is served in the reference frame");
    if (h->cfg.with_ctf && !h->ctf_ready)
        return set_err(h, PFTCC_ERR_STATE, "CTF is on but create_polar_absctfmats has not been called");
    if (!h->drefs_even) return set_err(h, PFTCC_ERR_STATE, "no derivative references (fdf_project_polar first)");
    ST(snorm_ready(h, 0, h->nrefs));
    std::vector<EuclidReq> rq(n);
    for (int i = 0; i < n; ++i) {
        if (req[i].iref < 1 || req[i].iref > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "cont_shift_grad: iref out of range");
        if (req[i].irot < 1 || req[i].irot > h->g.N) return set_err(h, PFTCC_ERR_INDEX, "cont_shift_grad: irot out of range");
        const int sl = slot_of(h, req[i].iptcl);
        if (sl < 0) return set_err(h, PFTCC_ERR_INDEX, "cont_shift_grad: particle not held");
        rq[i] = EuclidReq{req[i].iref - 1, sl, req[i].irot, 0, req[i].sx, req[i].sy};
    }
    ST(ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>((size_t)n * sizeof(EuclidReq), 4096), "requests"));
    ST(ensure(h, (void **)&h->d_dout, &h->dout_cap, (size_t)n * 6 * sizeof(double), "results"));
    CK(cudaMemcpyAsync(h->d_work, rq.data(), (size_t)n * sizeof(EuclidReq), cudaMemcpyHostToDevice, h->stream), "requests");
    CK(launch_cont_shift_grad(h, reinterpret_cast<const EuclidReq *>(h->d_work), n, h->d_dout), "cont_shift_grad kernel");
    std::vector<double> o((size_t)n * 6);
    CK(cudaMemcpyAsync(o.data(), h->d_dout, o.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "results");
    CK(cudaStreamSynchronize(h->stream), "cont_shift_grad");
    for (int i = 0; i < n; ++i) {
        f[i] = o[6 * (size_t)i];
        for (int d = 0; d < 5; ++d) grad5[5 * (size_t)i + d] = o[6 * (size_t)i + 1 + d];
    }
    return PFTCC_OK;
}

int pftcc_gencorr_cont_shift_grad_cc_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                               double *f, double *grad)
{
    if (!h || !shvec || !f || !grad) return set_err(h, PFTCC_ERR_ARG, "cont_shift_grad: bad arguments");
    pftcc_grad_req r{iref, iptcl, irot, 0, shvec[0], shvec[1], 0.0};
    return pftcc_cont_shift_grad_batch(h, 1, &r, f, grad);
}

int pftcc_orisrch_batch(pftcc_handle *h, int n, const pftcc_orisrch_req *req, int maxits, double pgtol, double factr,
                        pftcc_orisrch_out *out)
{
    if (!h || n < 0 || (n > 0 && (!req || !out)) || maxits < 1 || !(pgtol >= 0) || !(factr >= 0))
        return set_err(h, PFTCC_ERR_ARG, "orisrch_batch: bad arguments");
    for (int i = 0; i < n; ++i) {
        bool ok = std::isfinite(req[i].angerr_deg) && req[i].angerr_deg >= 0 && std::isfinite(req[i].maxhwshift) &&
                  req[i].maxhwshift >= 0;
        for (int v = 0; v < 3; ++v) ok = ok && std::isfinite(req[i].e[v]);
        if (!ok) return set_err(h, PFTCC_ERR_ARG, "orisrch_batch: angles and bounds must be finite and non-negative");
    }
    if (n == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    if (h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "the orientation gradient is served in the reference frame");
    if (!h->vol_cube) return set_err(h, PFTCC_ERR_STATE, "orisrch_batch: no volume (set_volume_ft first)");
    if (h->cfg.with_ctf && !h->ctf_ready)
        return set_err(h, PFTCC_ERR_STATE, "CTF is on but create_polar_absctfmats has not been called");
    return orisrch_batch(h, n, req, maxits, pgtol, factr, out);
}

int pftcc_gencorr_cont_grad_cc_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                         double *cc, double *dcc)
{
    if (!h || !shvec || !cc || !dcc) return set_err(h, PFTCC_ERR_ARG, "cont_grad: bad arguments");
    double g5[5];
    ST(pftcc_gencorr_cont_shift_grad_cc_for_rot_8(h, iref, iptcl, shvec, irot, cc, g5));
    for (int d = 0; d < 3; ++d) dcc[d] = g5[d];
    return PFTCC_OK;
}

int pftcc_polarize_refs(pftcc_handle *h, int first_iref, int n, const float *cmats, int iseven, int griddev)
{
    // polarize into the particle slots' layout through a temporary handle-less path:
    // the gridding is identical, only the destination differs (polarize :144-148)
    if (!h || !cmats || n < 0) return set_err(h, PFTCC_ERR_ARG, "polarize_refs: bad arguments");
    if (first_iref < 1 || first_iref + n - 1 > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "polarize_refs: range");
    cudaSetDevice(h->dev);
    ST(build_polarizer(h, griddev));
    const size_t img = (size_t)h->g.box * (h->g.box / 2 + 1) * sizeof(float2);
    const size_t KP = (size_t)h->g.K * h->g.P;
    ST(ensure(h, &h->pol_stage, &h->pol_stage_bytes, std::max<size_t>((size_t)n * img, 1), "polarize staging"));
    CK(cudaMemcpyAsync(h->pol_stage, cmats, (size_t)n * img, cudaMemcpyHostToDevice, h->stream), "upload");
    // reuse the particle kernel with a redirected destination
    float2 *save_p = h->ptcls;
    float *save_s = h->sqsums;
    h->ptcls = (iseven ? h->refs_even : h->refs_odd) + (size_t)(first_iref - 1) * KP;
    float *dummy = nullptr;
    ST(dev_alloc(h, (void **)&dummy, (size_t)n * sizeof(float), "ref sqsums"));
    h->sqsums = dummy;
    cudaError_t e = launch_polarize(h, (const float2 *)h->pol_stage, n, 0);
    h->ptcls = save_p;
    h->sqsums = save_s;
    cudaError_t e2 = cudaStreamSynchronize(h->stream);
    dev_free(h, dummy);
    CK(e, "polarize refs");
    CK(e2, "polarize refs");
    return PFTCC_OK;
}

int pftcc_memoize_ffts(pftcc_handle *h)
{
    // the exact path reads the particle pfts directly; the m-domain search prepares its
    // particle spectra lazily (they depend on the CTF matrices), so only invalidate here
    if (!h) return PFTCC_ERR_ARG;
    h->ws.ptcl_spectra_valid = 0;
    return PFTCC_OK;
}

// ---- correlators -----------------------------------------------------------------------------
static int ensure_small(pftcc_handle *h, size_t nwork, size_t ngroups, size_t nout, size_t nshifts)
{
    ST(ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>(nwork * sizeof(Work), 4096), "work"));
    ST(ensure(h, (void **)&h->d_groups, &h->group_cap, std::max<size_t>(ngroups * sizeof(Group), 256), "groups"));
    ST(ensure(h, (void **)&h->d_out, &h->out_cap, std::max<size_t>(nout * sizeof(float), 256), "out"));
    ST(ensure(h, (void **)&h->d_shifts, &h->shifts_cap, std::max<size_t>(nshifts * 2 * sizeof(float), 64), "shifts"));
    ST(ensure(h, (void **)&h->d_dout, &h->dout_cap, 4096, "dout"));
    return PFTCC_OK;
}

static int check_ctf_only(pftcc_handle *h)
{
    if (h->cfg.with_ctf && !h->ctf_ready)
        return set_err(h, PFTCC_ERR_STATE, "CTF is on but create_polar_absctfmats has not been called");
    return PFTCC_OK;
}

// the state an evaluation of the current objective needs (and, in the matched-filter mode, the
// references' current shell factors)
static int check_ctf_state(pftcc_handle *h)
{
    ST(check_ctf_only(h));
    ST(snorm_ready(h, 0, h->nrefs));
    if (h->objfun == PFTCC_OBJFUN_EUCLID) return euclid_ready(h, 1);
    return PFTCC_OK;
}

static int gencorrs_frame(pftcc_handle *h, int iref, int iptcl, const float *shvec, float *cc, int frame)
{
    REF_OR_FAIL(iref);
    SLOT_OR_FAIL(slot, iptcl);
    ST(ensure_small(h, 1, 1, h->g.N, 1));
    Work w{iref - 1, shvec ? 0 : -1, 0};
    Group gr{slot, 0, 1, 0};
    CK(cudaMemcpyAsync(h->d_work, &w, sizeof(w), cudaMemcpyHostToDevice, h->stream), "gencorrs");
    CK(cudaMemcpyAsync(h->d_groups, &gr, sizeof(gr), cudaMemcpyHostToDevice, h->stream), "gencorrs");
    if (shvec) CK(cudaMemcpyAsync(h->d_shifts, shvec, 2 * sizeof(float), cudaMemcpyHostToDevice, h->stream), "gencorrs");
    CK(launch_exact(h, h->d_groups, 1, h->d_work, h->d_shifts, MODE_FULL, frame, 1, h->d_out, nullptr),
       "gencorrs kernel");
    CK(cudaMemcpyAsync(cc, h->d_out, h->g.N * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "gencorrs");
    CK(cudaStreamSynchronize(h->stream), "gencorrs");
    return PFTCC_OK;
}

int pftcc_gencorrs(pftcc_handle *h, int iref, int iptcl, const float *shvec, float *cc)
{
    if (!h || !cc) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    ST(exact_objfun_ok(h));
    return gencorrs_frame(h, iref, iptcl, shvec, cc, exact_frame(h));
}

static int euclid_explicit_state(pftcc_handle *h)
{
    if (h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "the Euclidean objective is defined in the reference frame");
    ST(check_ctf_only(h));
    return euclid_ready(h, 1);
}

int pftcc_gencorrs_euclid(pftcc_handle *h, int iref, int iptcl, const float *shvec, float *euclids)
{
    if (!h || !euclids) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(euclid_explicit_state(h));
    return gencorrs_frame(h, iref, iptcl, shvec, euclids, FRAME_EUCLID);
}

// n single-rotation Euclidean requests: out3 [n][3] (with_f), shells [n][3][K] (want_shells)
static int euclid_rot_host(pftcc_handle *h, int n, const EuclidReq *rq, int with_f, int want_shells, double *out3,
                           double *shells)
{
    const int K = h->g.K;
    ST(ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>((size_t)n * sizeof(EuclidReq), 4096),
              "euclid requests"));
    const size_t per = (with_f ? 3 : 0) + (want_shells ? 3 * (size_t)K : 0);
    ST(ensure(h, (void **)&h->d_dout, &h->dout_cap, (size_t)n * per * sizeof(double), "euclid results"));
    double *o3 = with_f ? h->d_dout : nullptr;
    double *sh = want_shells ? h->d_dout + (with_f ? 3 * (size_t)n : 0) : nullptr;
    CK(cudaMemcpyAsync(h->d_work, rq, (size_t)n * sizeof(EuclidReq), cudaMemcpyHostToDevice, h->stream), "euclid");
    CK(launch_euclid_rot(h, reinterpret_cast<const EuclidReq *>(h->d_work), n, with_f, want_shells, o3, sh),
       "euclid kernel");
    if (with_f) CK(cudaMemcpyAsync(out3, o3, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "euclid");
    if (want_shells)
        CK(cudaMemcpyAsync(shells, sh, 3 * (size_t)n * K * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "euclid");
    CK(cudaStreamSynchronize(h->stream), "euclid");
    return PFTCC_OK;
}

// one rotation of the Euclidean objective: f3 = f, df/dsx, df/dsy (caller holds the lock and
// has checked the state)
static int euclid_single(pftcc_handle *h, int iref, int iptcl, double sx, double sy, int irot, double *f3)
{
    REF_OR_FAIL(iref);
    SLOT_OR_FAIL(slot, iptcl);
    if (irot < 1 || irot > h->g.N) return set_err(h, PFTCC_ERR_INDEX, "irot out of range");
    const EuclidReq rq{iref - 1, slot, irot, 0, sx, sy};
    return euclid_rot_host(h, 1, &rq, 1, 0, f3, nullptr);
}

int pftcc_gencorr_euclid_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot, double *f)
{
    if (!h || !f || !shvec) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(euclid_explicit_state(h));
    double o[3];
    ST(euclid_single(h, iref, iptcl, shvec[0], shvec[1], irot, o));
    *f = o[0];
    return PFTCC_OK;
}

int pftcc_gencorr_euclid_for_rot(pftcc_handle *h, int iref, int iptcl, const float *shvec, int irot, float *f)
{
    if (!h || !f || !shvec) return PFTCC_ERR_ARG;
    const double sh[2] = {(double)shvec[0], (double)shvec[1]};
    double v;
    ST(pftcc_gencorr_euclid_for_rot_8(h, iref, iptcl, sh, irot, &v));
    *f = (float)v;
    return PFTCC_OK;
}

int pftcc_gencorr_euclid_grad_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                        double *f, double *grad)
{
    if (!h || !f || !grad || !shvec) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(euclid_explicit_state(h));
    double o[3];
    ST(euclid_single(h, iref, iptcl, shvec[0], shvec[1], irot, o));
    *f = o[0];
    grad[0] = o[1];
    grad[1] = o[2];
    return PFTCC_OK;
}

int pftcc_gencorr_euclid_grad_only_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                             double *grad)
{
    double f;
    return pftcc_gencorr_euclid_grad_for_rot_8(h, iref, iptcl, shvec, irot, &f, grad);
}

int pftcc_sigma_contrib_batch(pftcc_handle *h, int n, const int *iref, const int *iptcl, const int *irot,
                              const float *shifts, float *sigma_contrib, float *ptcl_sumsq, float *ref_sumsq)
{
    if (!h || n < 0 || (n > 0 && (!iref || !iptcl || !irot || !shifts || !sigma_contrib)))
        return set_err(h, PFTCC_ERR_ARG, "sigma_contrib: bad arguments");
    if (n == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    if (h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "sigma_contrib is defined in the reference frame");
    ST(check_ctf_only(h));
    std::vector<EuclidReq> rq(n);
    for (int i = 0; i < n; ++i) {
        if (iref[i] < 1 || iref[i] > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "sigma_contrib: iref out of range");
        if (irot[i] < 1 || irot[i] > h->g.N) return set_err(h, PFTCC_ERR_INDEX, "sigma_contrib: irot out of range");
        const int sl = slot_of(h, iptcl[i]);
        if (sl < 0) return set_err(h, PFTCC_ERR_INDEX, "sigma_contrib: particle not held");
        rq[i] = EuclidReq{iref[i] - 1, sl, irot[i], 0, (double)shifts[2 * i], (double)shifts[2 * i + 1]};
    }
    const int K = h->g.K;
    std::vector<double> sh((size_t)n * 3 * K);
    ST(euclid_rot_host(h, n, rq.data(), 0, 1, nullptr, sh.data()));
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < K; ++k) {
            const double *b = &sh[(size_t)i * 3 * K];
            sigma_contrib[(size_t)i * K + k] = (float)b[k];
            if (ptcl_sumsq) ptcl_sumsq[(size_t)i * K + k] = (float)b[K + k];
            if (ref_sumsq) ref_sumsq[(size_t)i * K + k] = (float)b[2 * K + k];
        }
    return PFTCC_OK;
}

int pftcc_gencorr_sigma_contrib(pftcc_handle *h, int iref, int iptcl, const float *shvec, int irot,
                                float *sigma_contrib, float *ptcl_sumsq, float *ref_sumsq)
{
    if (!h || !shvec || !sigma_contrib) return set_err(h, PFTCC_ERR_ARG, "sigma_contrib: bad arguments");
    return pftcc_sigma_contrib_batch(h, 1, &iref, &iptcl, &irot, shvec, sigma_contrib, ptcl_sumsq, ref_sumsq);
}

static int for_rot_common(pftcc_handle *h, int iref, int iptcl, double sx, double sy, int irot, double *out5)
{
    REF_OR_FAIL(iref);
    SLOT_OR_FAIL(slot, iptcl);
    if (irot < 1 || irot > h->g.N) return set_err(h, PFTCC_ERR_INDEX, "irot out of range");
    if (h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "single-rotation correlations are served in the reference frame");
    ST(check_ctf_state(h));
    if (h->objfun == PFTCC_OBJFUN_EUCLID) {   // gencorr_for_rot_8 / gencorr_grad_for_rot_8 dispatch (:1632-1643, :1849-1861)
        out5[3] = out5[4] = 0.0;
        return euclid_single(h, iref, iptcl, sx, sy, irot, out5);
    }
    ST(ensure_small(h, 1, 1, h->g.N, 1));
    CK(launch_for_rot(h, iref - 1, slot, sx, sy, irot, h->cfg.match_filt, 1, 0.0, h->d_dout), "for_rot kernel");
    CK(cudaMemcpyAsync(out5, h->d_dout, 5 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "for_rot");
    CK(cudaStreamSynchronize(h->stream), "for_rot");
    return PFTCC_OK;
}

int pftcc_gencorr_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot, double *cc)
{
    if (!h || !cc || !shvec) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    double o[5];
    ST(for_rot_common(h, iref, iptcl, shvec[0], shvec[1], irot, o));
    *cc = o[0];
    return PFTCC_OK;
}

int pftcc_gencorr_for_rot(pftcc_handle *h, int iref, int iptcl, const float *shvec, int irot, float *cc)
{
    if (!h || !cc || !shvec) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    double o[5];
    ST(for_rot_common(h, iref, iptcl, (double)shvec[0], (double)shvec[1], irot, o));
    *cc = (float)o[0];
    return PFTCC_OK;
}

int pftcc_gencorr_grad_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot, double *f,
                                 double *grad)
{
    if (!h || !f || !grad || !shvec) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    double o[5];
    ST(for_rot_common(h, iref, iptcl, shvec[0], shvec[1], irot, o));
    *f = o[0];
    grad[0] = o[1];
    grad[1] = o[2];
    return PFTCC_OK;
}

int pftcc_gencorr_grad_only_for_rot_8(pftcc_handle *h, int iref, int iptcl, const double *shvec, int irot,
                                      double *grad)
{
    double f;
    return pftcc_gencorr_grad_for_rot_8(h, iref, iptcl, shvec, irot, &f, grad);
}

int pftcc_specscore_batch(pftcc_handle *h, int n, const int *iref, const int *iptcl, const int *irot,
                          const float *shifts, float *scores, float *frcs)
{
    if (!h || n < 0 || (n > 0 && (!iref || !iptcl || !irot || !scores)))
        return set_err(h, PFTCC_ERR_ARG, "specscore: bad arguments");
    if (n == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    std::vector<FrcReq> rq(n);
    for (int i = 0; i < n; ++i) {
        if (iref[i] < 1 || iref[i] > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "specscore: iref out of range");
        if (irot[i] < 1 || irot[i] > h->g.N) return set_err(h, PFTCC_ERR_INDEX, "specscore: irot out of range");
        const int sl = slot_of(h, iptcl[i]);
        if (sl < 0) return set_err(h, PFTCC_ERR_INDEX, "specscore: particle not held");
        rq[i] = FrcReq{iref[i] - 1, sl, irot[i], shifts ? 1 : 0, shifts ? (double)shifts[2 * i] : 0.0,
                       shifts ? (double)shifts[2 * i + 1] : 0.0};
    }
    const int Ks = h->g.Ks;
    const size_t rq_bytes = (size_t)n * sizeof(FrcReq), out_floats = (size_t)n * (1 + Ks);
    ST(ensure(h, (void **)&h->d_dout, &h->dout_cap, rq_bytes + out_floats * sizeof(float) + 256, "specscore"));
    char *base = (char *)h->d_dout;
    FrcReq *drq = (FrcReq *)base;
    float *dscore = (float *)(base + rq_bytes);
    float *dfrc = dscore + n;
    CK(cudaMemcpyAsync(drq, rq.data(), rq_bytes, cudaMemcpyHostToDevice, h->stream), "specscore upload");
    CK(launch_specscore(h, drq, n, frcs ? dfrc : nullptr, dscore), "specscore kernel");
    CK(cudaMemcpyAsync(scores, dscore, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "specscore");
    if (frcs)
        CK(cudaMemcpyAsync(frcs, dfrc, (size_t)n * Ks * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "genfrc");
    CK(cudaStreamSynchronize(h->stream), "specscore");
    return PFTCC_OK;
}

int pftcc_specscore(pftcc_handle *h, int iref, int iptcl, int irot, const float *shvec, float *score)
{
    if (!h || !score) return set_err(h, PFTCC_ERR_ARG, "specscore: bad arguments");
    return pftcc_specscore_batch(h, 1, &iref, &iptcl, &irot, shvec, score, nullptr);
}

int pftcc_genfrc(pftcc_handle *h, int iref, int iptcl, int irot, const float *shvec, float *frc)
{
    if (!h || !frc) return set_err(h, PFTCC_ERR_ARG, "genfrc: bad arguments");
    float score;
    return pftcc_specscore_batch(h, 1, &iref, &iptcl, &irot, shvec, &score, frc);
}

int pftcc_cp_refs(pftcc_handle *h, const pftcc_handle *src)
{
    if (!h || !src) return set_err(h, PFTCC_ERR_ARG, "cp_refs: bad arguments");
    if (src->nrefs != h->nrefs || src->g.K != h->g.K || src->g.P != h->g.P)
        return set_err(h, PFTCC_ERR_ARG, "cp_refs: the two objects' reference sets differ in shape");
    if (src->dev != h->dev) return set_err(h, PFTCC_ERR_ARG, "cp_refs: the two objects live on different devices");
    // both objects locked (std::scoped_lock orders the two locks, so two threads copying in
    // opposite directions cannot deadlock); src's references cannot change under the copy
    std::mutex &src_mtx = const_cast<pftcc_handle *>(src)->mtx;
    std::unique_lock<std::mutex> lk1, lk2;
    if (src == h) {
        lk1 = std::unique_lock<std::mutex>(h->mtx);
    } else {
        std::lock(h->mtx, src_mtx);
        lk1 = std::unique_lock<std::mutex>(h->mtx, std::adopt_lock);
        lk2 = std::unique_lock<std::mutex>(src_mtx, std::adopt_lock);
    }
    cudaSetDevice(h->dev);
    const size_t bytes = (size_t)h->nrefs * h->g.K * h->g.P * sizeof(float2);
    // self%pfts_refs_odd = self2%pfts_refs_odd; self%pfts_refs_even = self2%pfts_refs_even (:491-495)
    CK(cudaStreamSynchronize(src->stream), "cp_refs");
    CK(cudaMemcpyAsync(h->refs_odd, src->refs_odd, bytes, cudaMemcpyDeviceToDevice, h->stream), "cp_refs");
    CK(cudaMemcpyAsync(h->refs_even, src->refs_even, bytes, cudaMemcpyDeviceToDevice, h->stream), "cp_refs");
    CK(cudaStreamSynchronize(h->stream), "cp_refs");
    return PFTCC_OK;
}

int pftcc_set_ptcl_fcomp(pftcc_handle *h, int iptcl, int irot, int k, const float *comp)
{
    if (!h || !comp) return set_err(h, PFTCC_ERR_ARG, "set_ptcl_fcomp: bad arguments");
    SLOT_OR_FAIL(slot, iptcl);
    if (irot < 1 || irot > h->g.P || k < h->g.kfrom || k > h->g.kto)
        return set_err(h, PFTCC_ERR_INDEX, "set_ptcl_fcomp: irot or k out of range");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    // pfts_ptcls(irot, k, pinds(iptcl)) = comp (:471-476); the square sum is left as it is, as there
    float2 *dst = h->ptcls + ((size_t)slot * h->g.K + (k - h->g.kfrom)) * h->g.P + (irot - 1);
    CK(cudaMemcpyAsync(dst, comp, sizeof(float2), cudaMemcpyHostToDevice, h->stream), "set_ptcl_fcomp");
    CK(cudaStreamSynchronize(h->stream), "set_ptcl_fcomp");
    h->ws.ptcl_spectra_valid = 0;
    return PFTCC_OK;
}

int pftcc_calc_ptcl_pspec(pftcc_handle *h, int iptcl, float *pspec)
{
    if (!h || !pspec) return set_err(h, PFTCC_ERR_ARG, "calc_ptcl_pspec: bad arguments");
    SLOT_OR_FAIL(slot, iptcl);
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(ensure(h, (void **)&h->d_out, &h->out_cap, std::max<size_t>((size_t)h->g.K * sizeof(float), 256), "pspec"));
    CK(launch_ptcl_pspec(h, slot, h->d_out), "calc_ptcl_pspec kernel");
    CK(cudaMemcpyAsync(pspec, h->d_out, h->g.K * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "calc_ptcl_pspec");
    CK(cudaStreamSynchronize(h->stream), "calc_ptcl_pspec");
    return PFTCC_OK;
}

int pftcc_assign_pinds(const pftcc_handle *h, int *pinds)
{
    if (!h || !pinds) return PFTCC_ERR_ARG;
    // self%pinds(pfromto(1):pfromto(2)): each index's particle slot, 1-based, 0 where not held
    for (size_t i = 0; i < h->pinds.size(); ++i) pinds[i] = h->pinds[i];
    return PFTCC_OK;
}

int pftcc_calc_roinv_corrmat(pftcc_handle *h, float *corrmat)
{
    if (!h || !corrmat) return set_err(h, PFTCC_ERR_ARG, "calc_roinv_corrmat: bad arguments");
    if (h->nptcls != h->nrefs)
        return set_err(h, PFTCC_ERR_ARG, "nptcls == nrefs in pftcc required; calc_roinv_corrmat");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    ST(exact_objfun_ok(h));
    const int n = h->nptcls;
    // particle iptcl = pfrom + g (g = 0..n-1) is correlated with references 1..g (iref < iptcl),
    // the best rotation's value kept and the matrix symmetrised with 1 on the diagonal (:2207-2231)
    std::vector<int> slot_of_g(n, -1);
    for (int gq = 0; gq < n; ++gq) {
        const int gi = h->pfrom + gq;
        slot_of_g[gq] = gi <= h->pto ? h->pinds[gi - h->pfrom] - 1 : -1;
        if (slot_of_g[gq] < 0)
            return set_err(h, PFTCC_ERR_INDEX, "calc_roinv_corrmat: particles pfrom..pfrom+nptcls-1 must be held");
    }
    const size_t npairs = (size_t)n * (n - 1) / 2;
    std::vector<float> mat((size_t)n * n, 1.f);
    if (npairs > 0) {
        ST(ensure_small(h, npairs, n, npairs, 1));
        std::vector<Work> work(npairs);
        std::vector<Group> groups;
        size_t wi = 0;
        for (int ip = 1; ip < n; ++ip) {
            groups.push_back(Group{slot_of_g[ip], (int)wi, ip, (int)groups.size()});
            for (int ir = 0; ir < ip; ++ir, ++wi) work[wi] = Work{ir, -1, (long long)wi};
        }
        CK(cudaMemcpyAsync(h->d_work, work.data(), wi * sizeof(Work), cudaMemcpyHostToDevice, h->stream), "corrmat");
        CK(cudaMemcpyAsync(h->d_groups, groups.data(), groups.size() * sizeof(Group), cudaMemcpyHostToDevice, h->stream),
           "corrmat");
        CK(launch_exact(h, h->d_groups, (int)groups.size(), h->d_work, nullptr, MODE_ITEMMAX, exact_frame(h), 1,
                        h->d_out, nullptr), "corrmat kernel");
        std::vector<float> mx(npairs);
        CK(cudaMemcpyAsync(mx.data(), h->d_out, npairs * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "corrmat");
        CK(cudaStreamSynchronize(h->stream), "corrmat");
        wi = 0;
        for (int ip = 1; ip < n; ++ip)
            for (int ir = 0; ir < ip; ++ir, ++wi) {
                mat[(size_t)ir * n + ip] = mx[wi];
                mat[(size_t)ip * n + ir] = mx[wi];
            }
    }
    std::copy(mat.begin(), mat.end(), corrmat);
    return PFTCC_OK;
}

int pftcc_corr_all(pftcc_handle *h, int nshifts, const float *shifts, float *cc)
{
    if (!h || !cc || nshifts < 0 || (nshifts > 0 && !shifts)) return set_err(h, PFTCC_ERR_ARG, "corr_all: bad arguments");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    ST(exact_objfun_ok(h));
    const int ns = std::max(1, nshifts);
    const size_t per_ptcl = (size_t)h->nrefs * ns;
    // bounded output chunks of particles
    const size_t out_per_ptcl = per_ptcl * h->g.N;
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(h->nptcls, (size_t)(512u << 20) / (out_per_ptcl * 4)));
    ST(ensure_small(h, (size_t)chunk * per_ptcl, chunk, (size_t)chunk * out_per_ptcl, ns));
    if (nshifts > 0)
        CK(cudaMemcpyAsync(h->d_shifts, shifts, 2 * sizeof(float) * nshifts, cudaMemcpyHostToDevice, h->stream), "shifts");
    std::vector<Work> work((size_t)chunk * per_ptcl);
    std::vector<Group> groups(chunk);
    for (int c0 = 0; c0 < h->nptcls; c0 += chunk) {
        const int m = std::min(chunk, h->nptcls - c0);
        size_t wi = 0;
        for (int i = 0; i < m; ++i) {
            groups[i] = Group{c0 + i, (int)wi, (int)per_ptcl, i};
            for (int r = 0; r < h->nrefs; ++r)
                for (int s = 0; s < ns; ++s) {
                    work[wi] = Work{r, nshifts > 0 ? s : -1, (long long)(((size_t)i * h->nrefs + r) * ns + s) * h->g.N};
                    ++wi;
                }
        }
        CK(cudaMemcpyAsync(h->d_work, work.data(), wi * sizeof(Work), cudaMemcpyHostToDevice, h->stream), "work");
        CK(cudaMemcpyAsync(h->d_groups, groups.data(), m * sizeof(Group), cudaMemcpyHostToDevice, h->stream), "groups");
        CK(launch_exact(h, h->d_groups, m, h->d_work, h->d_shifts, MODE_FULL, exact_frame(h), 1, h->d_out, nullptr),
           "corr_all kernel");
        CK(cudaMemcpyAsync(cc + (size_t)c0 * out_per_ptcl, h->d_out, (size_t)m * out_per_ptcl * sizeof(float),
                           cudaMemcpyDeviceToHost, h->stream), "corr_all download");
        CK(cudaStreamSynchronize(h->stream), "corr_all");
    }
    return PFTCC_OK;
}

int pftcc_corr_all_prec(pftcc_handle *h, int nshifts, const float *shifts, int precision, float *cc)
{
    if (!h || !cc || nshifts < 0 || (nshifts > 0 && !shifts)) return set_err(h, PFTCC_ERR_ARG, "corr_all_prec: bad arguments");
    if (precision == PFTCC_PREC_EXACT) return pftcc_corr_all(h, nshifts, shifts, cc);
    if (precision != PFTCC_PREC_FP32 && precision != PFTCC_PREC_BF16X3)
        return set_err(h, PFTCC_ERR_ARG, "corr_all_prec: unknown precision");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    const size_t n = (size_t)h->nptcls * h->nrefs * std::max(1, nshifts) * h->g.N;
    ST(ensure(h, (void **)&h->d_out, &h->out_cap, n * sizeof(float), "corr_all_prec out"));
    ST(search_mdomain(h, nshifts, shifts, precision, 0, nullptr, h->d_out));
    CK(cudaMemcpyAsync(cc, h->d_out, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream), "corr_all_prec download");
    CK(cudaStreamSynchronize(h->stream), "corr_all_prec");
    return PFTCC_OK;
}

static int search_exact(pftcc_handle *h, int nshifts, const float *shifts, pftcc_best *out_dev)
{
    ST(exact_objfun_ok(h));
    const int ns = std::max(1, nshifts);
    const size_t per_ptcl = (size_t)h->nrefs * ns;
    ST(ensure_small(h, (size_t)h->nptcls * per_ptcl, h->nptcls, 1, ns));
    if (nshifts > 0)
        CK(cudaMemcpyAsync(h->d_shifts, shifts, 2 * sizeof(float) * nshifts, cudaMemcpyHostToDevice, h->stream), "shifts");
    std::vector<Work> work((size_t)h->nptcls * per_ptcl);
    std::vector<Group> groups(h->nptcls);
    size_t wi = 0;
    for (int i = 0; i < h->nptcls; ++i) {
        groups[i] = Group{i, (int)wi, (int)per_ptcl, i};
        for (int r = 0; r < h->nrefs; ++r)
            for (int s = 0; s < ns; ++s) work[wi++] = Work{r, nshifts > 0 ? s : -1, 0};
    }
    CK(cudaMemcpyAsync(h->d_work, work.data(), wi * sizeof(Work), cudaMemcpyHostToDevice, h->stream), "work");
    CK(cudaMemcpyAsync(h->d_groups, groups.data(), groups.size() * sizeof(Group), cudaMemcpyHostToDevice, h->stream),
       "groups");
    CK(launch_exact(h, h->d_groups, h->nptcls, h->d_work, h->d_shifts, MODE_BEST, exact_frame(h), 1, nullptr, out_dev),
       "search exact");
    return PFTCC_OK;
}

int pftcc_search_best_dev(pftcc_handle *h, int nshifts, const float *shifts, int precision, int ntop, void *out_dev)
{
    if (!h || !out_dev || nshifts < 0 || (nshifts > 0 && !shifts) || ntop < 0 || ntop > 8)
        return set_err(h, PFTCC_ERR_ARG, "search_best: bad arguments");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    if (precision == PFTCC_PREC_EXACT) {
        ST(search_exact(h, nshifts, shifts, (pftcc_best *)out_dev));
    } else if (precision == PFTCC_PREC_FP32 || precision == PFTCC_PREC_BF16X3) {
        ST(search_mdomain(h, nshifts, shifts, precision, ntop, (pftcc_best *)out_dev, nullptr));
    } else {
        return set_err(h, PFTCC_ERR_ARG, "search_best: unknown precision");
    }
    CK(cudaStreamSynchronize(h->stream), "search_best");
    return PFTCC_OK;
}

int pftcc_set_tuning(pftcc_handle *h, const pftcc_tuning *t)
{
    if (!h || !t) return set_err(h, PFTCC_ERR_ARG, "set_tuning: bad arguments");
    if (t->w_rows < 0 || t->w_cols < 0 || (t->s1_stages != 0 && (t->s1_stages < 2 || t->s1_stages > 4)))
        return set_err(h, PFTCC_ERR_ARG, "set_tuning: w_rows, w_cols >= 0 and s1_stages 0 or 2..4");
    std::lock_guard<std::mutex> lk(h->mtx);
    h->tune = *t;
    h->tune.from_wisdom = 0;
    return PFTCC_OK;
}

int pftcc_get_tuning(const pftcc_handle *h, pftcc_tuning *t)
{
    if (!h || !t) return PFTCC_ERR_ARG;
    *t = h->tune;
    return PFTCC_OK;
}

// the wisdom line of a search shape: the device and what decides the work's cut
static std::string wisdom_key(pftcc_handle *h, int nshifts, int precision, int ntop)
{
    cudaDeviceProp pr{};
    cudaGetDeviceProperties(&pr, h->dev);
    std::string dev = pr.name;
    for (char &c : dev)
        if (c == ' ') c = '_';
    return "pftcc-wisdom-v1 " + dev + " sms=" + std::to_string(pr.multiProcessorCount) + " nrots=" +
           std::to_string(h->g.N) + " shells=" + std::to_string(h->g.Ks) + " rows=" +
           std::to_string((long long)h->nrefs * std::max(1, nshifts)) + " cols=" + std::to_string(h->nptcls) +
           " prec=" + std::to_string(precision) + " frame=" + std::to_string(h->cfg.ctf_frame) + " ntop=" +
           std::to_string(ntop) + " objfun=" + std::to_string(h->objfun);
}

int pftcc_autotune(pftcc_handle *h, int nshifts, const float *shifts, int precision, int ntop, const char *wisdom,
                   pftcc_tuning *out)
{
    if (!h || nshifts < 0 || (nshifts > 0 && !shifts) || ntop < 0 || ntop > 8 ||
        (precision != PFTCC_PREC_FP32 && precision != PFTCC_PREC_BF16X3))
        return set_err(h, PFTCC_ERR_ARG, "autotune: bad arguments (FP32 or BF16X3 searches are tuned)");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    const std::string key = wisdom_key(h, nshifts, precision, ntop);
    if (wisdom) {
        if (FILE *f = std::fopen(wisdom, "r")) {
            char line[1024];
            pftcc_tuning t{};
            bool found = false;
            while (std::fgets(line, sizeof line, f)) {
                std::string l(line);
                const size_t arrow = l.find(" -> ");
                if (arrow == std::string::npos || l.substr(0, arrow) != key) continue;
                if (std::sscanf(l.c_str() + arrow + 4, "w_rows=%d w_cols=%d s1_stages=%d", &t.w_rows, &t.w_cols,
                                &t.s1_stages) == 3)
                    found = true;   // the last matching line wins
            }
            std::fclose(f);
            if (found) {
                h->tune = t;
                h->tune.from_wisdom = 1;
                if (out) *out = h->tune;
                return PFTCC_OK;
            }
        }
    }
    ST(ensure(h, (void **)&h->d_best, &h->best_cap, (size_t)h->nptcls * sizeof(pftcc_best), "best"));
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0), "autotune");
    CK(cudaEventCreate(&e1), "autotune");
    // one timed search (after an untimed one that sizes the workspace) per candidate
    auto timed = [&](const pftcc_tuning &t, float *ms) -> int {
        h->tune = t;
        for (int rep = 0; rep < 2; ++rep) {
            if (rep == 1) CK(cudaEventRecord(e0, h->stream), "autotune");
            ST(search_mdomain(h, nshifts, shifts, precision, ntop, h->d_best, nullptr));
            if (rep == 1) CK(cudaEventRecord(e1, h->stream), "autotune");
        }
        CK(cudaEventSynchronize(e1), "autotune");
        CK(cudaEventElapsedTime(ms, e0, e1), "autotune");
        return PFTCC_OK;
    };
    const int rows = (int)std::min<long long>((long long)h->nrefs * std::max(1, nshifts), 1 << 30);
    pftcc_tuning best{0, 0, 0, 0};
    float best_ms = 0.f;
    int st = timed(best, &best_ms);
    const int wr_c[] = {2048, 4096, 8192, 16384}, wc_c[] = {512, 1024, 2048, 4096, 8192}, s1_c[] = {2, 3, 4};
    for (int dim = 0; dim < 3 && st == PFTCC_OK; ++dim) {
        const int *vals = dim == 0 ? wc_c : dim == 1 ? wr_c : s1_c;
        const int nv = dim == 0 ? 5 : dim == 1 ? 4 : 3;
        for (int v = 0; v < nv && st == PFTCC_OK; ++v) {
            pftcc_tuning t = best;
            if (dim == 0) { if (vals[v] > h->nptcls + 127) continue; t.w_cols = vals[v]; }
            if (dim == 1) { if (vals[v] > rows + 63) continue; t.w_rows = vals[v]; }
            if (dim == 2) t.s1_stages = vals[v];
            float ms = 0.f;
            st = timed(t, &ms);
            if (st == PFTCC_ERR_OOM) { st = PFTCC_OK; continue; }   // a wave too large for the free memory
            if (st == PFTCC_OK && ms < best_ms) { best_ms = ms; best = t; }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    h->tune = best;
    h->tune.from_wisdom = 0;
    if (st != PFTCC_OK) return st;
    if (wisdom) {
        if (FILE *f = std::fopen(wisdom, "a")) {
            std::fprintf(f, "%s -> w_rows=%d w_cols=%d s1_stages=%d ms=%.3f\n", key.c_str(), best.w_rows, best.w_cols,
                         best.s1_stages, best_ms);
            std::fclose(f);
        }
    }
    if (out) *out = h->tune;
    return PFTCC_OK;
}

static int search_groups_args(pftcc_handle *h, int ngroups, const int *ref_first, const int *nref,
                              const int *slot_first, const int *nslot, int nshifts, const float *shifts, int ntop)
{
    if (!h || ngroups < 0 || (ngroups > 0 && (!ref_first || !nref || !slot_first || !nslot)) || nshifts < 0 ||
        (nshifts > 0 && !shifts) || ntop < 0 || ntop > 8)
        return set_err(h, PFTCC_ERR_ARG, "search_groups: bad arguments");
    return PFTCC_OK;
}

int pftcc_search_groups_dev(pftcc_handle *h, int ngroups, const int *ref_first, const int *nref, const int *slot_first,
                            const int *nslot, int nshifts, const float *shifts, int precision, int ntop, void *out_dev)
{
    ST(search_groups_args(h, ngroups, ref_first, nref, slot_first, nslot, nshifts, shifts, ntop));
    if (!out_dev) return set_err(h, PFTCC_ERR_ARG, "search_groups_dev: bad arguments");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    std::vector<int> r0(ngroups), s0(ngroups);
    for (int q = 0; q < ngroups; ++q) { r0[q] = ref_first[q] - 1; s0[q] = slot_first[q] - 1; }
    ST(search_mdomain_groups(h, ngroups, r0.data(), nref, s0.data(), nslot, nshifts, shifts, precision, ntop,
                             (pftcc_best *)out_dev, 0));
    return PFTCC_OK;
}

int pftcc_search_check(pftcc_handle *h)
{
    if (!h) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    return umma_check(h);
}

int pftcc_search_groups(pftcc_handle *h, int ngroups, const int *ref_first, const int *nref, const int *slot_first,
                        const int *nslot, int nshifts, const float *shifts, int precision, int ntop, pftcc_best *out)
{
    ST(search_groups_args(h, ngroups, ref_first, nref, slot_first, nslot, nshifts, shifts, ntop));
    if (!out) return set_err(h, PFTCC_ERR_ARG, "search_groups: bad arguments");
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    ST(check_ctf_state(h));
    ST(ensure(h, (void **)&h->d_best, &h->best_cap, (size_t)h->nptcls * sizeof(pftcc_best), "best"));
    std::vector<int> r0(ngroups), s0(ngroups);
    for (int q = 0; q < ngroups; ++q) { r0[q] = ref_first[q] - 1; s0[q] = slot_first[q] - 1; }
    ST(search_mdomain_groups(h, ngroups, r0.data(), nref, s0.data(), nslot, nshifts, shifts, precision, ntop, h->d_best,
                             1));
    CK(cudaMemcpyAsync(out, h->d_best, (size_t)h->nptcls * sizeof(pftcc_best), cudaMemcpyDeviceToHost, h->stream),
       "search download");
    CK(cudaStreamSynchronize(h->stream), "search_groups");
    return PFTCC_OK;
}

int pftcc_search_best(pftcc_handle *h, int nshifts, const float *shifts, int precision, int ntop, pftcc_best *out)
{
    if (!h || !out) return set_err(h, PFTCC_ERR_ARG, "search_best: bad arguments");
    {
        std::lock_guard<std::mutex> lk(h->mtx);
        cudaSetDevice(h->dev);
        ST(ensure(h, (void **)&h->d_best, &h->best_cap, (size_t)h->nptcls * sizeof(pftcc_best), "best"));
    }
    ST(pftcc_search_best_dev(h, nshifts, shifts, precision, ntop, h->d_best));
    CK(cudaMemcpy(out, h->d_best, (size_t)h->nptcls * sizeof(pftcc_best), cudaMemcpyDeviceToHost), "search download");
    return PFTCC_OK;
}

int pftcc_grad_batch(pftcc_handle *h, int nreq, const pftcc_grad_req *req, double *f, double *grad3)
{
    if (!h || nreq < 0 || (nreq > 0 && (!req || !f || !grad3))) return set_err(h, PFTCC_ERR_ARG, "grad_batch: bad arguments");
    if (nreq == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    if (h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "the adjoint is served in the reference frame");
    ST(check_ctf_state(h));
    return grad_batch_host(h, nreq, req, f, grad3);
}

int pftcc_refine_batch(pftcc_handle *h, int n, const pftcc_refine_req *req, const double *lb, const double *ub,
                       int maxits, double pgtol, double factr, pftcc_refine_out *out)
{
    if (!h || n < 0 || (n > 0 && (!req || !lb || !ub || !out)) || maxits < 1 || !(pgtol >= 0) || !(factr >= 0))
        return set_err(h, PFTCC_ERR_ARG, "refine_batch: bad arguments");
    for (long long e = 0; e < 3LL * n; ++e)
        if (!(lb[e] <= ub[e])) return set_err(h, PFTCC_ERR_ARG, "refine_batch: empty box");
    if (n == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    if (h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "the adjoint is served in the reference frame");
    ST(check_ctf_state(h));
    return refine_batch(h, n, req, lb, ub, maxits, pgtol, factr, out);
}

int pftcc_shsrch_batch(pftcc_handle *h, int mode, const pftcc_shsrch_opts *opts, int n, const pftcc_shsrch_req *req,
                       pftcc_shsrch_out *out)
{
    if (!h || !opts || n < 0 || (n > 0 && (!req || !out))) return set_err(h, PFTCC_ERR_ARG, "shsrch_batch: bad arguments");
    if (mode != PFTCC_SHSRCH_MINIMIZE && mode != PFTCC_SHSRCH_EXHAUSTIVE)
        return set_err(h, PFTCC_ERR_ARG, "shsrch_batch: mode must be PFTCC_SHSRCH_MINIMIZE or PFTCC_SHSRCH_EXHAUSTIVE");
    if (opts->maxits < 1 || opts->max_evals < 1) return set_err(h, PFTCC_ERR_ARG, "shsrch_batch: maxits and max_evals >= 1");
    if (n == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    if (h->cfg.ctf_frame != PFTCC_FRAME_REF)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "the shift search is served in the reference frame");
    // minimize_exhaustive's rotation window (:167-170)
    if (mode == PFTCC_SHSRCH_EXHAUSTIVE && opts->halfrot > 0.f &&
        (opts->halfrot >= 180.f || opts->halfrot < fabsf(h->angtab[1] - h->angtab[0])))
        return set_err(h, PFTCC_ERR_ARG, "shsrch_batch: invalid rotation boundary (halfrot)");
    std::vector<int> slots(n);
    for (int i = 0; i < n; ++i) {
        if (req[i].iref < 1 || req[i].iref > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "shsrch_batch: iref");
        const int sl = slot_of(h, req[i].iptcl);
        if (sl < 0) return set_err(h, PFTCC_ERR_INDEX, "shsrch_batch: particle not held");
        slots[i] = sl;
        if (mode == PFTCC_SHSRCH_MINIMIZE && !opts->opt_angle && (req[i].irot < 1 || req[i].irot > h->g.N))
            return set_err(h, PFTCC_ERR_INDEX, "shsrch_batch: irot");
        if (mode == PFTCC_SHSRCH_EXHAUSTIVE && req[i].irot > h->g.N) return set_err(h, PFTCC_ERR_INDEX, "shsrch_batch: irot");
        if (!(req[i].lims[0][0] <= req[i].lims[0][1]) || !(req[i].lims[1][0] <= req[i].lims[1][1]))
            return set_err(h, PFTCC_ERR_ARG, "shsrch_batch: empty shift box");
    }
    ST(check_ctf_state(h));
    ST(exact_objfun_ok(h));
    return shsrch_batch(h, mode, *opts, n, req, slots.data(), out);
}

}  // extern "C"

// pending requests of the adjoint, evaluated in one launch (the caller holds the lock)
int pftcc::grad_batch_host(pftcc_handle *h, int nreq, const pftcc_grad_req *req, double *f, double *grad3)
{
    std::vector<int> slots(nreq);
    for (int i = 0; i < nreq; ++i) {
        if (req[i].iref < 1 || req[i].iref > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "grad_batch: iref");
        if (req[i].irot < 1 || req[i].irot > h->g.N) return set_err(h, PFTCC_ERR_INDEX, "grad_batch: irot");
        const int s = slot_of(h, req[i].iptcl);
        if (s < 0) return set_err(h, PFTCC_ERR_INDEX, "grad_batch: iptcl");
        slots[i] = s;
    }
    // device layout: [req][slots][RotReq work area][out]
    const size_t rq_bytes = (size_t)nreq * sizeof(pftcc_grad_req);
    ST(ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>((size_t)nreq * 48, 4096), "grad work"));
    ST(ensure(h, (void **)&h->d_dout, &h->dout_cap, (size_t)nreq * 5 * sizeof(double) + rq_bytes + (size_t)nreq * 4 + 64,
              "grad out"));
    char *base = (char *)h->d_dout;
    double *dout = (double *)base;
    pftcc_grad_req *dreq = (pftcc_grad_req *)(base + (size_t)nreq * 5 * sizeof(double));
    int *dslots = (int *)((char *)dreq + rq_bytes);
    CK(cudaMemcpyAsync(dreq, req, rq_bytes, cudaMemcpyHostToDevice, h->stream), "grad upload");
    CK(cudaMemcpyAsync(dslots, slots.data(), (size_t)nreq * sizeof(int), cudaMemcpyHostToDevice, h->stream), "grad upload");
    CK(launch_grad_batch(h, dreq, dslots, nreq, dout), "grad kernel");
    std::vector<double> o((size_t)nreq * 5);
    CK(cudaMemcpyAsync(o.data(), dout, o.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "grad download");
    CK(cudaStreamSynchronize(h->stream), "grad");
    for (int i = 0; i < nreq; ++i) {
        f[i] = o[5 * i];
        grad3[3 * i] = o[5 * i + 1];
        grad3[3 * i + 1] = o[5 * i + 2];
        grad3[3 * i + 2] = o[5 * i + 3];
    }
    return PFTCC_OK;
}

extern "C" {

// ---- getters -------------------------------------------------------------------------------
int pftcc_get_nrots(const pftcc_handle *h, int *v) { if (!h || !v) return PFTCC_ERR_ARG; *v = h->g.N; return PFTCC_OK; }
int pftcc_get_pftsz(const pftcc_handle *h, int *v) { if (!h || !v) return PFTCC_ERR_ARG; *v = h->g.P; return PFTCC_OK; }
int pftcc_get_box(const pftcc_handle *h, int *v) { if (!h || !v) return PFTCC_ERR_ARG; *v = h->g.box; return PFTCC_OK; }
int pftcc_get_nrefs(const pftcc_handle *h, int *v) { if (!h || !v) return PFTCC_ERR_ARG; *v = h->nrefs; return PFTCC_OK; }
int pftcc_get_nptcls(const pftcc_handle *h, int *v) { if (!h || !v) return PFTCC_ERR_ARG; *v = h->nptcls; return PFTCC_OK; }
int pftcc_exists(const pftcc_handle *h, int *v) { if (!v) return PFTCC_ERR_ARG; *v = h != nullptr; return PFTCC_OK; }

int pftcc_get_pdim(const pftcc_handle *h, int pdim[3])
{
    if (!h || !pdim) return PFTCC_ERR_ARG;
    pdim[0] = h->g.P; pdim[1] = h->g.kfrom; pdim[2] = h->g.kto;
    return PFTCC_OK;
}

// get_rot :624-634
int pftcc_get_rot(const pftcc_handle *h, int roind, float *rot)
{
    if (!h || !rot) return PFTCC_ERR_ARG;
    if (roind < 1 || roind > h->g.N) return PFTCC_ERR_INDEX;
    *rot = h->angtab[roind - 1];
    return PFTCC_OK;
}

// get_roind :638-647: argmin of the cyclic angular distance, first minimum
int pftcc_get_roind(const pftcc_handle *h, float rot, int *roind)
{
    if (!h || !roind) return PFTCC_ERR_ARG;
    float best = INFINITY;
    int loc = 1;
    for (int i = 0; i < h->g.N; ++i) {
        float d = fabsf(h->angtab[i] - rot);
        if (d > 180.f) d = 360.f - d;
        if (d < best) { best = d; loc = i + 1; }
    }
    *roind = loc;
    return PFTCC_OK;
}

// get_coord :651-657
int pftcc_get_coord(const pftcc_handle *h, int rot, int k, float xy[2])
{
    if (!h || !xy) return PFTCC_ERR_ARG;
    if (rot < 1 || rot > h->g.N || k < h->g.kfrom || k > h->g.kto) return PFTCC_ERR_INDEX;
    const int ik = k - h->g.kfrom;
    xy[0] = h->h_polar[(size_t)ik * 2 * h->g.N + rot - 1];
    xy[1] = h->h_polar[(size_t)ik * 2 * h->g.N + h->g.N + rot - 1];
    return PFTCC_OK;
}

int pftcc_ptcl_iseven(const pftcc_handle *h, int iptcl, int *iseven)
{
    if (!h || !iseven) return PFTCC_ERR_ARG;
    const int s = slot_of(h, iptcl);
    if (s < 0) return PFTCC_ERR_INDEX;
    *iseven = h->iseven[s];
    return PFTCC_OK;
}

int pftcc_get_ref_pft(pftcc_handle *h, int iref, int iseven, float *pft)
{
    if (!h || !pft) return PFTCC_ERR_ARG;
    REF_OR_FAIL(iref);
    cudaSetDevice(h->dev);
    const size_t KP = (size_t)h->g.K * h->g.P;
    CK(cudaMemcpyAsync(pft, (iseven ? h->refs_even : h->refs_odd) + (iref - 1) * KP, KP * sizeof(float2),
                       cudaMemcpyDeviceToHost, h->stream), "get_ref_pft");
    CK(cudaStreamSynchronize(h->stream), "get_ref_pft");
    return PFTCC_OK;
}

int pftcc_get_ptcl_pft(pftcc_handle *h, int iptcl, float *pft)
{
    if (!h || !pft) return PFTCC_ERR_ARG;
    SLOT_OR_FAIL(slot, iptcl);
    cudaSetDevice(h->dev);
    const size_t KP = (size_t)h->g.K * h->g.P;
    CK(cudaMemcpyAsync(pft, h->ptcls + slot * KP, KP * sizeof(float2), cudaMemcpyDeviceToHost, h->stream), "get_ptcl_pft");
    CK(cudaStreamSynchronize(h->stream), "get_ptcl_pft");
    return PFTCC_OK;
}

int pftcc_get_sqsum_ptcl(pftcc_handle *h, int iptcl, float *sq)
{
    if (!h || !sq) return PFTCC_ERR_ARG;
    SLOT_OR_FAIL(slot, iptcl);
    cudaSetDevice(h->dev);
    CK(cudaMemcpyAsync(sq, h->sqsums + slot, sizeof(float), cudaMemcpyDeviceToHost, h->stream), "sqsum");
    CK(cudaStreamSynchronize(h->stream), "sqsum");
    return PFTCC_OK;
}

int pftcc_synchronize(pftcc_handle *h)
{
    if (!h) return PFTCC_ERR_ARG;
    cudaSetDevice(h->dev);
    CK(cudaStreamSynchronize(h->stream), "synchronize");
    return PFTCC_OK;
}

int pftcc_set_stream(pftcc_handle *h, void *stream)
{
    if (!h) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    CK(cudaStreamSynchronize(h->stream), "set_stream");
    if (!h->own_stream) h->own_stream = h->stream;
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return PFTCC_OK;
}

int pftcc_set_wait_limit(pftcc_handle *h, long long polls)
{
    if (!h || polls < 0) return set_err(h, PFTCC_ERR_ARG, "set_wait_limit: polls >= 0");
    std::lock_guard<std::mutex> lk(h->mtx);
    h->wait_limit = polls;
    return PFTCC_OK;
}

static void prof_collect(pftcc_handle *h)
{
    if (h->prof_pending.empty()) return;
    cudaStreamSynchronize(h->stream);
    for (auto &p : h->prof_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
            h->prof_ms[p.cls] += ms;
            h->prof_n[p.cls] += 1;
        }
        h->prof_pool.push_back(p.a);
        h->prof_pool.push_back(p.b);
    }
    h->prof_pending.clear();
    cudaGetLastError();
}

int pftcc_prof_enable(pftcc_handle *h, int on)
{
    if (!h) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    h->prof = on ? 1 : 0;
    return PFTCC_OK;
}

int pftcc_prof_read(pftcc_handle *h, int cls, double *ms, long long *n)
{
    if (!h || !ms || !n || cls < 0 || cls >= PFTCC_K_COUNT) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    prof_collect(h);
    *ms = h->prof_ms[cls];
    *n = h->prof_n[cls];
    return PFTCC_OK;
}

int pftcc_prof_reset(pftcc_handle *h)
{
    if (!h) return PFTCC_ERR_ARG;
    std::lock_guard<std::mutex> lk(h->mtx);
    cudaSetDevice(h->dev);
    prof_collect(h);
    for (int i = 0; i < PFTCC_K_COUNT; ++i) { h->prof_ms[i] = 0.0; h->prof_n[i] = 0; }
    return PFTCC_OK;
}

}  // extern "C"
