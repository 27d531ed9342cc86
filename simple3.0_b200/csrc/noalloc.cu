// noalloc.cu -- gencorrs for a batch of (reference, particle, shift) pairs without any
// device allocation.  It serves callers that cannot let a library call cudaMalloc:
// applications that hand all device memory to their own pool at start-up and budget
// it there (an allocation made behind the pool's back can fail or fragment it), and
// long-running services that must keep a fixed device footprint after start-up.
//
// The per-call work descriptors live in one file-scope device array of a fixed size
// (noalloc_scratch, 256 KiB, so at most 6553 pairs per call); every GPU that loads this
// library holds that array until the process exits.  In host code the array's name
// stands for a host-side shadow, not a device address, so the first call on each
// device resolves the address with cudaGetSymbolAddress (with that device current)
// and caches it; make that first call before any stream capture begins.  All calls
// share the array and each call rewrites the part it uses (nothing in it has to start
// at zero); calls whose work overlaps on the GPU race on it, so order them on one
// stream.
#include "pftcc_internal.cuh"

#include <mutex>

namespace pftcc {

constexpr size_t NOALLOC_SCRATCH_BYTES = 256 * 1024;
// per pair: one Work (16 B), one Group (16 B) and one shift (8 B)
constexpr int NOALLOC_PAIR_BYTES = (int)(sizeof(Work) + sizeof(Group) + 2 * sizeof(float));
static_assert(sizeof(Work) == 16 && sizeof(Group) == 16, "descriptor sizes");

static __device__ __align__(256) unsigned char noalloc_scratch[NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mtx;
static void *g_noalloc_ptr[64] = {};
static std::mutex g_noalloc_host_mtx;
static unsigned char g_noalloc_host[NOALLOC_SCRATCH_BYTES];

static int noalloc_base(pftcc_handle *h, void **base)
{
    std::lock_guard<std::mutex> lk(g_noalloc_mtx);
    if (h->dev < 0 || h->dev >= 64) return set_err(h, PFTCC_ERR_NODEV, "gencorrs_noalloc: device ordinal >= 64");
    if (!g_noalloc_ptr[h->dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, noalloc_scratch);
        if (e != cudaSuccess || !p) return cuda_err(h, e == cudaSuccess ? cudaErrorInvalidSymbol : e, "gencorrs_noalloc scratch");
        g_noalloc_ptr[h->dev] = p;
    }
    *base = g_noalloc_ptr[h->dev];
    return PFTCC_OK;
}

}  // namespace pftcc

using namespace pftcc;

extern "C" int pftcc_gencorrs_noalloc(pftcc_handle *h, int npairs, const int *iref, const int *iptcl,
                                      const float *shifts, float *cc_dev)
{
    if (!h || npairs < 0 || (npairs > 0 && (!iref || !iptcl || !cc_dev)))
        return set_err(h, PFTCC_ERR_ARG, "gencorrs_noalloc: bad arguments");
    const int max_pairs = (int)(NOALLOC_SCRATCH_BYTES / NOALLOC_PAIR_BYTES);
    if (npairs > max_pairs)
        return set_err(h, PFTCC_ERR_ARG, "gencorrs_noalloc: " + std::to_string(npairs) + " pairs exceed the " +
                                             std::to_string(max_pairs) + "-pair fixed scratch; split the batch");
    if (npairs == 0) return PFTCC_OK;
    std::lock_guard<std::mutex> lk(h->mtx);
    if (cudaSetDevice(h->dev) != cudaSuccess) return set_err(h, PFTCC_ERR_CUDA, "gencorrs_noalloc: cudaSetDevice");
    if (h->cfg.with_ctf && !h->ctf_ready)
        return set_err(h, PFTCC_ERR_STATE, "CTF is on but create_polar_absctfmats has not been called");
    if (h->objfun == PFTCC_OBJFUN_EUCLID && euclid_ready(h, 0) != PFTCC_OK) return PFTCC_ERR_STATE;
    if (exact_objfun_ok(h) != PFTCC_OK) return PFTCC_ERR_UNSUPPORTED;
    {   // matched-filter factors: computed into arrays that pftcc_new allocated
        const int st = snorm_ready(h, 0, h->nrefs);
        if (st != PFTCC_OK) return st;
    }
    // host-side descriptors (validated) in a fixed host buffer guarded by the global lock,
    // then one copy into the fixed device scratch
    std::lock_guard<std::mutex> lk2(g_noalloc_host_mtx);
    unsigned char *host = g_noalloc_host;
    const size_t host_bytes = (size_t)npairs * NOALLOC_PAIR_BYTES;
    Work *w = reinterpret_cast<Work *>(host);
    Group *g = reinterpret_cast<Group *>(w + npairs);
    float *s = reinterpret_cast<float *>(g + npairs);
    for (int i = 0; i < npairs; ++i) {
        if (iref[i] < 1 || iref[i] > h->nrefs) return set_err(h, PFTCC_ERR_INDEX, "gencorrs_noalloc: iref out of range");
        const int p = iptcl[i];
        const int slot = (p < h->pfrom || p > h->pto) ? -1 : h->pinds[p - h->pfrom] - 1;
        if (slot < 0) return set_err(h, PFTCC_ERR_INDEX, "gencorrs_noalloc: particle not held");
        w[i] = Work{iref[i] - 1, shifts ? i : -1, (long long)i * h->g.N};
        g[i] = Group{slot, i, 1, 0};
        s[2 * i] = shifts ? shifts[2 * i] : 0.f;
        s[2 * i + 1] = shifts ? shifts[2 * i + 1] : 0.f;
    }
    void *base = nullptr;
    int st = noalloc_base(h, &base);
    if (st != PFTCC_OK) return st;
    cudaError_t e = cudaMemcpyAsync(base, host, host_bytes, cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "gencorrs_noalloc upload");
    unsigned char *b = static_cast<unsigned char *>(base);
    const Work *dw = reinterpret_cast<const Work *>(b);
    const Group *dg = reinterpret_cast<const Group *>(b + (size_t)npairs * sizeof(Work));
    const float *ds = reinterpret_cast<const float *>(b + (size_t)npairs * (sizeof(Work) + sizeof(Group)));
    e = launch_exact(h, dg, npairs, dw, ds, MODE_FULL, exact_frame(h), 1, cc_dev, nullptr);
    if (e != cudaSuccess) return cuda_err(h, e, "gencorrs_noalloc kernel");
    // the host descriptors must outlive the copy
    e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "gencorrs_noalloc");
    return PFTCC_OK;
}
