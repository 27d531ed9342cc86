// k_strategy.cu -- the stochastic reference search of the 2D strategies on the GPU:
// stochastic neighbourhood hill climbing (strategy2D_snhc srch_snhc,
// simple_strategy2D_snhc.f90:33-93) with shcloc (simple_rnd.f90:273-295) for every held
// particle in one call, instead of one gencorrs round trip per visited reference.
//
// All correlations corr(particle, ref, rot) (no shift: the strategy calls
// gencorrs(iref, iptcl, corrs)) are computed once into device memory -- through the
// exact kernel in the handle's CTF frame, or the m-domain path (particle frame) in FP32
// or BF16-split precision -- and one warp per particle then replays the strategy:
// references in the caller's per-particle order, every visit counted against
// nrefs_bound (empty classes skipped after being counted), for each visited reference
// shcloc's uniform pick among the rotations with corr >= prev_corr, ending the search,
// or else the greedy best rotation, kept as the global best that is returned when no
// reference improves.  shcloc's random draw for visit isample of particle iptcl is a
// splitmix64 hash of (seed, iptcl, isample): u in [0,1) selects the k-th improving
// rotation in rotation order, k = floor(u * count).
#include "pftcc_internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace pftcc {

__device__ __forceinline__ double snhc_uniform(unsigned long long seed, int iptcl, int isample)
{
    unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(unsigned)iptcl +
                           0xD1B54A32D192ED03ULL * (unsigned long long)(unsigned)isample;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// one warp per particle slot; cc[slot][ref][rot]
__global__ void __launch_bounds__(256) k_snhc(const float *__restrict__ cc, int np, int nrefs, int N,
                                              const int *__restrict__ order, const int *__restrict__ pops,
                                              int nrefs_bound, const float *__restrict__ prev,
                                              unsigned long long seed, const int *__restrict__ gidx,
                                              pftcc_snhc_out *__restrict__ out)
{
    const int slot = (int)((blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (slot >= np) return;                      // whole warps leave together
    const float pf = prev[slot];
    const int iptcl = gidx[slot];
    float cc_glob = -INFINITY;
    int class_glob = 0, inpl_glob = 0, neval = 0, found = 0, best_ref = 0, best_rot = 0;
    float best_corr = 0.f;
    for (int isample = 1; isample <= nrefs; ++isample) {
        const int iref = order[(size_t)slot * nrefs + isample - 1];
        ++neval;
        if (neval > nrefs_bound) break;
        if (pops && pops[iref - 1] == 0) continue;
        const float *row = cc + ((size_t)slot * nrefs + iref - 1) * N;
        // improving rotations (corr - prev_corr not negative) and the first maximum
        int navail = 0, mi = 0x7fffffff;
        float mv = -INFINITY;
        for (int r = lane; r < N; r += 32) {
            const float v = row[r];
            navail += !(v < pf);
            if (v > mv || (v == mv && r < mi)) { mv = v; mi = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            navail += __shfl_xor_sync(0xffffffffu, navail, o);
            const float ov = __shfl_xor_sync(0xffffffffu, mv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, mi, o);
            if (ov > mv || (ov == mv && oi < mi)) { mv = ov; mi = oi; }
        }
        int inpl;
        float inpl_corr;
        if (navail == 0) {
            inpl = mi == 0x7fffffff ? 0 : mi;
            inpl_corr = row[inpl];
        } else {
            int k = (int)(snhc_uniform(seed, iptcl, isample) * navail);
            if (k >= navail) k = navail - 1;
            inpl = -1;
            for (int base = 0; base < N && inpl < 0; base += 32) {
                const int r = base + lane;
                const unsigned m = __ballot_sync(0xffffffffu, r < N && !(row[r < N ? r : 0] < pf));
                const int cnt = __popc(m);
                if (k < cnt) {
                    unsigned mm = m;
                    for (int q = 0; q < k; ++q) mm &= mm - 1;   // drop the k lowest set bits
                    inpl = base + __ffs(mm) - 1;
                } else {
                    k -= cnt;
                }
            }
            inpl_corr = row[inpl];
            best_ref = iref; best_rot = inpl + 1; best_corr = inpl_corr;
            found = 1;
        }
        if (inpl_corr > cc_glob) { cc_glob = inpl_corr; class_glob = iref; inpl_glob = inpl + 1; }
        if (found) break;
    }
    if (!found) { best_ref = class_glob; best_rot = inpl_glob; best_corr = class_glob ? cc_glob : 0.f; }
    if (lane == 0) {
        pftcc_snhc_out o;
        o.iref = best_ref; o.irot = best_rot; o.found_better = found; o.nrefs_eval = neval;
        o.corr = best_corr; o.pad[0] = o.pad[1] = o.pad[2] = 0;
        out[slot] = o;
    }
}

// every correlation (no shift) of the held particles into dst[slot][ref][rot] on the device
static int corr_all_device(pftcc_handle *h, int precision, float *dst)
{
    if (precision == PFTCC_PREC_FP32 || precision == PFTCC_PREC_BF16X3)
        return search_mdomain(h, 0, nullptr, precision, 0, nullptr, dst);
    const int ok = exact_objfun_ok(h);
    if (ok != PFTCC_OK) return ok;
    const size_t per_ptcl = (size_t)h->nrefs;
    const int chunk = (int)std::max<size_t>(1, std::min<size_t>(h->nptcls, 65536 / std::max<size_t>(1, per_ptcl) + 1));
    int st = ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>((size_t)chunk * per_ptcl * sizeof(Work), 4096),
                    "work");
    if (st) return st;
    st = ensure(h, (void **)&h->d_groups, &h->group_cap, std::max<size_t>((size_t)chunk * sizeof(Group), 256), "groups");
    if (st) return st;
    std::vector<Work> work((size_t)chunk * per_ptcl);
    std::vector<Group> groups(chunk);
    for (int c0 = 0; c0 < h->nptcls; c0 += chunk) {
        const int m = std::min(chunk, h->nptcls - c0);
        size_t wi = 0;
        for (int i = 0; i < m; ++i) {
            groups[i] = Group{c0 + i, (int)wi, (int)per_ptcl, i};
            for (int r = 0; r < h->nrefs; ++r, ++wi) work[wi] = Work{r, -1, (long long)((size_t)i * h->nrefs + r) * h->g.N};
        }
        cudaError_t e = cudaMemcpyAsync(h->d_work, work.data(), wi * sizeof(Work), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(h->d_groups, groups.data(), m * sizeof(Group), cudaMemcpyHostToDevice, h->stream);
        if (e == cudaSuccess)
            e = launch_exact(h, h->d_groups, m, h->d_work, nullptr, MODE_FULL, exact_frame(h), 1,
                             dst + (size_t)c0 * per_ptcl * h->g.N, nullptr);
        if (e != cudaSuccess) return cuda_err(h, e, "snhc correlations");
    }
    return PFTCC_OK;
}

}  // namespace pftcc

using namespace pftcc;

extern "C" int pftcc_search_snhc(pftcc_handle *h, const int *order, const float *prev_corr, const int *cls_pops,
                                 int nrefs_bound, unsigned long long seed, int precision, pftcc_snhc_out *out)
{
    if (!h || !order || !prev_corr || !out || nrefs_bound < 1)
        return set_err(h, PFTCC_ERR_ARG, "search_snhc: bad arguments");
    if (precision != PFTCC_PREC_EXACT && precision != PFTCC_PREC_FP32 && precision != PFTCC_PREC_BF16X3)
        return set_err(h, PFTCC_ERR_ARG, "search_snhc: unknown precision");
    if (precision != PFTCC_PREC_EXACT && h->cfg.ctf_frame != PFTCC_FRAME_PTCL)
        return set_err(h, PFTCC_ERR_UNSUPPORTED, "search_snhc: the FP32/BF16 paths serve the particle CTF frame");
    const int np = h->nptcls, nr = h->nrefs, N = h->g.N;
    if (np == 0) return PFTCC_OK;
    for (size_t e = 0; e < (size_t)np * nr; ++e)
        if (order[e] < 1 || order[e] > nr) return set_err(h, PFTCC_ERR_INDEX, "search_snhc: order holds an invalid iref");
    const size_t cc_bytes = (size_t)np * nr * N * sizeof(float);
    if (cc_bytes > (32ull << 30))
        return set_err(h, PFTCC_ERR_ARG, "search_snhc: nptcls * nrefs * nrots exceeds the 32 GiB correlation buffer; "
                                         "hold fewer particles per call");
    std::lock_guard<std::mutex> lk(h->mtx);
    if (cudaSetDevice(h->dev) != cudaSuccess) return set_err(h, PFTCC_ERR_CUDA, "search_snhc: cudaSetDevice");
    if (h->cfg.with_ctf && !h->ctf_ready)
        return set_err(h, PFTCC_ERR_STATE, "CTF is on but create_polar_absctfmats has not been called");
    if (h->objfun == PFTCC_OBJFUN_EUCLID) {
        const int est = euclid_ready(h, 1);
        if (est != PFTCC_OK) return est;
    }
    {
        const int sst = snorm_ready(h, 0, h->nrefs);
        if (sst != PFTCC_OK) return sst;
    }
    // global particle index of each slot (the random draws are keyed by it)
    std::vector<int> gidx(np, 0);
    for (int p = h->pfrom; p <= h->pto; ++p) {
        const int sl = h->pinds[p - h->pfrom] - 1;
        if (sl >= 0 && sl < np) gidx[sl] = p;
    }
    int st = ensure(h, (void **)&h->d_out, &h->out_cap, cc_bytes, "snhc correlations");
    if (st) return st;
    const size_t aux = (size_t)np * nr * sizeof(int) + (size_t)np * (sizeof(float) + sizeof(int)) +
                       (size_t)nr * sizeof(int) + (size_t)np * sizeof(pftcc_snhc_out) + 1024;
    st = ensure(h, (void **)&h->d_dout, &h->dout_cap, aux, "snhc buffers");
    if (st) return st;
    char *base = (char *)h->d_dout;
    pftcc_snhc_out *dout = (pftcc_snhc_out *)base;
    int *dorder = (int *)(base + (size_t)np * sizeof(pftcc_snhc_out));
    float *dprev = (float *)(dorder + (size_t)np * nr);
    int *dgidx = (int *)(dprev + np);
    int *dpops = dgidx + np;
    cudaError_t e = cudaMemcpyAsync(dorder, order, (size_t)np * nr * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dprev, prev_corr, np * sizeof(float), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dgidx, gidx.data(), np * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    if (e == cudaSuccess && cls_pops)
        e = cudaMemcpyAsync(dpops, cls_pops, nr * sizeof(int), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "search_snhc upload");
    st = corr_all_device(h, precision, h->d_out);
    if (st) return st;
    if (precision == PFTCC_PREC_BF16X3 && (st = umma_check(h)) != PFTCC_OK) return st;
    {
        PFTCC_LAUNCH(h);
        KTimer kt(h, PFTCC_K_OTHER);
        k_snhc<<<(np * 32 + 255) / 256, 256, 0, h->stream>>>(h->d_out, np, nr, N, dorder, cls_pops ? dpops : nullptr,
                                                            nrefs_bound, dprev, seed, dgidx, dout);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, np * sizeof(pftcc_snhc_out), cudaMemcpyDeviceToHost, h->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
    if (e != cudaSuccess) return cuda_err(h, e, "search_snhc");
    return PFTCC_OK;
}
