// refine.cu -- batched continuous refinement of (shift_x, shift_y, defocus) per
// (reference, particle, rotation) problem: the bound-constrained L-BFGS of lbfgsb.h
// minimises -corr, and every round's pending function+gradient requests of all
// unfinished problems are served by ONE launch of the adjoint kernel (grad_batch_host).
// Each problem has its own box, as the reference bounds every particle's shift search
// around its own prior (simple_pftcc_shsrch_grad.f90:44-68).
#include "pftcc_internal.cuh"
#include "lbfgsb.h"

#include <vector>

namespace pftcc {

int refine_batch(pftcc_handle *h, int n, const pftcc_refine_req *req, const double *lb, const double *ub, int maxits,
                 double pgtol, double factr, pftcc_refine_out *out)
{
    constexpr int NV = 3;
    std::vector<double> x0((size_t)n * NV);
    for (int i = 0; i < n; ++i)
        for (int v = 0; v < NV; ++v) x0[(size_t)i * NV + v] = req[i].x0[v];
    std::vector<pftcc_grad_req> batch;
    std::vector<double> corr, g3;
    auto eval = [&](int nb, const int *idx, const double *xt, double *f, double *g) -> int {
        batch.resize(nb);
        for (int b = 0; b < nb; ++b) {
            const pftcc_refine_req &r = req[idx[b]];
            batch[b] = pftcc_grad_req{r.iref, r.iptcl, r.irot, 0, xt[NV * b], xt[NV * b + 1], xt[NV * b + 2]};
        }
        corr.assign(nb, 0.0);
        g3.assign((size_t)NV * nb, 0.0);
        const int st = grad_batch_host(h, nb, batch.data(), corr.data(), g3.data());
        if (st != PFTCC_OK) return st;
        for (int b = 0; b < nb; ++b) {             // cost = -corr
            f[b] = -corr[b];
            for (int v = 0; v < NV; ++v) g[NV * b + v] = -g3[(size_t)NV * b + v];
        }
        return 0;
    };
    std::vector<lbfgsb::Result<NV>> res(n);
    const int st = lbfgsb::minimize_batch(n, x0.data(), lb, ub, maxits, pgtol, factr, eval, res.data());
    if (st != 0) return st;
    for (int i = 0; i < n; ++i) {
        pftcc_refine_out &o = out[i];
        for (int v = 0; v < NV; ++v) o.x[v] = res[i].x[v];
        o.f = -res[i].f;
        o.nevals = res[i].nevals;
        o.niter = res[i].niter;
        o.converged = res[i].converged;
        o.pad = 0;
    }
    return PFTCC_OK;
}

}  // namespace pftcc
