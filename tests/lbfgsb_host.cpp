// Host test shim: runs the refinement's batched bound-constrained L-BFGS
// (simple3.0_b200/csrc/lbfgsb.h, the same source the library compiles) with the cost
// and gradient supplied by a C callback, so the optimiser logic is tested on the CPU
// against analytic functions and the oracle's correlation and adjoint.
#include "lbfgsb.h"

extern "C" {

typedef int (*lbfgsb_eval_fn)(int nb, const int *idx, const double *xt, double *f, double *g);

int lbfgsb_run(int n, const double *x0, const double *lb, const double *ub, int maxits, double pgtol, double factr,
               lbfgsb_eval_fn cb, double *x_out, double *f_out, int *nevals, int *niter, int *converged)
{
    std::vector<pftcc::lbfgsb::Result<3>> res(n);
    auto eval = [&](int nb, const int *idx, const double *xt, double *f, double *g) { return cb(nb, idx, xt, f, g); };
    const int st = pftcc::lbfgsb::minimize_batch(n, x0, lb, ub, maxits, pgtol, factr, eval, res.data());
    for (int i = 0; i < n; ++i) {
        for (int v = 0; v < 3; ++v) x_out[3 * i + v] = res[i].x[v];
        f_out[i] = res[i].f;
        nevals[i] = res[i].nevals;
        niter[i] = res[i].niter;
        converged[i] = res[i].converged;
    }
    return st;
}

}  // extern "C"
