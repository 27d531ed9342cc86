// C entry points around the library's L-BFGS-B (simple3.0_b200/csrc/lbfgsb3.h), one problem
// per object in reverse communication, so that the oracle's restatement of the reference's
// shift search (oracle/shsrch.py) steps the same optimiser the library does while every
// cost and gradient comes from the oracle's FP64 correlations.  TEST INFRASTRUCTURE ONLY.
#include "lbfgsb3.h"

using Solver2 = pftcc::lbfgsb3::Solver<2>;

extern "C" {

void *lb3_new(const double *x0, const double *lb, const double *ub, double factr, double pgtol, double ftol,
              double gtol, double xtol, int m)
{
    Solver2 *s = new Solver2();
    pftcc::lbfgsb3::Options o;
    o.factr = factr; o.pgtol = pgtol; o.ftol = ftol; o.gtol = gtol; o.xtol = xtol; o.m = m;
    s->start(x0, lb, ub, o);
    return s;
}

void lb3_free(void *p) { delete static_cast<Solver2 *>(p); }
int lb3_task(void *p) { return static_cast<Solver2 *>(p)->task; }
int lb3_nfgv(void *p) { return static_cast<Solver2 *>(p)->nfgv; }
double lb3_f(void *p) { return static_cast<Solver2 *>(p)->f; }

void lb3_x(void *p, double *x)
{
    const Solver2 *s = static_cast<Solver2 *>(p);
    x[0] = s->x[0]; x[1] = s->x[1];
}

void lb3_xt(void *p, double *x)
{
    const Solver2 *s = static_cast<Solver2 *>(p);
    x[0] = s->xt[0]; x[1] = s->xt[1];
}

int lb3_evaluated(void *p, double f, const double *g) { return static_cast<Solver2 *>(p)->evaluated(f, g); }
int lb3_proceed(void *p) { return static_cast<Solver2 *>(p)->proceed(); }

}  // extern "C"
