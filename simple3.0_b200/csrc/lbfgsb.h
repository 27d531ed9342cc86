// lbfgsb.h -- batched bound-constrained limited-memory BFGS for small problems
// (a few variables), host C++ with no CUDA dependency, in reverse communication: every
// round collects the pending cost+gradient requests of all unfinished problems and
// hands them to ONE caller-supplied evaluation (the GPU adjoint launch for the
// refinement; analytic functions or the oracle in the host tests).
//
// The reference minimises -corr over the shift with L-BFGS-B in reverse communication
// (simple_opt_lbfgsb.f90:103-129 drives setulb; the cost is -gencorr_for_rot_8 and the
// gradient -gencorr_grad_for_rot_8, simple_pftcc_shsrch_grad.f90:85-131), with the
// defaults factr = 1e7, pgtol = 1e-5, m = 15 (simple_opt_spec.f90:23-24,271).  This
// driver follows the published algorithm of Byrd, Lu, Nocedal & Zhu (1995, "A limited
// memory algorithm for bound constrained optimization"): the quasi-Newton matrix B is
// the BFGS update of theta*I by the stored correction pairs; each iteration finds the
// generalised Cauchy point along the projected steepest-descent path, minimises the
// quadratic model over the free variables (direct primal method, backtracked into the
// box), and line-searches along the resulting direction (backtracking on the Armijo
// condition).  Convergence: projected gradient max-norm <= pgtol, or relative reduction
// (f_k - f_k+1)/max(|f_k|,|f_k+1|,1) <= factr * machine epsilon.
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

namespace pftcc {
namespace lbfgsb {

template <int NV>
struct Result {
    double x[NV], f;
    int nevals, niter, converged;
};

template <int NV>
struct Prob {
    double x[NV], f = 0, g[NV];
    double lb[NV], ub[NV];
    double xt[NV];                        // trial point being evaluated
    double d[NV], dg0 = 0, alpha = 1;     // line search state
    int ls_iter = 0;
    std::vector<double> S, Y;             // stored pairs, NV each
    double theta = 1.0;
    int iter = 0, nevals = 0, state = 0;  // 0 start, 1 line search, 2 done
    int converged = 0;
};

template <int NV>
inline double proj_grad_norm(const Prob<NV> &p)
{
    double m = 0;
    for (int i = 0; i < NV; ++i) {
        double v = p.x[i] - p.g[i];
        v = std::min(std::max(v, p.lb[i]), p.ub[i]);
        m = std::max(m, std::fabs(v - p.x[i]));
    }
    return m;
}

// dense B = BFGS updates of theta*I with the stored pairs (oldest first)
template <int NV>
inline void form_B(const Prob<NV> &p, double B[NV][NV])
{
    for (int i = 0; i < NV; ++i)
        for (int j = 0; j < NV; ++j) B[i][j] = i == j ? p.theta : 0.0;
    const int np = (int)p.S.size() / NV;
    for (int q = 0; q < np; ++q) {
        const double *s = &p.S[q * NV], *y = &p.Y[q * NV];
        double Bs[NV] = {0, 0, 0}, sBs = 0, ys = 0;
        for (int i = 0; i < NV; ++i) {
            for (int j = 0; j < NV; ++j) Bs[i] += B[i][j] * s[j];
            ys += y[i] * s[i];
        }
        for (int i = 0; i < NV; ++i) sBs += s[i] * Bs[i];
        if (sBs <= 0 || ys <= 0) continue;
        for (int i = 0; i < NV; ++i)
            for (int j = 0; j < NV; ++j) B[i][j] += -Bs[i] * Bs[j] / sBs + y[i] * y[j] / ys;
    }
}

// generalised Cauchy point, then the subspace minimiser backtracked into the box
template <int NV>
inline void direction(const Prob<NV> &p, double d[NV])
{
    double B[NV][NV];
    form_B(p, B);
    // breakpoints of the projected path x(t) = P(x - t g)
    double tb[NV];
    for (int i = 0; i < NV; ++i) {
        if (p.g[i] < 0) tb[i] = (p.x[i] - p.ub[i]) / p.g[i];
        else if (p.g[i] > 0) tb[i] = (p.x[i] - p.lb[i]) / p.g[i];
        else tb[i] = DBL_MAX;
        if (tb[i] < 0) tb[i] = 0;
    }
    int order[NV];
    for (int i = 0; i < NV; ++i) order[i] = i;
    std::sort(order, order + NV, [&](int a, int b) { return tb[a] < tb[b]; });
    double xc[NV], dir[NV];
    bool fixed[NV];
    for (int i = 0; i < NV; ++i) {
        xc[i] = p.x[i];
        fixed[i] = tb[i] == 0;
        dir[i] = fixed[i] ? 0.0 : -p.g[i];
    }
    double tprev = 0;
    for (int seg = 0; seg <= NV; ++seg) {
        const double tnext = seg < NV ? tb[order[seg]] : DBL_MAX;
        if (tnext <= tprev && seg < NV) { fixed[order[seg]] = true; dir[order[seg]] = 0; continue; }
        // model derivative along dir from xc: f' = g.dir + (xc - x)^T B dir, f'' = dir^T B dir
        double z[NV], Bd[NV] = {0, 0, 0};
        for (int i = 0; i < NV; ++i) z[i] = xc[i] - p.x[i];
        for (int i = 0; i < NV; ++i)
            for (int j = 0; j < NV; ++j) Bd[i] += B[i][j] * dir[j];
        double f1 = 0, f2 = 0;
        for (int i = 0; i < NV; ++i) { f1 += p.g[i] * dir[i] + z[i] * Bd[i]; f2 += dir[i] * Bd[i]; }
        if (f1 >= 0) break;
        const double dt = f2 > 0 ? -f1 / f2 : DBL_MAX;
        if (tprev + dt < tnext) {
            for (int i = 0; i < NV; ++i) xc[i] += dt * dir[i];
            break;
        }
        if (seg == NV) break;
        const double step = tnext - tprev;
        for (int i = 0; i < NV; ++i) xc[i] += step * dir[i];
        const int v = order[seg];
        xc[v] = dir[v] < 0 ? p.lb[v] : p.ub[v];
        fixed[v] = true;
        dir[v] = 0;
        tprev = tnext;
    }
    for (int i = 0; i < NV; ++i) xc[i] = std::min(std::max(xc[i], p.lb[i]), p.ub[i]);
    // subspace minimisation over the free variables at the Cauchy point
    int fr[NV], nf = 0;
    for (int i = 0; i < NV; ++i)
        if (xc[i] > p.lb[i] && xc[i] < p.ub[i]) fr[nf++] = i;
    double xbar[NV] = {xc[0], xc[1], xc[2]};
    if (nf > 0) {
        double r[NV];
        for (int i = 0; i < NV; ++i) {
            r[i] = p.g[i];
            for (int j = 0; j < NV; ++j) r[i] += B[i][j] * (xc[j] - p.x[j]);
        }
        // solve B_FF du = -r_F (Gaussian elimination with partial pivoting, nf <= NV)
        double A[NV][NV + 1];
        for (int a = 0; a < nf; ++a) {
            for (int b = 0; b < nf; ++b) A[a][b] = B[fr[a]][fr[b]];
            A[a][nf] = -r[fr[a]];
        }
        bool ok = true;
        for (int c = 0; c < nf && ok; ++c) {
            int piv = c;
            for (int a = c + 1; a < nf; ++a)
                if (std::fabs(A[a][c]) > std::fabs(A[piv][c])) piv = a;
            if (std::fabs(A[piv][c]) < 1e-300) { ok = false; break; }
            for (int b = 0; b <= nf; ++b) std::swap(A[c][b], A[piv][b]);
            for (int a = 0; a < nf; ++a)
                if (a != c) {
                    const double fct = A[a][c] / A[c][c];
                    for (int b = c; b <= nf; ++b) A[a][b] -= fct * A[c][b];
                }
        }
        if (ok) {
            double du[NV];
            for (int a = 0; a < nf; ++a) du[a] = A[a][nf] / A[a][a];
            double amax = 1.0;
            for (int a = 0; a < nf; ++a) {
                const int i = fr[a];
                if (du[a] > 0) amax = std::min(amax, (p.ub[i] - xc[i]) / du[a]);
                else if (du[a] < 0) amax = std::min(amax, (p.lb[i] - xc[i]) / du[a]);
            }
            amax = std::max(amax, 0.0);
            for (int a = 0; a < nf; ++a) xbar[fr[a]] = xc[fr[a]] + amax * du[a];
        }
    }
    for (int i = 0; i < NV; ++i) d[i] = xbar[i] - p.x[i];
}

// Minimise n independent problems.  x0, lb, ub are [n][NV]; eval(nb, idx, xt, f, g)
// evaluates the cost and its gradient of problems idx[0..nb) at the points xt[nb][NV]
// into f[nb] and g[nb][NV] and returns 0, or a non-zero status that aborts the run.
// The result of a problem does not depend on which other problems share the batch.
template <int NV, class Eval>
int minimize_batch(int n, const double *x0, const double *lb, const double *ub, int maxits, double pgtol,
                   double factr, Eval &&eval, Result<NV> *out)
{
    const double eps = DBL_EPSILON, ftol = 1e-3;
    const int mem = 15;
    std::vector<Prob<NV>> P(n);
    for (int i = 0; i < n; ++i) {
        for (int v = 0; v < NV; ++v) {
            P[i].lb[v] = lb[i * NV + v];
            P[i].ub[v] = ub[i * NV + v];
            P[i].x[v] = std::min(std::max(x0[i * NV + v], P[i].lb[v]), P[i].ub[v]);
            P[i].xt[v] = P[i].x[v];
        }
    }
    std::vector<int> who;
    std::vector<double> xt, f, g;
    for (int round = 0; round < 64 * std::max(1, maxits); ++round) {
        who.clear();
        xt.clear();
        for (int i = 0; i < n; ++i) {
            if (P[i].state == 2) continue;
            who.push_back(i);
            xt.insert(xt.end(), P[i].xt, P[i].xt + NV);
        }
        if (who.empty()) break;
        f.assign(who.size(), 0.0);
        g.assign(NV * who.size(), 0.0);
        const int st = eval((int)who.size(), who.data(), xt.data(), f.data(), g.data());
        if (st != 0) return st;
        for (size_t b = 0; b < who.size(); ++b) {
            Prob<NV> &p = P[who[b]];
            const double ft = f[b];
            const double *gt = &g[NV * b];
            ++p.nevals;
            if (p.state == 0) {
                p.f = ft;
                for (int v = 0; v < NV; ++v) p.g[v] = gt[v];
            } else {
                // line search: Armijo test at xt = P(x + alpha d)
                if (ft <= p.f + ftol * p.alpha * p.dg0 || p.ls_iter >= 20) {
                    if (ft > p.f) {                      // no decrease at all: stop here
                        p.state = 2;
                        p.converged = 0;
                        continue;
                    }
                    double s[NV], y[NV], sy = 0, yy = 0;
                    for (int v = 0; v < NV; ++v) {
                        s[v] = p.xt[v] - p.x[v];
                        y[v] = gt[v] - p.g[v];
                        sy += s[v] * y[v];
                        yy += y[v] * y[v];
                    }
                    const double fold = p.f;
                    for (int v = 0; v < NV; ++v) { p.x[v] = p.xt[v]; p.g[v] = gt[v]; }
                    p.f = ft;
                    ++p.iter;
                    if (sy > eps * yy) {
                        p.S.insert(p.S.end(), s, s + NV);
                        p.Y.insert(p.Y.end(), y, y + NV);
                        if ((int)p.S.size() > mem * NV) {
                            p.S.erase(p.S.begin(), p.S.begin() + NV);
                            p.Y.erase(p.Y.begin(), p.Y.begin() + NV);
                        }
                        p.theta = yy / sy;
                    }
                    if ((fold - p.f) / std::max(std::max(std::fabs(fold), std::fabs(p.f)), 1.0) <= factr * eps) {
                        p.state = 2;
                        p.converged = 1;
                        continue;
                    }
                } else {
                    // backtrack: safeguarded quadratic interpolation
                    const double a = p.alpha;
                    double an = -p.dg0 * a * a / (2.0 * (ft - p.f - p.dg0 * a));
                    if (!(an > 0.1 * a)) an = 0.1 * a;
                    if (an > 0.5 * a) an = 0.5 * a;
                    p.alpha = an;
                    ++p.ls_iter;
                    for (int v = 0; v < NV; ++v)
                        p.xt[v] = std::min(std::max(p.x[v] + p.alpha * p.d[v], p.lb[v]), p.ub[v]);
                    continue;
                }
            }
            // new iterate: test convergence, compute the next direction
            if (proj_grad_norm(p) <= pgtol) { p.state = 2; p.converged = 1; continue; }
            if (p.iter >= maxits) { p.state = 2; p.converged = 0; continue; }
            direction(p, p.d);
            p.dg0 = 0;
            double dn = 0;
            for (int v = 0; v < NV; ++v) { p.dg0 += p.g[v] * p.d[v]; dn += p.d[v] * p.d[v]; }
            if (!(p.dg0 < 0) || dn == 0) { p.state = 2; p.converged = proj_grad_norm(p) <= 10 * pgtol; continue; }
            // first iteration: the step along the steepest-descent direction scaled to length one
            p.alpha = (p.iter == 0 && p.S.empty()) ? std::min(1.0, 1.0 / std::sqrt(dn)) : 1.0;
            p.ls_iter = 0;
            for (int v = 0; v < NV; ++v) p.xt[v] = std::min(std::max(p.x[v] + p.alpha * p.d[v], p.lb[v]), p.ub[v]);
            p.state = 1;
        }
    }
    for (int i = 0; i < n; ++i) {
        Result<NV> &o = out[i];
        for (int v = 0; v < NV; ++v) o.x[v] = P[i].x[v];
        o.f = P[i].f;
        o.nevals = P[i].nevals;
        o.niter = P[i].iter;
        o.converged = P[i].converged;
    }
    return 0;
}

}  // namespace lbfgsb
}  // namespace pftcc
