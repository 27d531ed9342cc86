// lbfgsb3.h -- one bound-constrained limited-memory BFGS problem in reverse communication,
// stepping the way the reference's optimiser does (simple_opt_lbfgsb.f90, L-BFGS-B 3.0:
// setulb/mainlb driven by task strings 'FG' and 'NEW_X', lbfgsb_minimize :103-129), host
// C++ with no CUDA dependency.  Written from the published algorithms:
//   * Byrd, Lu, Nocedal & Zhu (1995), "A limited memory algorithm for bound constrained
//     optimization": B = the BFGS update of theta*I by the stored pairs, the generalised
//     Cauchy point along the projected steepest-descent path, the subspace minimiser over
//     the free variables by the direct primal method;
//   * Morales & Nocedal (2011), "Remark on algorithm 778": the subspace step is first
//     projected onto the box and kept when that is a descent direction, else truncated;
//   * More & Thuente (1994), "Line search algorithms with guaranteed sufficient decrease":
//     the safeguarded cubic/quadratic interpolation search on the strong Wolfe conditions
//     with parameters ftol, gtol, xtol.
// The driver rules follow the reference's mainlb: termination when the projected gradient's
// max-norm <= pgtol or (f_old - f) <= factr * eps * max(|f_old|, |f|, 1); the first step of
// a problem with every variable bounded is 1 with the step bounded by 1; a line search that
// fails or needs 20 evaluations restarts from steepest descent once the memory is cleared,
// and ends the run when the memory is already empty; a pair is stored only when its
// curvature y.s exceeds eps * (-g_old.d) * stp.  The caller evaluates the cost where task
// == FG and may change its cost function where task == NEW_X (the reference's opt_callback
// re-picks the in-plane rotation there, simple_pftcc_shsrch_grad.f90:139-144).
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

namespace pftcc {
namespace lbfgsb3 {

// ---- More & Thuente line search (reverse communication) ----------------------------------
struct LineSearch {
    double ftol = 1e-3, gtol = 0.9, xtol = 0.1, stpmin = 0.0, stpmax = 1e10;
    bool brackt = false;
    int stage = 1;
    double finit = 0, ginit = 0, gtest = 0, width = 0, width1 = 0;
    double stx = 0, fx = 0, gx = 0, sty = 0, fy = 0, gy = 0, stmin = 0, stmax = 0;

    // f, g: value and directional derivative at step 0; stp the first trial step.
    // false when no descent is possible (g >= 0) or the first step is outside [stpmin, stpmax]
    bool begin(double f, double g, double stp)
    {
        if (!(g < 0.0) || stp < stpmin || stp > stpmax) return false;
        brackt = false;
        stage = 1;
        finit = f;
        ginit = g;
        gtest = ftol * ginit;
        width = stpmax - stpmin;
        width1 = 2.0 * width;
        stx = 0.0; fx = finit; gx = ginit;
        sty = 0.0; fy = finit; gy = ginit;
        stmin = 0.0;
        stmax = stp + 4.0 * stp;
        return true;
    }

    // safeguarded step of the interval update (the four cases of More & Thuente, section 4)
    void step(double &sx, double &fxv, double &dx, double &sy, double &fyv, double &dy, double &stp, double fp, double dp,
              double lo, double hi)
    {
        const double sgnd = dp * (dx / std::fabs(dx));
        double stpf;
        if (fp > fxv) {
            // higher value: the minimum is bracketed; cubic or the midpoint towards the quadratic
            const double theta = 3.0 * (fxv - fp) / (stp - sx) + dx + dp;
            const double s = std::max(std::fabs(theta), std::max(std::fabs(dx), std::fabs(dp)));
            double gamma = s * std::sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
            if (stp < sx) gamma = -gamma;
            const double p = (gamma - dx) + theta, q = ((gamma - dx) + gamma) + dp;
            const double stpc = sx + (p / q) * (stp - sx);
            const double stpq = sx + ((dx / ((fxv - fp) / (stp - sx) + dx)) / 2.0) * (stp - sx);
            stpf = std::fabs(stpc - sx) < std::fabs(stpq - sx) ? stpc : stpc + (stpq - stpc) / 2.0;
            brackt = true;
        } else if (sgnd < 0.0) {
            // derivatives of opposite sign: bracketed; the step farther from stp of cubic and secant
            const double theta = 3.0 * (fxv - fp) / (stp - sx) + dx + dp;
            const double s = std::max(std::fabs(theta), std::max(std::fabs(dx), std::fabs(dp)));
            double gamma = s * std::sqrt((theta / s) * (theta / s) - (dx / s) * (dp / s));
            if (stp > sx) gamma = -gamma;
            const double p = (gamma - dp) + theta, q = ((gamma - dp) + gamma) + dx;
            const double stpc = stp + (p / q) * (sx - stp);
            const double stpq = stp + (dp / (dp - dx)) * (sx - stp);
            stpf = std::fabs(stpc - stp) > std::fabs(stpq - stp) ? stpc : stpq;
            brackt = true;
        } else if (std::fabs(dp) < std::fabs(dx)) {
            // lower value, same-sign derivative decreasing in magnitude
            const double theta = 3.0 * (fxv - fp) / (stp - sx) + dx + dp;
            const double s = std::max(std::fabs(theta), std::max(std::fabs(dx), std::fabs(dp)));
            double gamma = s * std::sqrt(std::max(0.0, (theta / s) * (theta / s) - (dx / s) * (dp / s)));
            if (stp > sx) gamma = -gamma;
            const double p = (gamma - dp) + theta, q = (gamma + (dx - dp)) + gamma;
            const double r = p / q;
            double stpc;
            if (r < 0.0 && gamma != 0.0) stpc = stp + r * (sx - stp);
            else stpc = stp > sx ? hi : lo;
            const double stpq = stp + (dp / (dp - dx)) * (sx - stp);
            if (brackt) {
                stpf = std::fabs(stpc - stp) < std::fabs(stpq - stp) ? stpc : stpq;
                stpf = stp > sx ? std::min(stp + 0.66 * (sy - stp), stpf) : std::max(stp + 0.66 * (sy - stp), stpf);
            } else {
                stpf = std::fabs(stpc - stp) > std::fabs(stpq - stp) ? stpc : stpq;
                stpf = std::max(lo, std::min(hi, stpf));
            }
        } else {
            // lower value, derivative not decreasing: cubic towards the other end, or the bound
            if (brackt) {
                const double theta = 3.0 * (fp - fyv) / (sy - stp) + dy + dp;
                const double s = std::max(std::fabs(theta), std::max(std::fabs(dy), std::fabs(dp)));
                double gamma = s * std::sqrt((theta / s) * (theta / s) - (dy / s) * (dp / s));
                if (stp > sy) gamma = -gamma;
                const double p = (gamma - dp) + theta, q = ((gamma - dp) + gamma) + dy;
                stpf = stp + (p / q) * (sy - stp);
            } else {
                stpf = stp > sx ? hi : lo;
            }
        }
        // the new interval
        if (fp > fxv) {
            sy = stp; fyv = fp; dy = dp;
        } else {
            if (sgnd < 0.0) { sy = sx; fyv = fxv; dy = dx; }
            sx = stp; fxv = fp; dx = dp;
        }
        stp = stpf;
    }

    // f, g at the trial step stp: 0 = evaluate again at the updated stp, 1 = the strong Wolfe
    // conditions hold, 2 = stop with a warning (interval too small or a bound reached; stp
    // is then the step to accept)
    int next(double f, double g, double &stp)
    {
        const double ftest = finit + stp * gtest;
        if (stage == 1 && f <= ftest && g >= 0.0) stage = 2;
        if (brackt && (stp <= stmin || stp >= stmax)) return 2;
        if (brackt && stmax - stmin <= xtol * stmax) return 2;
        if (stp == stpmax && f <= ftest && g <= gtest) return 2;
        if (stp == stpmin && (f > ftest || g >= gtest)) return 2;
        if (f <= ftest && std::fabs(g) <= gtol * (-ginit)) return 1;
        if (stage == 1 && f <= fx && f > ftest) {
            // the modified function psi(stp) = f - stp * gtest until a sufficient decrease is seen
            double fm = f - stp * gtest, fxm = fx - stx * gtest, fym = fy - sty * gtest;
            double gm = g - gtest, gxm = gx - gtest, gym = gy - gtest;
            step(stx, fxm, gxm, sty, fym, gym, stp, fm, gm, stmin, stmax);
            fx = fxm + stx * gtest; fy = fym + sty * gtest;
            gx = gxm + gtest; gy = gym + gtest;
        } else {
            step(stx, fx, gx, sty, fy, gy, stp, f, g, stmin, stmax);
        }
        if (brackt) {
            if (std::fabs(sty - stx) >= 0.66 * width1) stp = stx + 0.5 * (sty - stx);
            width1 = width;
            width = std::fabs(sty - stx);
            stmin = std::min(stx, sty);
            stmax = std::max(stx, sty);
        } else {
            stmin = stp + 1.1 * (stp - stx);
            stmax = stp + 4.0 * (stp - stx);
        }
        stp = std::max(stp, stpmin);
        stp = std::min(stp, stpmax);
        if ((brackt && (stp <= stmin || stp >= stmax)) || (brackt && stmax - stmin <= xtol * stmax)) stp = stx;
        return 0;
    }
};

struct Options {
    double factr = 1e7, pgtol = 1e-5;           // termination (simple_opt_spec.f90:23-24)
    double ftol = 1e-3, gtol = 0.9, xtol = 0.1; // line search
    int m = 15;                                  // stored pairs (simple_opt_spec.f90:271)
};

enum Task { FG = 0, NEW_X = 1, CONVERGED = 2, ABNORMAL = 3 };

template <int NV>
struct Solver {
    Options o;
    double lb[NV], ub[NV];
    double x[NV], f = 0, g[NV];          // current iterate
    double xt[NV];                       // the point to evaluate while task == FG
    double d[NV], z[NV], t[NV], r[NV];   // direction, subspace point, saved iterate and gradient
    double fold = 0, gdold = 0, stp = 1, stpmx = 1, sbgnrm = 0;
    std::vector<double> S, Y;
    double theta = 1.0;
    int iter = 0, nfgv = 0, ifun = 0, phase = 0;
    Task task = FG;
    LineSearch ls;

    void start(const double *x0, const double *lo, const double *hi, const Options &opt)
    {
        o = opt;
        for (int i = 0; i < NV; ++i) {
            lb[i] = lo[i];
            ub[i] = hi[i];
            x[i] = std::min(std::max(x0[i], lb[i]), ub[i]);
            xt[i] = x[i];
        }
        S.clear(); Y.clear();
        theta = 1.0;
        iter = nfgv = ifun = 0;
        phase = 0;
        task = FG;
    }

    double proj_grad_norm() const
    {
        double m = 0;
        for (int i = 0; i < NV; ++i) {
            double gi = g[i];
            if (gi < 0) gi = std::max(x[i] - ub[i], gi);
            else gi = std::min(x[i] - lb[i], gi);
            m = std::max(m, std::fabs(gi));
        }
        return m;
    }

    // B = theta I updated by the stored pairs, oldest first
    void form_B(double B[NV][NV]) const
    {
        for (int i = 0; i < NV; ++i)
            for (int j = 0; j < NV; ++j) B[i][j] = i == j ? theta : 0.0;
        const int np = (int)S.size() / NV;
        for (int q = 0; q < np; ++q) {
            const double *s = &S[(size_t)q * NV], *y = &Y[(size_t)q * NV];
            double Bs[NV], sBs = 0, ys = 0;
            for (int i = 0; i < NV; ++i) {
                Bs[i] = 0;
                for (int j = 0; j < NV; ++j) Bs[i] += B[i][j] * s[j];
                ys += y[i] * s[i];
            }
            for (int i = 0; i < NV; ++i) sBs += s[i] * Bs[i];
            if (sBs <= 0 || ys <= 0) continue;
            for (int i = 0; i < NV; ++i)
                for (int j = 0; j < NV; ++j) B[i][j] += -Bs[i] * Bs[j] / sBs + y[i] * y[j] / ys;
        }
    }

    // generalised Cauchy point, then the subspace step (projected when that descends, else
    // truncated at the box); the result in z
    void cauchy_subspace()
    {
        double B[NV][NV];
        form_B(B);
        double tb[NV];
        for (int i = 0; i < NV; ++i) {
            if (g[i] < 0) tb[i] = (x[i] - ub[i]) / g[i];
            else if (g[i] > 0) tb[i] = (x[i] - lb[i]) / g[i];
            else tb[i] = DBL_MAX;
            if (tb[i] < 0) tb[i] = 0;
        }
        int order[NV];
        for (int i = 0; i < NV; ++i) order[i] = i;
        std::sort(order, order + NV, [&](int a, int b) { return tb[a] < tb[b]; });
        double xc[NV], dir[NV];
        for (int i = 0; i < NV; ++i) {
            xc[i] = x[i];
            dir[i] = tb[i] == 0 ? 0.0 : -g[i];
        }
        double tprev = 0;
        for (int seg = 0; seg <= NV; ++seg) {
            const double tnext = seg < NV ? tb[order[seg]] : DBL_MAX;
            if (seg < NV && tnext <= tprev) { dir[order[seg]] = 0; continue; }
            double zz[NV], Bd[NV];
            for (int i = 0; i < NV; ++i) {
                zz[i] = xc[i] - x[i];
                Bd[i] = 0;
                for (int j = 0; j < NV; ++j) Bd[i] += B[i][j] * dir[j];
            }
            double f1 = 0, f2 = 0;
            for (int i = 0; i < NV; ++i) { f1 += g[i] * dir[i] + zz[i] * Bd[i]; f2 += dir[i] * Bd[i]; }
            if (f1 >= 0) break;
            const double dt = f2 > 0 ? -f1 / f2 : DBL_MAX;
            if (tprev + dt < tnext) {
                for (int i = 0; i < NV; ++i) xc[i] += dt * dir[i];
                break;
            }
            if (seg == NV) break;
            const double stepv = tnext - tprev;
            for (int i = 0; i < NV; ++i) xc[i] += stepv * dir[i];
            const int v = order[seg];
            xc[v] = dir[v] < 0 ? lb[v] : ub[v];
            dir[v] = 0;
            tprev = tnext;
        }
        for (int i = 0; i < NV; ++i) { xc[i] = std::min(std::max(xc[i], lb[i]), ub[i]); z[i] = xc[i]; }
        int fr[NV], nf = 0;
        for (int i = 0; i < NV; ++i)
            if (xc[i] > lb[i] && xc[i] < ub[i]) fr[nf++] = i;
        if (nf == 0 || S.empty()) return;      // the first iteration stops at the Cauchy point
        double rr[NV];
        for (int i = 0; i < NV; ++i) {
            rr[i] = g[i];
            for (int j = 0; j < NV; ++j) rr[i] += B[i][j] * (xc[j] - x[j]);
        }
        double A[NV][NV + 1];
        for (int a = 0; a < nf; ++a) {
            for (int b = 0; b < nf; ++b) A[a][b] = B[fr[a]][fr[b]];
            A[a][nf] = -rr[fr[a]];
        }
        for (int c = 0; c < nf; ++c) {
            int piv = c;
            for (int a = c + 1; a < nf; ++a)
                if (std::fabs(A[a][c]) > std::fabs(A[piv][c])) piv = a;
            if (std::fabs(A[piv][c]) < 1e-300) return;
            for (int b = 0; b <= nf; ++b) std::swap(A[c][b], A[piv][b]);
            for (int a = 0; a < nf; ++a)
                if (a != c) {
                    const double fct = A[a][c] / A[c][c];
                    for (int b = c; b <= nf; ++b) A[a][b] -= fct * A[c][b];
                }
        }
        double du[NV];
        for (int a = 0; a < nf; ++a) du[a] = A[a][nf] / A[a][a];
        // the projected subspace point, kept unless a bound is hit and it ascends
        double xp[NV];
        bool hit = false;
        for (int i = 0; i < NV; ++i) xp[i] = z[i];
        for (int a = 0; a < nf; ++a) {
            const int i = fr[a];
            xp[i] = std::min(std::max(z[i] + du[a], lb[i]), ub[i]);
            if (xp[i] == lb[i] || xp[i] == ub[i]) hit = true;
        }
        if (!hit) { for (int i = 0; i < NV; ++i) z[i] = xp[i]; return; }
        double ddp = 0;
        for (int i = 0; i < NV; ++i) ddp += (xp[i] - x[i]) * g[i];
        if (!(ddp > 0)) { for (int i = 0; i < NV; ++i) z[i] = xp[i]; return; }
        // truncated step: the largest alpha <= 1 keeping z + alpha du in the box
        double alpha = 1.0;
        int ibd = -1;
        for (int a = 0; a < nf; ++a) {
            const int i = fr[a];
            double tmp = alpha;
            if (du[a] < 0) {
                const double t2 = lb[i] - z[i];
                if (t2 >= 0) tmp = 0;
                else if (du[a] * alpha < t2) tmp = t2 / du[a];
            } else if (du[a] > 0) {
                const double t2 = ub[i] - z[i];
                if (t2 <= 0) tmp = 0;
                else if (du[a] * alpha > t2) tmp = t2 / du[a];
            }
            if (tmp < alpha) { alpha = tmp; ibd = a; }
        }
        if (alpha < 1.0 && ibd >= 0) {
            const int i = fr[ibd];
            z[i] = du[ibd] > 0 ? ub[i] : lb[i];
            du[ibd] = 0;
        }
        for (int a = 0; a < nf; ++a) z[fr[a]] += alpha * du[a];
    }

    // a new search direction and the first trial point of its line search (task FG), or
    // the end of the run
    Task begin_iteration()
    {
        for (int attempt = 0; attempt < 2; ++attempt) {
            cauchy_subspace();
            double dtd = 0, gd = 0;
            for (int i = 0; i < NV; ++i) { d[i] = z[i] - x[i]; dtd += d[i] * d[i]; gd += g[i] * d[i]; }
            // the longest step that keeps x + stp d in the box: 1 on the first iteration
            stpmx = 1e10;
            if (iter == 0) {
                stpmx = 1.0;
            } else {
                for (int i = 0; i < NV; ++i) {
                    if (d[i] < 0) {
                        const double a2 = lb[i] - x[i];
                        if (a2 >= 0) stpmx = 0;
                        else if (d[i] * stpmx < a2) stpmx = a2 / d[i];
                    } else if (d[i] > 0) {
                        const double a2 = ub[i] - x[i];
                        if (a2 <= 0) stpmx = 0;
                        else if (d[i] * stpmx > a2) stpmx = a2 / d[i];
                    }
                }
            }
            stp = 1.0;   // every variable is bounded: the first step is 1 (not 1 / |d|)
            for (int i = 0; i < NV; ++i) { t[i] = x[i]; r[i] = g[i]; }
            fold = f;
            ifun = 0;
            gdold = gd;
            ls.ftol = o.ftol; ls.gtol = o.gtol; ls.xtol = o.xtol; ls.stpmin = 0.0; ls.stpmax = stpmx;
            if (dtd > 0 && ls.begin(f, gd, stp)) {
                for (int i = 0; i < NV; ++i) xt[i] = z[i];     // stp == 1: the subspace point itself
                phase = 1;
                return task = FG;
            }
            // no descent along d: restart from steepest descent once, else stop
            if (S.empty()) return task = ABNORMAL;
            S.clear(); Y.clear();
            theta = 1.0;
        }
        return task = ABNORMAL;
    }

    // the cost and its gradient at xt (task FG)
    Task evaluated(double fv, const double *gv)
    {
        ++nfgv;
        if (phase == 0) {
            f = fv;
            for (int i = 0; i < NV; ++i) g[i] = gv[i];
            sbgnrm = proj_grad_norm();
            if (sbgnrm <= o.pgtol) return task = CONVERGED;
            return begin_iteration();
        }
        ++ifun;
        double gd = 0;
        for (int i = 0; i < NV; ++i) gd += gv[i] * d[i];
        double s = stp;
        const int st = ls.next(fv, gd, s);
        if (st == 0 && ifun < 20) {
            stp = s;
            for (int i = 0; i < NV; ++i) xt[i] = stp == 1.0 ? z[i] : stp * d[i] + t[i];
            return task = FG;
        }
        if (st == 0) {
            // the line search needed too many evaluations: back to the iterate it started from
            for (int i = 0; i < NV; ++i) { x[i] = t[i]; g[i] = r[i]; }
            f = fold;
            if (S.empty()) return task = ABNORMAL;
            S.clear(); Y.clear();
            theta = 1.0;
            return begin_iteration();
        }
        // accepted: the new iterate
        for (int i = 0; i < NV; ++i) { x[i] = xt[i]; g[i] = gv[i]; }
        f = fv;
        ++iter;
        sbgnrm = proj_grad_norm();
        gdnew = gd;
        return task = NEW_X;
    }

    // after NEW_X: termination tests, the update, the next direction
    Task proceed()
    {
        if (sbgnrm <= o.pgtol) return task = CONVERGED;
        const double ddum = std::max(std::max(std::fabs(fold), std::fabs(f)), 1.0);
        if (fold - f <= o.factr * DBL_EPSILON * ddum) return task = CONVERGED;
        double s[NV], y[NV], rr = 0;
        for (int i = 0; i < NV; ++i) {
            s[i] = stp * d[i];
            y[i] = g[i] - r[i];
            rr += y[i] * y[i];
        }
        const double dr = (gdnew - gdold) * stp;
        if (dr > DBL_EPSILON * (-gdold * stp)) {
            S.insert(S.end(), s, s + NV);
            Y.insert(Y.end(), y, y + NV);
            if ((int)S.size() > o.m * NV) {
                S.erase(S.begin(), S.begin() + NV);
                Y.erase(Y.begin(), Y.begin() + NV);
            }
            theta = rr / dr;
        }
        return begin_iteration();
    }

    double gdnew = 0;
};

}  // namespace lbfgsb3
}  // namespace pftcc
