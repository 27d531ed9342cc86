// shsrch.cu -- the reference's in-plane shift search (simple_pftcc_shsrch_grad.f90,
// pftcc_shsrch_grad) for many (reference, particle) problems at once.
//
// Every problem runs the reference's control flow as a host state machine; each round
// collects the evaluation every unfinished problem is waiting for and serves them with
// one launch per kind:
//   ROT  the single-rotation correlation and its shift gradient at (irot, shift) --
//        gencorr_grad_for_rot_8 / gencorr_for_rot_8 (k_for_rot, stored |CTF|; for the
//        Euclidean objective gencorr_euclid_grad_for_rot_8, k_euclid_rot);
//   SCAN gencorrs over all rotations at one or more shifts with maxloc (the exact kernel,
//        MODE_BEST: first shift in the problem's list order, lowest rotation on ties --
//        the reference's loops with a strict improvement test), optionally restricted to
//        a rotation mask (minimize_exhaustive's halfrot).
// The optimiser is lbfgsb3.h's L-BFGS-B, with the reference's settings for this search
// (:67-68: line search ftol 1e-1, gtol 1e-3; factr 1e7, pgtol 1e-5 and 15 pairs by
// default, simple_opt_spec.f90:23-24,271).  Each L-BFGS-B run starts from the shift
// rounded to single precision (lbfgsb_minimize sets spec%x_8 = spec%x, :71), stops when its
// evaluations exceed maxits (checked at every new iterate, :120-122), and reports the last
// iterate rounded to single precision.
#include "pftcc_internal.cuh"
#include "lbfgsb3.h"

#include <cmath>
#include <vector>

namespace pftcc {

namespace {

enum Kind { K_NONE = 0, K_ROT = 1, K_SCAN = 2 };

// phases of one problem's control flow
enum Phase {
    P_START,        // MINIMIZE opt_angle: gencorrs at zero shift
    P_COARSE_ANG,   // coarse_search_opt_angle grid
    P_ROT0,         // MINIMIZE fixed angle: the cost at zero shift
    P_COARSE_ROT,   // coarse_search grid at the fixed angle (one ROT per grid point)
    P_LBFGS,        // an L-BFGS-B run (ROT requests; SCAN at each new iterate when opt_angle)
    P_REPICK,       // gencorrs after a run (opt_angle)
    P_EX_GRID,      // minimize_exhaustive: coarse grid
    P_EX_REF1,      //   first refinement ring
    P_EX_REF2,      //   second refinement ring
    P_EX_ROT,       //   the cost at the grid's best before refinement
    P_DONE
};

struct Problem {
    int iref0, slot;
    float lo[2], hi[2];
    Phase phase = P_START;
    int cur = 0;                  // cur_inpl_idx (1-based)
    int cycle = 0;                // L-BFGS-B runs done
    double lowest_overall = 0;    // lowest_cost_overall
    float xs[2] = {0.f, 0.f};     // ospec%x (single precision)
    lbfgsb3::Solver<2> opt;
    int lbfgs_pending_newx = 0;   // a NEW_X awaiting its in-plane re-pick
    int nevals = 0;
    // the request this problem waits for
    Kind kind = K_NONE;
    double rx = 0, ry = 0;        // ROT shift
    int rirot = 0;                // ROT rotation
    std::vector<float> sc;        // SCAN shifts (x, y pairs, in loop order)
    bool masked = false;
    int scan_base = 0;            // index of sc's first shift in the launch's shift list
    // results of the request
    double f = 0, g[2] = {0, 0};
    pftcc_best best{};
    // minimize_exhaustive state
    float step[2] = {0, 0};
    float ex_shift[2] = {0, 0};   // the grid's best shift so far
    float optcc = 0;
    int ex_irot = 0;
    int grid_i = 0;               // coarse_search: next grid point
    double grid_best = 0;
    double grid_xy[2] = {0, 0};
    // output
    pftcc_shsrch_out out{};
};

}  // namespace

int shsrch_batch(pftcc_handle *h, int mode, const pftcc_shsrch_opts &o, int n, const pftcc_shsrch_req *req,
                 const int *slots, pftcc_shsrch_out *out)
{
    const int N = h->g.N;
    const bool eu = h->objfun == PFTCC_OBJFUN_EUCLID;
    lbfgsb3::Options lo;
    lo.ftol = 1e-1;
    lo.gtol = 1e-3;
    std::vector<Problem> pr(n);
    std::vector<uint8_t> masks;
    const bool use_mask = mode == PFTCC_SHSRCH_EXHAUSTIVE && o.halfrot > 0.f;
    if (use_mask) masks.assign((size_t)n * N, 0);
    // get_rot (:624-634) and rotmat2d (simple_math.f90:1550-1559) in single precision
    auto rotate = [&](int irot, float x, float y, float *res) {
        const float a = h->angtab[irot - 1] * 3.14159265f / 180.f;
        const float c = cosf(a), s = sinf(a);
        res[0] = x * c - y * s;     // matmul([x, y], [[c, s], [-s, c]])
        res[1] = x * s + y * c;
    };
    auto scan1 = [&](Problem &p, float x, float y) {
        p.kind = K_SCAN;
        p.sc.assign({x, y});
        p.masked = false;
    };
    auto rot_req = [&](Problem &p, double x, double y, int irot) {
        p.kind = K_ROT;
        p.rx = x;
        p.ry = y;
        p.rirot = irot;
    };
    // an L-BFGS-B run from p.xs (single precision) at p.cur
    auto start_lbfgs = [&](Problem &p) {
        const double x0[2] = {(double)p.xs[0], (double)p.xs[1]};
        const double lb[2] = {(double)p.lo[0], (double)p.lo[1]}, ub[2] = {(double)p.hi[0], (double)p.hi[1]};
        p.opt.start(x0, lb, ub, lo);
        p.phase = P_LBFGS;
        p.lbfgs_pending_newx = 0;
        rot_req(p, p.opt.xt[0], p.opt.xt[1], p.cur);
    };
    // the end of an L-BFGS-B run: x back in single precision, then the caller's next step
    auto end_lbfgs = [&](Problem &p) {
        p.xs[0] = (float)p.opt.x[0];
        p.xs[1] = (float)p.opt.x[1];
        ++p.cycle;
        if (mode == PFTCC_SHSRCH_MINIMIZE && o.opt_angle) {
            p.phase = P_REPICK;
            scan1(p, p.xs[0], p.xs[1]);
            return;
        }
        const float lowest_cost = (float)p.opt.f;
        if (mode == PFTCC_SHSRCH_MINIMIZE) {
            // fixed angle (:328-336)
            if (lowest_cost < p.lowest_overall) {
                p.out.found_better = 1;
                p.out.irot = p.cur;
                p.out.corr = -lowest_cost;
                rotate(p.cur, p.xs[0], p.xs[1], p.out.shift);
            } else {
                p.out.irot = 0;
            }
        } else {
            // minimize_exhaustive (:238-250): the refined or the coarse solution
            float cx = p.ex_shift[0], cy = p.ex_shift[1];
            if (lowest_cost < p.lowest_overall) {
                p.lowest_overall = lowest_cost;
                cx = p.xs[0];
                cy = p.xs[1];
                p.out.found_better = 1;
            }
            p.out.corr = (float)(-p.lowest_overall);
            p.out.irot = p.ex_irot;
            rotate(p.ex_irot, cx, cy, p.out.shift);
        }
        p.phase = P_DONE;
        p.kind = K_NONE;
    };
    // the L-BFGS-B run after an evaluation or a re-pick
    auto drive_lbfgs = [&](Problem &p, lbfgsb3::Task t) {
        while (true) {
            if (t == lbfgsb3::FG) { rot_req(p, p.opt.xt[0], p.opt.xt[1], p.cur); return; }
            if (t == lbfgsb3::NEW_X) {
                if (o.opt_angle) {
                    // opt_callback: the in-plane index re-picked at the new iterate (:139-144)
                    p.lbfgs_pending_newx = 1;
                    scan1(p, (float)p.opt.x[0], (float)p.opt.x[1]);
                    return;
                }
                if (p.opt.nfgv > o.maxits) { end_lbfgs(p); return; }
                t = p.opt.proceed();
                continue;
            }
            end_lbfgs(p);   // converged or stopped
            return;
        }
    };
    // the 5 x 5 grid of coarse_search / coarse_search_opt_angle (:340-389)
    auto coarse_point = [&](const Problem &p, int i, double &x, double &y) {
        const double stepx = (double)(p.hi[0] - p.lo[0]) / 5.0, stepy = (double)(p.hi[1] - p.lo[1]) / 5.0;
        const int ix = i / 5, iy = i % 5;
        x = (double)p.lo[0] + stepx / 2.0 + (double)ix * stepx;
        y = (double)p.lo[1] + stepy / 2.0 + (double)iy * stepy;
    };
    // minimize_exhaustive's rings around the current best: (i, j) in {-1, 0, 1}^2 without (0, 0)
    auto ring = [&](Problem &p, float frac) {
        p.kind = K_SCAN;
        p.masked = use_mask;
        p.sc.clear();
        const float cx = p.ex_shift[0], cy = p.ex_shift[1];
        for (int i = -1; i <= 1; ++i)
            for (int j = -1; j <= 1; ++j) {
                if (i == 0 && j == 0) continue;
                p.sc.push_back(cx + (float)i * p.step[0] / frac);
                p.sc.push_back(cy + (float)j * p.step[1] / frac);
            }
    };

    // ---- initial requests
    for (int i = 0; i < n; ++i) {
        Problem &p = pr[i];
        p.iref0 = req[i].iref - 1;
        p.slot = slots[i];
        p.lo[0] = req[i].lims[0][0]; p.hi[0] = req[i].lims[0][1];
        p.lo[1] = req[i].lims[1][0]; p.hi[1] = req[i].lims[1][1];
        if (mode == PFTCC_SHSRCH_MINIMIZE && o.opt_angle) {
            p.phase = P_START;
            scan1(p, 0.f, 0.f);
        } else if (mode == PFTCC_SHSRCH_MINIMIZE) {
            p.cur = req[i].irot;
            p.phase = P_ROT0;
            rot_req(p, 0.0, 0.0, p.cur);
        } else {
            // minimize_exhaustive (:159-199)
            int irot = req[i].irot <= 0 ? 1 : req[i].irot;    // get_roind(0.) = 1
            p.ex_irot = irot;
            if (use_mask) {
                const float r0 = h->angtab[irot - 1];
                for (int s = 0; s < N; ++s) {
                    float dang = fabsf(h->angtab[s] - r0);
                    if (dang > 180.f) dang = fabsf(dang - 360.f);
                    masks[(size_t)i * N + s] = dang <= o.halfrot;
                }
            }
            const int nsx = std::max(1, (int)floorf((p.hi[0] - p.lo[0]) / 4.f));
            const int nsy = std::max(1, (int)floorf((p.hi[1] - p.lo[1]) / 4.f));
            p.step[0] = (p.hi[0] - p.lo[0]) / (float)(2 * nsx + 1);
            p.step[1] = (p.hi[1] - p.lo[1]) / (float)(2 * nsy + 1);
            p.phase = P_EX_GRID;
            p.kind = K_SCAN;
            p.masked = use_mask;
            for (int a = -nsx; a <= nsx; ++a)
                for (int b = -nsy; b <= nsy; ++b) {
                    p.sc.push_back((float)a * p.step[0]);
                    p.sc.push_back((float)b * p.step[1]);
                }
        }
    }

    // ---- device buffers (small per-call areas, grown on demand)
    std::vector<int> who_rot, who_scan;
    std::vector<RotReqH> rq;
    std::vector<EuclidReq> eq;
    std::vector<Work> work;
    std::vector<Group> groups;
    std::vector<float> shifts;
    std::vector<uint8_t> gmask;
    std::vector<double> o5;
    std::vector<pftcc_best> bres;
    for (int round = 0;; ++round) {
        who_rot.clear();
        who_scan.clear();
        for (int i = 0; i < n; ++i) {
            if (pr[i].kind == K_ROT) who_rot.push_back(i);
            else if (pr[i].kind == K_SCAN) who_scan.push_back(i);
        }
        if (who_rot.empty() && who_scan.empty()) break;
        if (round > 1000000) return set_err(h, PFTCC_ERR_STATE, "shsrch_batch: no progress");
        cudaError_t e;
        // ROT: value and shift gradient per request
        if (!who_rot.empty()) {
            const int nr = (int)who_rot.size();
            const size_t req_bytes = (size_t)nr * (eu ? sizeof(EuclidReq) : sizeof(RotReqH));
            const size_t out_stride = eu ? 3 : 5;
            int st = ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>(req_bytes, 4096), "shsrch requests");
            if (st) return st;
            st = ensure(h, (void **)&h->d_dout, &h->dout_cap, (size_t)nr * out_stride * sizeof(double), "shsrch out");
            if (st) return st;
            if (eu) {
                eq.resize(nr);
                for (int b = 0; b < nr; ++b) {
                    const Problem &p = pr[who_rot[b]];
                    eq[b] = EuclidReq{p.iref0, p.slot, p.rirot, 0, p.rx, p.ry};
                }
                if ((e = cudaMemcpyAsync(h->d_work, eq.data(), req_bytes, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
                    return cuda_err(h, e, "shsrch upload");
                if ((e = launch_euclid_rot(h, reinterpret_cast<const EuclidReq *>(h->d_work), nr, 1, 0, h->d_dout,
                                           nullptr)) != cudaSuccess)
                    return cuda_err(h, e, "shsrch euclid");
            } else {
                rq.resize(nr);
                for (int b = 0; b < nr; ++b) {
                    const Problem &p = pr[who_rot[b]];
                    rq[b] = RotReqH{p.iref0, p.slot, p.rirot, 0, p.rx, p.ry, 0.0};
                }
                if ((e = cudaMemcpyAsync(h->d_work, rq.data(), req_bytes, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess)
                    return cuda_err(h, e, "shsrch upload");
                if ((e = launch_rot_reqs(h, h->d_work, nr, h->d_dout)) != cudaSuccess) return cuda_err(h, e, "shsrch rot");
            }
            o5.resize((size_t)nr * out_stride);
            if ((e = cudaMemcpyAsync(o5.data(), h->d_dout, o5.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                     h->stream)) != cudaSuccess)
                return cuda_err(h, e, "shsrch download");
            if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "shsrch rot");
            for (int b = 0; b < nr; ++b) {
                Problem &p = pr[who_rot[b]];
                p.f = o5[out_stride * b];
                p.g[0] = o5[out_stride * b + 1];
                p.g[1] = o5[out_stride * b + 2];
            }
        }
        // SCAN: maxloc of gencorrs over the problem's shift list
        if (!who_scan.empty()) {
            const int ng = (int)who_scan.size();
            work.clear();
            groups.clear();
            shifts.clear();
            bool any_mask = false;
            for (int b = 0; b < ng; ++b) {
                Problem &p = pr[who_scan[b]];
                const int ns = (int)p.sc.size() / 2;
                p.scan_base = (int)(shifts.size() / 2);
                groups.push_back(Group{p.slot, (int)work.size(), ns, b});
                for (int s = 0; s < ns; ++s) work.push_back(Work{p.iref0, (int)(shifts.size() / 2) + s, 0});
                shifts.insert(shifts.end(), p.sc.begin(), p.sc.end());
                any_mask |= p.masked;
            }
            if (any_mask) {
                gmask.assign((size_t)ng * N, 1);
                for (int b = 0; b < ng; ++b)
                    if (pr[who_scan[b]].masked)
                        std::copy(masks.begin() + (size_t)who_scan[b] * N, masks.begin() + (size_t)(who_scan[b] + 1) * N,
                                  gmask.begin() + (size_t)b * N);
            }
            const size_t wbytes = work.size() * sizeof(Work), gbytes = groups.size() * sizeof(Group);
            const size_t sbytes = shifts.size() * sizeof(float), mbytes = any_mask ? gmask.size() : 0;
            int st = ensure(h, (void **)&h->d_work, &h->work_cap, std::max<size_t>(wbytes, 4096), "shsrch work");
            if (st) return st;
            st = ensure(h, (void **)&h->d_groups, &h->group_cap, std::max<size_t>(gbytes + mbytes, 256), "shsrch groups");
            if (st) return st;
            st = ensure(h, (void **)&h->d_shifts, &h->shifts_cap, std::max<size_t>(sbytes, 64), "shsrch shifts");
            if (st) return st;
            st = ensure(h, (void **)&h->d_best, &h->best_cap, (size_t)ng * sizeof(pftcc_best), "shsrch best");
            if (st) return st;
            uint8_t *dmask = any_mask ? reinterpret_cast<uint8_t *>(h->d_groups) + gbytes : nullptr;
            if ((e = cudaMemcpyAsync(h->d_work, work.data(), wbytes, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(h->d_groups, groups.data(), gbytes, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
                (e = cudaMemcpyAsync(h->d_shifts, shifts.data(), sbytes, cudaMemcpyHostToDevice, h->stream)) != cudaSuccess ||
                (any_mask && (e = cudaMemcpyAsync(dmask, gmask.data(), mbytes, cudaMemcpyHostToDevice, h->stream)) !=
                                 cudaSuccess))
                return cuda_err(h, e, "shsrch upload");
            if ((e = launch_exact(h, h->d_groups, ng, h->d_work, h->d_shifts, MODE_BEST, exact_frame(h), 1, nullptr,
                                  h->d_best, dmask)) != cudaSuccess)
                return cuda_err(h, e, "shsrch gencorrs");
            bres.resize(ng);
            if ((e = cudaMemcpyAsync(bres.data(), h->d_best, (size_t)ng * sizeof(pftcc_best), cudaMemcpyDeviceToHost,
                                     h->stream)) != cudaSuccess)
                return cuda_err(h, e, "shsrch download");
            if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "shsrch gencorrs");
            for (int b = 0; b < ng; ++b) pr[who_scan[b]].best = bres[b];
        }
        // advance every problem that was served
        auto advance = [&](Problem &p) {
            const Kind k = p.kind;
            p.kind = K_NONE;
            const float *sc = p.sc.data();
            const pftcc_best &bb = p.best;
            const int sloc = bb.ishift - p.scan_base;    // the winning shift's position in sc
            switch (p.phase) {
            case P_START:            // :268-271
                p.cur = bb.irot;
                p.lowest_overall = -(double)bb.corr;
                if (o.coarse_init) {
                    p.phase = P_COARSE_ANG;
                    p.kind = K_SCAN;
                    p.masked = false;
                    p.sc.clear();
                    for (int i = 0; i < 25; ++i) {
                        double x, y;
                        coarse_point(p, i, x, y);
                        p.sc.push_back((float)x);
                        p.sc.push_back((float)y);
                    }
                    return;
                }
                p.xs[0] = p.xs[1] = 0.f;
                start_lbfgs(p);
                return;
            case P_COARSE_ANG:       // :272-279, coarse_search_opt_angle :364-389
                if (bb.irot > 0) {
                    double x, y;
                    coarse_point(p, sloc, x, y);
                    p.xs[0] = (float)x;
                    p.xs[1] = (float)y;
                    p.cur = bb.irot;
                }
                start_lbfgs(p);
                return;
            case P_ROT0:             // :301-302
                p.lowest_overall = -p.f;
                if (o.coarse_init) {
                    p.phase = P_COARSE_ROT;
                    p.grid_i = 0;
                    p.grid_best = HUGE_VAL;
                    p.grid_xy[0] = p.grid_xy[1] = 0.0;
                    double x, y;
                    coarse_point(p, 0, x, y);
                    rot_req(p, x, y, p.cur);
                    return;
                }
                p.xs[0] = p.xs[1] = 0.f;
                start_lbfgs(p);
                return;
            case P_COARSE_ROT: {     // coarse_search :340-362, then :308-314
                double x, y;
                coarse_point(p, p.grid_i, x, y);
                const double cost = -p.f;
                if (cost < p.grid_best) { p.grid_best = cost; p.grid_xy[0] = x; p.grid_xy[1] = y; }
                if (++p.grid_i < 25) {
                    coarse_point(p, p.grid_i, x, y);
                    rot_req(p, x, y, p.cur);
                    return;
                }
                p.xs[0] = p.xs[1] = 0.f;
                if (p.grid_best < p.lowest_overall) {
                    p.lowest_overall = p.grid_best;
                    p.xs[0] = (float)p.grid_xy[0];
                    p.xs[1] = (float)p.grid_xy[1];
                }
                start_lbfgs(p);
                return;
            }
            case P_LBFGS: {
                if (k == K_SCAN) {   // the re-pick at a new iterate
                    p.cur = bb.irot;
                    p.lbfgs_pending_newx = 0;
                    if (p.opt.nfgv > o.maxits) { end_lbfgs(p); return; }
                    drive_lbfgs(p, p.opt.proceed());
                    return;
                }
                ++p.nevals;
                const double gg[2] = {-p.g[0], -p.g[1]};
                drive_lbfgs(p, p.opt.evaluated(-p.f, gg));
                return;
            }
            case P_REPICK: {         // :283-298
                const int loc = bb.irot;
                if (loc != p.cur && p.cycle < o.max_evals) {
                    p.cur = loc;
                    start_lbfgs(p);
                    return;
                }
                p.cur = loc;
                const float lowest_cost = -bb.corr;
                if ((double)lowest_cost < p.lowest_overall) {
                    p.out.found_better = 1;
                    p.out.irot = p.cur;
                    p.out.corr = -lowest_cost;
                    rotate(p.cur, p.xs[0], p.xs[1], p.out.shift);
                } else {
                    p.out.irot = 0;
                }
                p.phase = P_DONE;
                return;
            }
            case P_EX_GRID:          // :183-199
            case P_EX_REF1:          // :200-215
            case P_EX_REF2: {        // :216-231
                if (bb.irot > 0) {
                    const bool first = p.phase == P_EX_GRID;
                    if (first || bb.corr > p.optcc) {
                        p.optcc = bb.corr;
                        p.ex_irot = bb.irot;
                        p.ex_shift[0] = sc[2 * sloc];
                        p.ex_shift[1] = sc[2 * sloc + 1];
                    }
                }
                if (p.phase == P_EX_GRID) { p.phase = P_EX_REF1; ring(p, 2.f); return; }
                if (p.phase == P_EX_REF1) { p.phase = P_EX_REF2; ring(p, 4.f); return; }
                // :232-237: the cost at the grid's best, then the refinement
                p.cur = p.ex_irot;
                p.xs[0] = p.ex_shift[0];
                p.xs[1] = p.ex_shift[1];
                p.phase = P_EX_ROT;
                rot_req(p, p.xs[0], p.xs[1], p.cur);
                return;
            }
            case P_EX_ROT:
                p.lowest_overall = (double)(-(float)p.f);   // -gencorr_for_rot (single precision)
                start_lbfgs(p);
                return;
            default:
                return;
            }
        };
        for (int i : who_rot) advance(pr[i]);
        for (int i : who_scan) advance(pr[i]);
    }
    for (int i = 0; i < n; ++i) {
        Problem &p = pr[i];
        p.out.nevals = p.nevals;
        p.out.ncycles = p.cycle;
        out[i] = p.out;
    }
    return PFTCC_OK;
}

}  // namespace pftcc
