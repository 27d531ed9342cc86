"""Precision of every GPU path at config-1 scale against the CPU FP64 oracle, beside the
error of the reference's own FP32 FFT loop on the same correlations.

Workload: the config-1 geometry (box 128, 360 rotations, shells 2..40, 500 references,
the 9 x 9 shift grid of 0.5 px) with the configs' astigmatic CTFs; a sample of particles.
Every correlation (particle x reference x shift x rotation) of each path is compared with
the FP64 oracle (oracle.iter_allcorrs64, pinned against the direct sums in
tests/test_oracle.py):

  reference frame (the drop-in gencorrs_cc_2):  the exact kernel, and beside it the
      reference's FP32 FFT loop (calc_corrs_over_k :1132-1162, restated in the oracle);
  particle frame (the m-domain search):  the exact kernel, FP32 m-domain, raw BF16 hi+lo.

Errors, for every path and for the reference's loop:
  * max / mean |dcc|;
  * elementwise relative error |dcc| / max(|cc|, 1e-3);
  * normwise relative error: per correlation function (one particle, reference and
    shift over all rotations) max_rot |dcc| / max_rot |cc|, its maximum and mean.
The exact kernel (the drop-in gencorrs, direct sums) is gated elementwise at max(1e-5, the
reference loop's own elementwise error).  The m-domain paths reduce over the shells in
the frequency domain, so their rounding is spread evenly over the rotations of a
correlation function (an FFT's error is relative to the function's norm), while the
reference's loop adds the shells' correlation functions rotation by rotation; the
m-domain paths are therefore gated normwise at max(1e-5 (FP32) or 1e-4 (BF16 split), the
reference loop's own normwise error), and their elementwise errors are reported beside.
Best (ref, shift, rot) per particle: identical to the oracle's, except where the oracle's
own values at the two poses differ by less than the path's gate relative to the best.
The searches (BF16 split with the FP32 re-score of the top 8, in both frames) are held to
the same rule, and their reported correlations to the elementwise FP32 gate.  Beside
them the deviation of the particle-frame objective from the reference's at the configs'
astigmatism is measured (it is reported, not gated).

PFTCC_PREC_PTCLS / PFTCC_PREC_REF_PTCLS set the two sample sizes; PFTCC_PRECISION_REPORT
names a file that receives the measured figures as JSON."""
import json
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NPT_PTCL = int(os.environ.get("PFTCC_PREC_PTCLS", "8"))
NPT_REF = int(os.environ.get("PFTCC_PREC_REF_PTCLS", "2"))
REPORT = os.environ.get("PFTCC_PRECISION_REPORT")
FLOOR = 1e-3
TOL = {"exact": 1e-5, "fp32": 1e-5, "bf16x3": 1e-4}


class Errors:
    """running error statistics of one path against the FP64 oracle, plus the oracle's
    value at the path's best pose per particle"""

    def __init__(self, got):
        self.got = got                                         # (np, nrefs, ns, N) float32
        npt = got.shape[0]
        flat = got.reshape(npt, -1)
        self.pick = flat.argmax(1)                              # the path's best pose per particle
        self.max_abs = self.sum_abs = self.max_rel = self.sum_rel = 0.0
        self.max_nrm = self.sum_nrm = 0.0
        self.count = self.nfun = 0
        self.oracle_at_pick = np.full(npt, np.nan)

    def add(self, r0, r1, want):
        g = self.got[:, r0:r1].astype(np.float64)
        d = np.abs(g - want)
        rel = d / np.maximum(np.abs(want), FLOOR)
        self.max_abs = max(self.max_abs, float(d.max()))
        self.sum_abs += float(d.sum())
        self.max_rel = max(self.max_rel, float(rel.max()))
        self.sum_rel += float(rel.sum())
        self.count += d.size
        nrm = d.max(-1) / np.abs(want).max(-1)
        self.max_nrm = max(self.max_nrm, float(nrm.max()))
        self.sum_nrm += float(nrm.sum())
        self.nfun += nrm.size
        per_ref = int(np.prod(self.got.shape[2:]))
        for p, k in enumerate(self.pick):
            if r0 * per_ref <= k < r1 * per_ref:
                self.oracle_at_pick[p] = want[p].reshape(-1)[k - r0 * per_ref]

    def summary(self):
        return {"max_abs_dcc": self.max_abs, "mean_abs_dcc": self.sum_abs / max(1, self.count),
                "max_rel_err_floor1e-3": self.max_rel, "mean_rel_err_floor1e-3": self.sum_rel / max(1, self.count),
                "max_normwise_rel_err": self.max_nrm, "mean_normwise_rel_err": self.sum_nrm / max(1, self.nfun),
                "correlations": self.count}


class Best:
    """the oracle's best pose and value per particle"""

    def __init__(self, npt, per_ref):
        self.val = np.full(npt, -np.inf)
        self.idx = np.zeros(npt, np.int64)
        self.per_ref = per_ref

    def add(self, r0, want):
        flat = want.reshape(want.shape[0], -1)
        k = flat.argmax(1)
        v = flat[np.arange(flat.shape[0]), k]
        better = v > self.val
        self.val[better] = v[better]
        self.idx[better] = k[better] + r0 * self.per_ref


def pose_agreement(best: Best, pick, oracle_at_pick, tol):
    """fraction identical; every mismatch must be excused by an oracle gap below tol (relative)"""
    same = pick == best.idx
    gap = (best.val - oracle_at_pick) / np.abs(best.val)
    excused = (~same) & (gap < tol)
    return float(same.mean()), int(excused.sum()), int(((~same) & ~excused).sum())


@pytest.fixture(scope="module")
def sample(pkg, O):
    w = pkg.synth.config1()
    shifts = np.asarray(w.shift_grid, np.float32)
    refs, R = pkg.synth.make_refs(w)
    refs = refs.numpy()
    npt = max(NPT_PTCL, NPT_REF)
    parts = pkg.synth.make_particles(w, R, count=npt)
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    ctfs = np.stack([O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                               float(parts.angast[i]))) for i in range(npt)])
    def ctfp(n):
        return pkg.ctfparams_array(n, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca, dfx=parts.dfx[:n],
                                   dfy=parts.dfy[:n], angast=parts.angast[:n])
    return w, shifts, refs, parts, g, t, ctfs, ctfp


def _handle(pkg, w, refs, parts, ctfp, n, frame):
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, n), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame=frame)
    pc.set_refs(1, refs, True)
    pc.set_refs(1, refs, False)
    pc.polarize_ptcls(0, parts.cmat[:n].numpy())
    pc.create_polar_absctfmats(ctfp(n))
    return pc


def _pose_index(out, ns, N):
    return (out["iref"].astype(np.int64) - 1) * ns * N + out["ishift"].astype(np.int64) * N + \
        out["irot"].astype(np.int64) - 1


def test_precision_against_fp64_oracle(pkg, O, sample):
    w, shifts, refs, parts, g, t, ctfs, ctfp = sample
    ns, N = len(shifts), w.nrots
    per_ref = ns * N
    report = {"workload": f"config-1 geometry: {w.nrefs} refs x {ns} shifts x {N} rots, box {w.box}, "
                          f"shells {w.kfrom}..{w.kto}, astigmatic CTF",
              "floor": FLOOR, "oracle": "CPU FP64 (oracle.iter_allcorrs64)"}
    t0 = time.time()

    # ---------------- reference frame: the drop-in gencorrs and the reference's FP32 loop
    nref = NPT_REF
    pc = _handle(pkg, w, refs, parts, ctfp, nref, "ref")
    pfts_r = np.stack([pc.get_ptcl_pft(i + 1) for i in range(nref)])
    exact_ref = Errors(pc.corr_all(shifts).reshape(nref, w.nrefs, ns, N))
    srch_ref = pc.search_best(shifts, "bf16x3", ntop=8)
    pc.kill()
    loop = Errors(np.stack([O.fftpath_allcorrs(g, refs, pfts_r[i], ctfs[i], shifts)[0] for i in range(nref)]))
    best_ref = Best(nref, per_ref)
    srch_ref_pick = _pose_index(srch_ref, ns, N)
    srch_ref_at = np.full(nref, np.nan)
    ref_frame_vals = {}
    for r0, r1, want in O.iter_allcorrs64(g, t, refs, pfts_r, ctfs[:nref], shifts, frame="ref"):
        exact_ref.add(r0, r1, want)
        loop.add(r0, r1, want)
        best_ref.add(r0, want)
        for p, k in enumerate(srch_ref_pick):
            if r0 * per_ref <= k < r1 * per_ref:
                srch_ref_at[p] = want[p].reshape(-1)[k - r0 * per_ref]
        ref_frame_vals[r0] = want
    report["reference_fp32_fft_loop"] = loop.summary()
    report["exact_ref_frame"] = exact_ref.summary()
    # elementwise gate of the exact kernel, normwise gates of the m-domain paths
    gate = {"exact": max(TOL["exact"], loop.max_rel), "fp32": max(TOL["fp32"], loop.max_nrm),
            "bf16x3": max(TOL["bf16x3"], loop.max_nrm)}
    report["gates"] = {"exact (elementwise, floor 1e-3)": gate["exact"], "fp32 (normwise)": gate["fp32"],
                       "bf16x3 (normwise)": gate["bf16x3"]}

    # ---------------- particle frame: exact kernel, FP32 m-domain, raw BF16 split, search
    npt = NPT_PTCL
    pc = _handle(pkg, w, refs, parts, ctfp, npt, "ptcl")
    pfts = np.stack([pc.get_ptcl_pft(i + 1) for i in range(npt)])
    assert np.array_equal(pfts[:nref], pfts_r)
    paths = {p: Errors(pc.corr_all_prec(shifts, p).reshape(npt, w.nrefs, ns, N)) for p in ("exact", "fp32", "bf16x3")}
    srch = pc.search_best(shifts, "bf16x3", ntop=8)
    pc.kill()
    best = Best(npt, per_ref)
    srch_pick = _pose_index(srch, ns, N)
    srch_at = np.full(npt, np.nan)
    frame_dev_max = 0.0
    for r0, r1, want in O.iter_allcorrs64(g, t, refs, pfts, ctfs[:npt], shifts, frame="ptcl"):
        for e in paths.values():
            e.add(r0, r1, want)
        best.add(r0, want)
        for p, k in enumerate(srch_pick):
            if r0 * per_ref <= k < r1 * per_ref:
                srch_at[p] = want[p].reshape(-1)[k - r0 * per_ref]
        frame_dev_max = max(frame_dev_max, float(np.abs(want[:nref] - ref_frame_vals[r0]).max()))
    for p, e in paths.items():
        report[f"{p}_ptcl_frame"] = e.summary()

    # ---------------- best poses
    poses = {}
    for p, e in paths.items():
        same, exc, bad = pose_agreement(best, e.pick, e.oracle_at_pick, gate[p])
        poses[f"{p}_ptcl_frame"] = {"identical": same, "excused": exc, "unexcused": bad}
    same, exc, bad = pose_agreement(best_ref, exact_ref.pick, exact_ref.oracle_at_pick, gate["exact"])
    poses["exact_ref_frame"] = {"identical": same, "excused": exc, "unexcused": bad}
    same, exc, bad = pose_agreement(best_ref, loop.pick, loop.oracle_at_pick, gate["fp32"])
    poses["reference_fp32_fft_loop"] = {"identical": same, "excused": exc, "unexcused": bad}
    same, exc, bad = pose_agreement(best, srch_pick, srch_at, gate["fp32"])
    poses["search_bf16x3_rescore_ptcl_frame"] = {"identical": same, "excused": exc, "unexcused": bad}
    same, exc, bad = pose_agreement(best_ref, srch_ref_pick, srch_ref_at, gate["exact"])
    poses["search_bf16x3_rescore_ref_frame"] = {"identical": same, "excused": exc, "unexcused": bad}
    report["best_pose"] = poses
    d_srch = np.abs(srch["corr"].astype(np.float64) - srch_at) / np.maximum(np.abs(srch_at), FLOOR)
    d_srch_ref = np.abs(srch_ref["corr"].astype(np.float64) - srch_ref_at) / np.maximum(np.abs(srch_ref_at), FLOOR)
    report["search_corr_max_rel_err"] = {"ptcl_frame": float(d_srch.max()), "ref_frame": float(d_srch_ref.max())}
    # the particle-frame objective against the reference's at the configs' astigmatism
    bi_ref = best_ref.idx
    bi_ptcl = best.idx[:nref]
    report["ptcl_vs_ref_frame_objective"] = {"max_abs_dcc": frame_dev_max,
                                             "best_pose_identical": float((bi_ref == bi_ptcl).mean()),
                                             "particles": nref}
    report["sample"] = {"ptcl_frame_particles": npt, "ref_frame_particles": nref}
    report["seconds"] = round(time.time() - t0, 1)
    if REPORT:
        with open(REPORT, "w") as f:
            json.dump(report, f, indent=1)
    print(json.dumps(report))

    # ---------------- gates
    assert exact_ref.max_rel <= gate["exact"], report
    assert paths["exact"].max_rel <= gate["exact"], report
    for p in ("fp32", "bf16x3"):
        assert paths[p].max_nrm <= gate[p], (p, report)
    for name, v in poses.items():
        assert v["unexcused"] == 0, (name, report)
    assert d_srch.max() <= gate["exact"], report
    assert d_srch_ref.max() <= gate["exact"], report
