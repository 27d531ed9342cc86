"""GPU parity tests of the m-domain search (particle-frame CTF) through the C ABI:
every correlation of the FP32 and BF16-split paths against the FP64 oracle, the
search's best (ref, rot, shift) against the exact path, the re-score in the
reference frame, parity groups, padding and transform-length edge cases.

Error measure: the normalised cross-correlation lies in [-1, 1], so errors are
relative to that full scale, |cc - cc_fp64| <= 1e-5 (plain FP32) and <= 1e-4 (BF16
hi+lo split).  Relative errors with |cc| floored at 1e-2 are printed as well: an
FFT-based evaluation carries its rounding relative to the whole correlation
function, so near-zero values show larger relative errors than the peaks that
decide the search (tests/test_gpu_precision.py measures both against the reference's
own FP32 loop at config-1 scale).  Best poses: identical to the exhaustive exact
search's for every particle, except where the exact correlations at the two poses
differ by less than the FP32 tolerance relative to the best."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL_FP32 = 1e-5
TOL_BF16 = 1e-4


def abserr(a, b):
    return float(np.max(np.abs(np.asarray(a, np.float64) - b)))


def relerr(a, b, floor=1e-2):
    return float(np.max(np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), floor)))


def build(pkg, w, frame="ptcl", eo=None, ctf=True):
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    refs = refs.numpy()
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=ctf, ctf_frame=frame,
           eoarr=eo)
    pc.set_refs(1, refs, True)
    pc.set_refs(1, (refs * np.complex64(0.8 + 0.2j)).astype(np.complex64), False)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    if ctf:
        pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                       dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    return pc, refs, parts


def oracle_all(O, w, pc, refs, parts, shifts, particles, nrefs):
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    out = {}
    for i in particles:
        c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                      float(parts.angast[i])))
        pft = pc.get_ptcl_pft(i + 1)
        for r in range(nrefs):
            for s in range(len(shifts)):
                out[i, r, s] = O.gencorrs_ptclframe(g, t, refs[r], pft, c, shifts[s].astype(np.float64))
    return out


def same_pose(a, b):
    return (a["iref"] == b["iref"]) & (a["irot"] == b["irot"]) & (a["ishift"] == b["ishift"])


def pose_index(a, ns, nrots):
    return (a["iref"].astype(np.int64) - 1) * ns * nrots + np.maximum(a["ishift"], 0).astype(np.int64) * nrots + \
        a["irot"].astype(np.int64) - 1


def assert_poses(got, ex, allcc, ns, nrots, tol):
    """best poses identical to the exhaustive exact search's, except where the exact
    correlations at the two poses differ by less than tol relative to the best (a near-tie
    that the path's tolerance cannot order); returns the identical fraction"""
    gi, ei = pose_index(got, ns, nrots), pose_index(ex, ns, nrots)
    rows = np.arange(len(gi))
    best = allcc[rows, ei].astype(np.float64)
    gap = (best - allcc[rows, gi]) / np.abs(best)
    same = gi == ei
    bad = np.where(~same & ~(gap < tol))[0]
    assert bad.size == 0, f"unexcused best-pose mismatches at particles {bad.tolist()} (gaps {gap[bad].tolist()})"
    return float(same.mean())


@pytest.mark.parametrize("cfgname", ["config0", "config1", "geometry_c"])
def test_mdomain_fp32_every_correlation(pkg, O, cfgname):
    w = getattr(pkg.synth, cfgname)(nrefs=3, nptcls=4)
    pc, refs, parts = build(pkg, w)
    shifts = np.array([[0.0, 0.0], [1.0, -0.5], [-2.0, 1.5]], np.float32)
    cc = pc.corr_all_prec(shifts, "fp32")
    want = oracle_all(O, w, pc, refs, parts, shifts, range(w.nptcls), 3)
    ea = max(abserr(cc[k], v) for k, v in want.items())
    er = max(relerr(cc[k], v) for k, v in want.items())
    print(f"fp32 m-domain {cfgname}: max |dcc| {ea:.2e}, max rel (floor 1e-2) {er:.2e}")
    assert ea < TOL_FP32
    # the exact path in the particle frame agrees as well
    assert abserr(cc, pc.corr_all(shifts)) < TOL_FP32


@pytest.mark.parametrize("cfgname", ["config0", "config1", "geometry_c"])
def test_mdomain_bf16x3_every_correlation(pkg, O, cfgname):
    """tcgen05 BF16 hi+lo split contraction: every correlation against the FP64 oracle"""
    w = getattr(pkg.synth, cfgname)(nrefs=5, nptcls=130)
    pc, refs, parts = build(pkg, w)
    shifts = np.array([[0.0, 0.0], [1.0, -0.5], [-2.0, 1.5]], np.float32)
    cc = pc.corr_all_prec(shifts, "bf16x3")
    c32 = pc.corr_all_prec(shifts, "fp32")
    assert abserr(cc, c32) < TOL_BF16
    want = oracle_all(O, w, pc, refs, parts, shifts, list(range(0, w.nptcls, 29)) + [w.nptcls - 1], 5)
    ea = max(abserr(cc[k], v) for k, v in want.items())
    er = max(relerr(cc[k], v) for k, v in want.items())
    print(f"bf16x3 {cfgname}: max |dcc| {ea:.2e}, max rel (floor 1e-2) {er:.2e}")
    assert ea < TOL_BF16


def test_search_fp32_matches_exact(pkg):
    w = pkg.synth.config0(nrefs=20, nptcls=40)
    pc, refs, parts = build(pkg, w)
    shifts = np.array(pkg.synth.shift_grid(1.0, 0.5), np.float32)
    ex = pc.search_best(shifts, "exact")
    allcc = pc.corr_all(shifts).reshape(w.nptcls, -1)
    for ntop in (0, 8):
        md = pc.search_best(shifts, "fp32", ntop=ntop)
        assert_poses(md, ex, allcc, len(shifts), w.nrots, TOL_FP32)
        assert np.max(np.abs(md["corr"] - ex["corr"])) < TOL_FP32


def test_search_no_shift_and_parity_groups(pkg):
    """mixed even/odd particles use their own reference set; no shift grid = gencorrs_cc_1"""
    w = pkg.synth.config0(nrefs=7, nptcls=70)
    eo = [i % 3 == 0 for i in range(70)]
    pc, refs, parts = build(pkg, w, eo=[0 if e else 1 for e in eo])
    ex = pc.search_best(None, "exact")
    md = pc.search_best(None, "fp32", ntop=4)
    assert_poses(md, ex, pc.corr_all(None).reshape(w.nptcls, -1), 1, w.nrots, TOL_FP32)
    assert np.all(md["ishift"] == -1) and np.all(ex["ishift"] == -1)
    assert np.max(np.abs(md["corr"] - ex["corr"])) < TOL_FP32


def test_search_reference_frame_rescore(pkg):
    """REF-frame handle: the m-domain search screens in the particle frame and the
    top-8 re-score returns reference-frame correlations; agreement with the
    exhaustive reference-frame search is reported"""
    w = pkg.synth.config0(nrefs=16, nptcls=48)
    pc, refs, parts = build(pkg, w, frame="ref")
    shifts = np.array(pkg.synth.shift_grid(1.0, 0.5), np.float32)
    ex = pc.search_best(shifts, "exact")
    allcc = pc.corr_all(shifts).reshape(w.nptcls, -1)
    for prec in ("fp32", "bf16x3"):
        rs = pc.search_best(shifts, prec, ntop=8)
        frac = assert_poses(rs, ex, allcc, len(shifts), w.nrots, TOL_FP32)
        print(f"reference-frame agreement after the top-8 re-score ({prec}): {frac:.3f}")
        same = same_pose(rs, ex)
        assert np.max(np.abs(rs["corr"][same] - ex["corr"][same])) < 1e-6
    assert np.all(rs["corr"] <= ex["corr"] + 1e-6)


def test_search_odd_sizes(pkg):
    """one reference, one particle, ragged tiles"""
    shifts = np.array([[0.5, 0.5]], np.float32)
    for nr, npt in ((1, 1), (3, 65), (2, 129)):
        w = pkg.synth.config0(nrefs=nr, nptcls=npt)
        pc, refs, parts = build(pkg, w)
        ex = pc.search_best(shifts, "exact")
        allcc = pc.corr_all(shifts).reshape(npt, -1)
        for prec in ("fp32", "bf16x3"):
            md = pc.search_best(shifts, prec, ntop=min(2, nr))
            assert_poses(md, ex, allcc, 1, w.nrots, TOL_FP32)
            assert np.max(np.abs(md["corr"] - ex["corr"])) < TOL_FP32


def test_true_pose_recovered(pkg):
    """with the generating reference among the candidates the search finds the true
    reference and in-plane angle for most particles at SNR 0.1"""
    w = pkg.synth.config0(nrefs=10, nptcls=30)
    pc, refs, parts = build(pkg, w)
    shifts = np.array(pkg.synth.shift_grid(3.0, 1.0), np.float32)
    md = pc.search_best(shifts, "bf16x3", ntop=8)
    ok_ref = md["iref"] - 1 == parts.ref
    d = np.abs((md["irot"] - 1) - parts.psi * w.nrots / 360.0)
    ok_rot = np.minimum(d, w.nrots - d) <= 2.0
    assert (ok_ref & ok_rot).mean() > 0.6


def test_search_bf16x3_rescored_matches_exact(pkg):
    w = pkg.synth.config0(nrefs=24, nptcls=200)
    pc, refs, parts = build(pkg, w)
    shifts = np.array(pkg.synth.shift_grid(1.0, 0.5), np.float32)
    ex = pc.search_best(shifts, "exact")
    bf = pc.search_best(shifts, "bf16x3", ntop=8)
    frac = assert_poses(bf, ex, pc.corr_all(shifts).reshape(w.nptcls, -1), len(shifts), w.nrots, TOL_FP32)
    print(f"bf16x3 + FP32 re-score best-pose agreement with the exact path: {frac:.4f}")
    assert np.max(np.abs(bf["corr"] - ex["corr"])) < TOL_FP32
    raw = pc.search_best(shifts, "bf16x3", ntop=0)
    assert np.max(np.abs(raw["corr"] - ex["corr"])) < TOL_BF16


def test_bf16x3_parity_groups(pkg):
    """mixed even/odd particles starting mid-tile in the packed particle operand"""
    w = pkg.synth.config0(nrefs=6, nptcls=300)
    eo = [0 if i % 5 else 1 for i in range(300)]
    pc, refs, parts = build(pkg, w, eo=eo)
    shifts = np.array([[0.0, 0.0], [0.5, 0.5]], np.float32)
    ex = pc.search_best(shifts, "exact")
    bf = pc.search_best(shifts, "bf16x3", ntop=3)
    assert_poses(bf, ex, pc.corr_all(shifts).reshape(w.nptcls, -1), len(shifts), w.nrots, TOL_FP32)
    assert np.max(np.abs(bf["corr"] - ex["corr"])) < TOL_FP32


def test_generic_transform_length(pkg, O):
    """nrots/2 = 50 has no compile-time transform: the generic radix loop serves it"""
    w = pkg.synth.config0(nrefs=3, nptcls=5, nrots=100)
    pc, refs, parts = build(pkg, w)
    shifts = np.array([[0.0, 0.0], [1.0, 1.0]], np.float32)
    cc = pc.corr_all_prec(shifts, "fp32")
    want = oracle_all(O, w, pc, refs, parts, shifts, range(w.nptcls), 3)
    assert max(abserr(cc[k], v) for k, v in want.items()) < TOL_FP32
    ex = pc.search_best(shifts, "exact")
    md = pc.search_best(shifts, "fp32", ntop=2)
    assert_poses(md, ex, pc.corr_all(shifts).reshape(w.nptcls, -1), len(shifts), w.nrots, TOL_FP32)
    assert np.max(np.abs(md["corr"] - ex["corr"])) < TOL_FP32
