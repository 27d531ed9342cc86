"""GPU parity tests of the m-domain search (particle-frame CTF) through the C ABI:
every correlation of the FP32 path against the FP64 oracle, the search's best
(ref, rot, shift) against the exact path, the re-score in the reference frame,
parity groups and padding edge cases."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL_FP32 = 1e-5      # plain FP32 bar, |cc| floored at 1e-2 (precision)


def relerr(a, b, floor=1e-2):
    return np.max(np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), floor))


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


@pytest.mark.parametrize("cfgname", ["config0", "config1", "geometry_c"])
def test_mdomain_fp32_every_correlation(pkg, O, cfgname):
    w = getattr(pkg.synth, cfgname)(nrefs=3, nptcls=4)
    pc, refs, parts = build(pkg, w)
    shifts = np.array([[0.0, 0.0], [1.0, -0.5], [-2.0, 1.5]], np.float32)
    cc = pc.corr_all_prec(shifts, "fp32")
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    worst = 0.0
    for i in range(w.nptcls):
        c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                      float(parts.angast[i])))
        pft = pc.get_ptcl_pft(i + 1)
        for r in range(3):
            for s in range(3):
                want = O.gencorrs_ptclframe(g, t, refs[r], pft, c, shifts[s].astype(np.float64))
                worst = max(worst, relerr(cc[i, r, s], want))
    assert worst < TOL_FP32, worst
    # the exact path in the particle frame agrees as well
    ex = pc.corr_all(shifts)
    assert relerr(cc, ex) < TOL_FP32


def test_search_fp32_matches_exact(pkg):
    w = pkg.synth.config0(nrefs=20, nptcls=40)
    pc, refs, parts = build(pkg, w)
    shifts = np.array(pkg.synth.shift_grid(1.0, 0.5), np.float32)
    ex = pc.search_best(shifts, "exact")
    md = pc.search_best(shifts, "fp32", ntop=0)
    allcc = pc.corr_all(shifts).reshape(w.nptcls, -1)
    agree = 0
    for i in range(w.nptcls):
        srt = np.sort(allcc[i])[::-1]
        if (md["iref"][i], md["irot"][i], md["ishift"][i]) == (ex["iref"][i], ex["irot"][i], ex["ishift"][i]):
            agree += 1
        else:
            assert srt[0] - srt[1] < 1e-5     # only near-ties may differ
        assert abs(md["corr"][i] - ex["corr"][i]) < 1e-5
    assert agree >= w.nptcls - 1
    # re-score of the top 8 in FP32 gives the exact path's answer
    rs = pc.search_best(shifts, "fp32", ntop=8)
    assert np.array_equal(rs["iref"], ex["iref"]) and np.array_equal(rs["irot"], ex["irot"])
    assert np.array_equal(rs["ishift"], ex["ishift"]) and np.array_equal(rs["corr"], ex["corr"])


def test_search_no_shift_and_parity_groups(pkg):
    """mixed even/odd particles use their own reference set; no shift grid = gencorrs_cc_1"""
    w = pkg.synth.config0(nrefs=7, nptcls=70)
    eo = [i % 3 == 0 for i in range(70)]
    pc, refs, parts = build(pkg, w, eo=[0 if e else 1 for e in eo])
    ex = pc.search_best(None, "exact")
    md = pc.search_best(None, "fp32", ntop=4)
    assert np.array_equal(md["iref"], ex["iref"]) and np.array_equal(md["irot"], ex["irot"])
    assert np.all(md["ishift"] == -1) and np.all(ex["ishift"] == -1)
    assert np.array_equal(md["corr"], ex["corr"])


def test_search_reference_frame_rescore(pkg):
    """REF-frame handle: the m-domain search screens in the particle frame and the
    top-8 re-score returns reference-frame correlations; report agreement with the
    exhaustive reference-frame search"""
    w = pkg.synth.config0(nrefs=16, nptcls=48)
    pc, refs, parts = build(pkg, w, frame="ref")
    shifts = np.array(pkg.synth.shift_grid(1.0, 0.5), np.float32)
    ex = pc.search_best(shifts, "exact")
    rs = pc.search_best(shifts, "fp32", ntop=8)
    same = (rs["iref"] == ex["iref"]) & (rs["irot"] == ex["irot"]) & (rs["ishift"] == ex["ishift"])
    assert same.mean() >= 0.9
    # where they agree the correlation is the reference-frame value
    assert np.max(np.abs(rs["corr"][same] - ex["corr"][same])) < 1e-6
    assert np.all(rs["corr"] <= ex["corr"] + 1e-6)


def test_search_odd_sizes(pkg):
    """one reference, one particle, ragged tiles"""
    w = pkg.synth.config0(nrefs=1, nptcls=1)
    pc, refs, parts = build(pkg, w)
    shifts = np.array([[0.5, 0.5]], np.float32)
    ex = pc.search_best(shifts, "exact")
    md = pc.search_best(shifts, "fp32", ntop=1)
    assert tuple(md[0]) == tuple(ex[0])
    w = pkg.synth.config0(nrefs=3, nptcls=65)
    pc, refs, parts = build(pkg, w)
    ex = pc.search_best(shifts, "exact")
    md = pc.search_best(shifts, "fp32", ntop=2)
    assert np.array_equal(md["iref"], ex["iref"]) and np.array_equal(md["corr"], ex["corr"])


def test_true_pose_recovered(pkg):
    """with the generating reference among the candidates the search finds the true
    reference and in-plane angle for most particles at SNR 0.1"""
    w = pkg.synth.config0(nrefs=10, nptcls=30)
    pc, refs, parts = build(pkg, w)
    shifts = np.array(pkg.synth.shift_grid(3.0, 1.0), np.float32)
    md = pc.search_best(shifts, "fp32", ntop=8)
    ok_ref = md["iref"] - 1 == parts.ref
    d = np.abs((md["irot"] - 1) - parts.psi * w.nrots / 360.0)
    ok_rot = np.minimum(d, w.nrots - d) <= 2.0
    assert (ok_ref & ok_rot).mean() > 0.6


TOL_BF16 = 1e-4      # BF16 hi+lo split bar, |cc| floored at 1e-2


@pytest.mark.parametrize("cfgname", ["config0", "config1", "geometry_c"])
def test_mdomain_bf16x3_every_correlation(pkg, O, cfgname):
    """tcgen05 BF16 hi+lo split contraction: every correlation against the FP64 oracle"""
    w = getattr(pkg.synth, cfgname)(nrefs=5, nptcls=130)
    pc, refs, parts = build(pkg, w)
    shifts = np.array([[0.0, 0.0], [1.0, -0.5], [-2.0, 1.5]], np.float32)
    cc = pc.corr_all_prec(shifts, "bf16x3")
    c32 = pc.corr_all_prec(shifts, "fp32")
    assert relerr(cc, c32) < TOL_BF16
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    worst = 0.0
    for i in list(range(0, w.nptcls, 29)) + [w.nptcls - 1]:
        c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                      float(parts.angast[i])))
        pft = pc.get_ptcl_pft(i + 1)
        for r in range(5):
            for s in range(3):
                want = O.gencorrs_ptclframe(g, t, refs[r], pft, c, shifts[s].astype(np.float64))
                worst = max(worst, relerr(cc[i, r, s], want))
    assert worst < TOL_BF16, worst


def test_search_bf16x3_rescored_matches_exact(pkg):
    w = pkg.synth.config0(nrefs=24, nptcls=200)
    pc, refs, parts = build(pkg, w)
    shifts = np.array(pkg.synth.shift_grid(1.0, 0.5), np.float32)
    ex = pc.search_best(shifts, "exact")
    bf = pc.search_best(shifts, "bf16x3", ntop=8)
    assert np.array_equal(bf["iref"], ex["iref"]) and np.array_equal(bf["irot"], ex["irot"])
    assert np.array_equal(bf["ishift"], ex["ishift"]) and np.array_equal(bf["corr"], ex["corr"])
    raw = pc.search_best(shifts, "bf16x3", ntop=0)
    assert np.max(np.abs(raw["corr"] - ex["corr"]) / np.maximum(np.abs(ex["corr"]), 1e-2)) < TOL_BF16


def test_bf16x3_parity_groups(pkg):
    """mixed even/odd particles starting mid-tile in the packed particle operand"""
    w = pkg.synth.config0(nrefs=6, nptcls=300)
    eo = [0 if i % 5 else 1 for i in range(300)]
    pc, refs, parts = build(pkg, w, eo=eo)
    shifts = np.array([[0.0, 0.0], [0.5, 0.5]], np.float32)
    ex = pc.search_best(shifts, "exact")
    bf = pc.search_best(shifts, "bf16x3", ntop=3)
    assert np.array_equal(bf["iref"], ex["iref"]) and np.array_equal(bf["corr"], ex["corr"])


def test_generic_transform_length(pkg, O):
    """nrots/2 = 50 has no compile-time transform: the generic radix loop serves it"""
    w = pkg.synth.config0(nrefs=3, nptcls=5, nrots=100)
    pc, refs, parts = build(pkg, w)
    shifts = np.array([[0.0, 0.0], [1.0, 1.0]], np.float32)
    cc = pc.corr_all_prec(shifts, "fp32")
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    worst = 0.0
    for i in range(w.nptcls):
        c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                      float(parts.angast[i])))
        pft = pc.get_ptcl_pft(i + 1)
        for r in range(3):
            for s in range(2):
                worst = max(worst, relerr(cc[i, r, s], O.gencorrs_ptclframe(g, t, refs[r], pft, c,
                                                                            shifts[s].astype(np.float64))))
    assert worst < TOL_FP32, worst
    ex = pc.search_best(shifts, "exact")
    md = pc.search_best(shifts, "fp32", ntop=2)
    assert np.array_equal(md["iref"], ex["iref"]) and np.array_equal(md["irot"], ex["irot"])
