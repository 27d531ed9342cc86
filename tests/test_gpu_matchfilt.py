"""GPU parity of the matched-filter mode (match_filt = params_glob%l_match_filt) against the
oracle: the correlators apply shellnorm_and_filter_ref(_8) to the reference (shell k <= kstop
scaled by ref_optlp / sqrt(its mean power), simple_polarft_corrcalc.f90:756-807), so they equal
the oracle's correlators on the reference so scaled -- gencorrs_cc_1/_2, gencorr_cc_for_rot_8 and
its gradient (the match_filt branch), the m-domain search's values; prep_matchfilt (:987-1095)
against the oracle's restatement; set_ref_optlp's state check.  Tolerances: the exact
correlators 2e-5 with |cc| floored at 1e-2 (twice the plain mode's gate: with every shell at unit
power the high shells, whose FP32 operand rounding is the error, weigh as much as the low ones),
the m-domain values 1e-5 absolute, the filtered particle 2e-6 of its largest component."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def build(pkg, w, frame, ctf=True):
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    refs = refs.numpy()
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), kstop=w.kto - 3, ctf=ctf,
           ctf_frame=frame, match_filt=True)
    pc.set_refs(1, refs, True)
    pc.set_refs(1, refs, False)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    if ctf:
        pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                       dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    rng = np.random.default_rng(2)
    opt = {}
    for r in (1, 3):
        opt[r] = rng.uniform(0.3, 1.0, w.kto - 3 - w.kfrom + 1).astype(np.float32)
        pc.set_ref_optlp(r, opt[r])
    return pc, refs, parts, opt


def scaled(O, g, ref, optlp):
    s = O.shellnorm_factors(g, ref, optlp)
    out = ref.astype(np.complex64).copy()
    out[:g.Ks] = (out[:g.Ks] * s[:, None].astype(np.float32)).astype(np.complex64)
    return out


def relerr(a, b, floor=1e-2):
    return float(np.max(np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), floor)))


def test_matchfilt_correlators(pkg, O):
    w = pkg.synth.config0(nrefs=3, nptcls=3)
    pc, refs, parts, opt = build(pkg, w, "ref")
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box, kstop=w.kto - 3)
    t = O.tables(g)
    try:
        for i in range(3):
            c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                          float(parts.angast[i])))
            pft = pc.get_ptcl_pft(i + 1)
            for r in (1, 2, 3):
                rs = scaled(O, g, refs[r - 1], opt.get(r))
                assert relerr(pc.gencorrs(r, i + 1), O.gencorrs(g, t, rs, pft, c, None)) < 2e-5
                sh = [0.6, -0.8]
                assert relerr(pc.gencorrs(r, i + 1, sh), O.gencorrs(g, t, rs, pft, c, sh)) < 2e-5
                for irot in (1, 50):
                    want = O.gencorr_for_rot(g, t, rs, pft, irot, c, np.array(sh), True)
                    assert abs(pc.gencorr_for_rot_8(r, i + 1, np.array(sh), irot) - want) < 1e-6
                    f, gr = pc.gencorr_grad_for_rot_8(r, i + 1, np.array(sh), irot)
                    fo, go = O.gencorr_grad3(g, t, rs, pft, irot, c, None, np.array(sh), True)
                    assert abs(f - fo) < 1e-6 and np.max(np.abs(gr - go[:2])) < 1e-6 * max(1, np.max(np.abs(go)))
        # the batched exact search sees the same factors
        cc = pc.corr_all(None)
        pft = pc.get_ptcl_pft(2)
        c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[1]), float(parts.dfy[1]),
                                      float(parts.angast[1])))
        assert relerr(cc[1, 2, 0], O.gencorrs(g, t, scaled(O, g, refs[2], opt[3]), pft, c, None)) < 2e-5
    finally:
        pc.kill()


def test_matchfilt_mdomain(pkg, O):
    w = pkg.synth.config0(nrefs=3, nptcls=4)
    pc, refs, parts, opt = build(pkg, w, "ptcl")
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box, kstop=w.kto - 3)
    t = O.tables(g)
    shifts = np.array([[0, 0], [0.5, -1.0]], np.float32)
    try:
        cc = pc.corr_all_prec(shifts, "fp32")
        worst = 0.0
        for i in range(4):
            c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                          float(parts.angast[i])))
            pft = pc.get_ptcl_pft(i + 1)
            for r in range(3):
                rs = scaled(O, g, refs[r], opt.get(r + 1))
                for s in range(2):
                    want = O.gencorrs_ptclframe(g, t, rs, pft, c, shifts[s].astype(np.float64))
                    worst = max(worst, float(np.max(np.abs(cc[i, r, s] - want))))
        print(f"matched-filter m-domain FP32: max |dcc| {worst:.2e}")
        assert worst < 1e-5
    finally:
        pc.kill()


def test_prep_matchfilt(pkg, O):
    w = pkg.synth.config0(nrefs=3, nptcls=4)
    pc, refs, parts, opt = build(pkg, w, "ref")
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box, kstop=w.kto - 3)
    t = O.tables(g)
    try:
        before = [pc.get_ptcl_pft(i + 1) for i in range(4)]
        reqs = [(1, 1, 1), (2, 3, 40), (3, 0, 5), (4, 2, 100)]     # iref 0: nothing to do
        pc.prep_matchfilt_batch(*[np.array(v) for v in zip(*reqs)])
        for ip, ir, irot in reqs:
            got = pc.get_ptcl_pft(ip)
            if ir == 0:
                assert np.array_equal(got, before[ip - 1])
                continue
            c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[ip - 1]),
                                          float(parts.dfy[ip - 1]), float(parts.angast[ip - 1])))
            want = O.prep_matchfilt(g, refs[ir - 1], before[ip - 1], irot, c, opt.get(ir))
            assert np.max(np.abs(got - want)) < 2e-6 * np.max(np.abs(want))
            sq = np.sum(np.abs(want[:g.Ks].astype(np.complex128)) ** 2)
            assert abs(pc.get_sqsum_ptcl(ip) - sq) < 1e-5 * sq
        pc.prep_matchfilt(2, 1, 7)          # the single-request form
    finally:
        pc.kill()
    pc = pkg.polarft_corrcalc()
    pc.new(1, (1, 1), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=False)
    with pytest.raises(pkg.PftccError) as e:
        pc.set_ref_optlp(1, np.ones(w.kto - w.kfrom + 1, np.float32))
    assert e.value.status == pkg._lib.ERR_STATE
    pc.kill()


def test_pssnr_mode(pkg, O):
    """l_pssnr (pftcc_set_pssnr): the correlators use the reference scaled to power ssnr k per
    shell (shellnorm_and_filter_ref :763-770), the m-domain search too, and prep_matchfilt
    rescales the particle by sqrt(k / power) sqrt(1 + ssnr |CTF|^2) (:999-1019)"""
    w = pkg.synth.config0(nrefs=3, nptcls=3)
    pc, refs, parts, opt = build(pkg, w, "ref")
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box, kstop=w.kto - 3)
    t = O.tables(g)
    try:
        pc.set_pssnr(True)
        for i in range(3):
            c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                          float(parts.angast[i])))
            pft = pc.get_ptcl_pft(i + 1)
            for r in (1, 2, 3):
                s = O.shellnorm_factors(g, refs[r - 1], opt.get(r), pssnr=True)
                rs = refs[r - 1].astype(np.complex64).copy()
                rs[:g.Ks] = (rs[:g.Ks] * s[:, None].astype(np.float32)).astype(np.complex64)
                assert relerr(pc.gencorrs(r, i + 1, [0.4, 0.3]), O.gencorrs(g, t, rs, pft, c, [0.4, 0.3])) < 2e-5
                want = O.gencorr_for_rot(g, t, rs, pft, 7, c, np.array([0.4, 0.3]), True)
                assert abs(pc.gencorr_for_rot_8(r, i + 1, np.array([0.4, 0.3]), 7) - want) < 1e-6
        # prep_matchfilt in the pssnr mode against the oracle
        before = pc.get_ptcl_pft(2)
        c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[1]), float(parts.dfy[1]),
                                      float(parts.angast[1])))
        pc.prep_matchfilt(2, 3, 11)
        want = O.prep_matchfilt_pssnr(g, before, c, opt[3])
        got = pc.get_ptcl_pft(2)
        assert np.max(np.abs(got - want)) < 2e-6 * np.max(np.abs(want))
        sq = np.sum(np.abs(got[:g.Ks].astype(np.complex128)) ** 2)
        assert abs(pc.get_sqsum_ptcl(2) - sq) < 1e-5 * sq
        pc.set_pssnr(False)
    finally:
        pc.kill()
    # the mode needs the matched filter
    plain = pkg.polarft_corrcalc()
    plain.new(1, (1, 1), box=64, nrots=128, kfromto=(2, 20), ctf=False)
    with pytest.raises(pkg.PftccError) as e:
        plain.set_pssnr(True)
    assert e.value.status == pkg._lib.ERR_STATE
    plain.kill()
