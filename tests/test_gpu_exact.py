"""GPU parity tests of the exact FP32 path through the C ABI against the FP64 oracle:
gridding, CTF matrices, gencorrs (cc_1 / cc_2, both CTF frames), the single-rotation
correlators and gradients, the batched corr_all / search_best, edge cases and
error codes.  Tolerance: 1e-5 relative with |cc| floored at 1e-2.  The floor: the reference
prepares the reference as (ref * ctf) * shmat in FP32 (gencorrs_cc_2 :1526-1528),
and that operand rounding alone leaves ~3e-8 absolute error on every correlation,
i.e. up to 3e-5 relative on correlations near 1e-3."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-5


def relerr(a, b):
    return np.max(np.abs(np.asarray(a, np.float64) - b) / np.maximum(np.abs(b), 1e-2))


def setup(pkg, w, frame="ref", ctf=True, kstop=None, eo=None, mask=None):
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    refs = refs.numpy()
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), kstop=kstop, ctf=ctf,
           ctf_frame=frame, eoarr=eo, ptcl_mask=mask)
    pc.set_refs(1, refs, True)
    pc.set_refs(1, (refs * np.complex64(0.9 - 0.1j)).astype(np.complex64), False)
    n = pc.get_nptcls()
    pc.polarize_ptcls(0, parts.cmat.numpy()[:n])
    if ctf:
        pc.create_polar_absctfmats(pkg.ctfparams_array(n, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                       dfx=parts.dfx[:n], dfy=parts.dfy[:n], angast=parts.angast[:n]))
    return pc, refs, parts


def oracle_ctx(O, w, parts, i, ctf=True):
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    c = None
    if ctf:
        c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                      float(parts.angast[i])))
    return g, t, c


@pytest.mark.parametrize("cfgname", ["config0", "config1"])
def test_polarize_matches_oracle(pkg, O, cfgname):
    w = getattr(pkg.synth, cfgname)(nrefs=2, nptcls=3)
    pc, refs, parts = setup(pkg, w)
    for i in range(3):
        g, t, _ = oracle_ctx(O, w, parts, i)
        want = O.polarize(g, t, parts.cmat[i].numpy())
        got = pc.get_ptcl_pft(i + 1)
        assert np.max(np.abs(got - want)) / np.max(np.abs(want)) < 2e-6
        sq = np.sum(np.abs(want[: g.Ks]) ** 2)
        assert abs(pc.get_sqsum_ptcl(i + 1) - sq) / sq < 1e-5


@pytest.mark.parametrize("cfgname", ["config0", "config1"])
@pytest.mark.parametrize("frame", ["ref", "ptcl"])
def test_gencorrs_matches_oracle(pkg, O, cfgname, frame):
    w = getattr(pkg.synth, cfgname)(nrefs=3, nptcls=3)
    pc, refs, parts = setup(pkg, w, frame=frame)
    fn = O.gencorrs if frame == "ref" else O.gencorrs_ptclframe
    for i in range(3):
        g, t, c = oracle_ctx(O, w, parts, i)
        pft = pc.get_ptcl_pft(i + 1)
        for r in range(3):
            for sh in (None, [0.0, 0.0], [1.5, -0.5], [-2.0, 2.0]):
                if frame == "ptcl" and sh is None:
                    continue
                got = pc.gencorrs(r + 1, i + 1, sh)
                want = fn(g, t, refs[r], pft, c, None if sh is None else np.asarray(sh, np.float64))
                assert relerr(got, want) < TOL, (i, r, sh)


@pytest.mark.parametrize("cfgname", ["config0", "config1"])
def test_specscore_matches_oracle(pkg, O, cfgname):
    """genfrc / calc_frc shell correlations and specscore against the oracle, single
    and batched, with and without a shift; a reference with itself scores 1"""
    w = getattr(pkg.synth, cfgname)(nrefs=3, nptcls=3)
    pc, refs, parts = setup(pkg, w)
    reqs = []
    for i in range(3):
        g, t, c = oracle_ctx(O, w, parts, i)
        pft = pc.get_ptcl_pft(i + 1)
        for r in range(3):
            for irot in (1, 17, w.nrots - 3):
                for sh in (None, [1.25, -0.75]):
                    shv = None if sh is None else np.asarray(sh, np.float64)
                    want_frc = O.genfrc(g, t, refs[r], pft, irot, c, shv)
                    got_frc = pc.genfrc(r + 1, i + 1, irot, sh)
                    assert np.max(np.abs(got_frc - want_frc)) < 1e-5, (i, r, irot, sh)
                    want = O.specscore(g, t, refs[r], pft, irot, c, shv)
                    assert abs(pc.specscore(r + 1, i + 1, irot, sh) - want) < 1e-5
                    if sh is not None:
                        reqs.append((r + 1, i + 1, irot, sh, want, want_frc))
    scores, frcs = pc.specscore_batch([q[0] for q in reqs], [q[1] for q in reqs], [q[2] for q in reqs],
                                      np.array([q[3] for q in reqs]), want_frc=True)
    assert np.max(np.abs(scores - np.array([q[4] for q in reqs]))) < 1e-5
    assert np.max(np.abs(frcs - np.array([q[5] for q in reqs]))) < 1e-5
    # self-correlation without CTF: a particle slot holding the reference itself
    pc2 = pkg.polarft_corrcalc()
    pc2.new(1, (1, 1), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=False)
    pc2.set_refs(1, refs[:1], True)
    pc2.set_ptcl_pft(1, refs[0])
    assert abs(pc2.specscore(1, 1, 1) - 1.0) < 1e-6
    with pytest.raises(pkg.PftccError):
        pc2.specscore(1, 1, w.nrots + 1)
    pc2.kill()


def test_corr_all_and_search_exact(pkg, O):
    w = pkg.synth.config0(nrefs=5, nptcls=7)
    pc, refs, parts = setup(pkg, w)
    shifts = np.array([[0, 0], [0.5, -1.0], [-1.5, 1.0]], np.float32)
    cc = pc.corr_all(shifts)
    assert cc.shape == (7, 5, 3, w.nrots)
    worst = 0.0
    for i in range(7):
        g, t, c = oracle_ctx(O, w, parts, i)
        pft = pc.get_ptcl_pft(i + 1)
        for r in range(5):
            for s in range(3):
                worst = max(worst, relerr(cc[i, r, s], O.gencorrs(g, t, refs[r], pft, c, shifts[s].astype(np.float64))))
    assert worst < TOL
    best = pc.search_best(shifts, "exact")
    flat = cc.reshape(7, -1)
    for i in range(7):
        j = int(np.argmax(flat[i]))
        r, s, rot = np.unravel_index(j, (5, 3, w.nrots))
        assert (best["iref"][i], best["ishift"][i], best["irot"][i]) == (r + 1, s, rot + 1)
        assert best["corr"][i] == flat[i, j]


def test_eo_parity_and_kstop(pkg, O):
    """odd particles correlate with the odd references (prep_ref4corr :970-974); with
    kstop < kto cc_1 sums sqsum_ref to kstop and cc_2 over all shells (:984 vs :1531)"""
    w = pkg.synth.config0(nrefs=2, nptcls=4)
    pc, refs, parts = setup(pkg, w, kstop=15, eo=[0, 1, 0, 1])
    odd = (refs * np.complex64(0.9 - 0.1j)).astype(np.complex64)
    g0 = O.geom(w.nrots, w.kfrom, w.kto, w.box, kstop=15)
    t = O.tables(g0)
    for i in range(4):
        c = O.ctfmat(g0, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                       float(parts.angast[i])))
        pft = pc.get_ptcl_pft(i + 1)
        r = refs[1] if i % 2 == 0 else odd[1]
        assert pc.ptcl_iseven(i + 1) == (i % 2 == 0)
        assert relerr(pc.gencorrs(2, i + 1), O.gencorrs(g0, t, r, pft, c, None)) < TOL
        assert relerr(pc.gencorrs(2, i + 1, [0.5, 0.5]), O.gencorrs(g0, t, r, pft, c, [0.5, 0.5])) < TOL


def test_for_rot_and_gradients(pkg, O):
    w = pkg.synth.config0(nrefs=2, nptcls=3)
    for mf in (False, True):
        refs, R = pkg.synth.make_refs(w)
        parts = pkg.synth.make_particles(w, R)
        refs = refs.numpy()
        pc = pkg.polarft_corrcalc()
        pc.new(w.nrefs, (1, 3), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), match_filt=mf)
        pc.set_refs(1, refs, True)
        pc.polarize_ptcls(0, parts.cmat.numpy())
        pc.create_polar_absctfmats(pkg.ctfparams_array(3, dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
        for i in range(3):
            g, t, c = oracle_ctx(O, w, parts, i)
            pft = pc.get_ptcl_pft(i + 1)
            ref0 = refs[0]
            if mf:   # match_filt: the reference shell-normalised first (shellnorm_and_filter_ref_8, ref_optlp = 1)
                s = O.shellnorm_factors(g, refs[0])
                ref0 = refs[0].copy()
                ref0[:g.Ks] = (ref0[:g.Ks] * s[:, None].astype(np.float32)).astype(np.complex64)
            for irot in (1, 40, 128):
                sh = np.array([0.7, -0.3])
                want = O.gencorr_for_rot(g, t, ref0, pft, irot, c, sh, mf)
                assert abs(pc.gencorr_for_rot_8(1, i + 1, sh, irot) - want) < 1e-6
                assert abs(pc.gencorr_for_rot(1, i + 1, sh, irot) - want) < 1e-5
                f, gr = pc.gencorr_grad_for_rot_8(1, i + 1, sh, irot)
                fo, go = O.gencorr_grad3(g, t, ref0, pft, irot, c, None, sh, mf)
                assert abs(f - fo) < 1e-6
                assert np.max(np.abs(gr - go[:2])) < 1e-6 * max(1, np.max(np.abs(go)))
                assert np.allclose(pc.gencorr_grad_only_for_rot_8(1, i + 1, sh, irot), gr)
        pc.kill()


def test_grad_batch_defocus(pkg, O):
    """adjoint: d f / d(shift_x, shift_y, defocus) against the FP64 oracle (CTF recomputed in FP64)"""
    w = pkg.synth.config0(nrefs=2, nptcls=3)
    pc, refs, parts = setup(pkg, w)
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    reqs = [(1, 1, 5, 0.3, -0.2, 0.0), (2, 2, 77, -1.0, 0.5, 0.05), (1, 3, 128, 0.0, 0.0, -0.1)]
    f, g3 = pc.grad_batch(*[np.array(v) for v in zip(*reqs)])
    for n, (ir, ip, irot, sx, sy, ddf) in enumerate(reqs):
        i = ip - 1
        cp = O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]) + ddf, float(parts.dfy[i]) + ddf,
                        float(parts.angast[i]))
        pft = pc.get_ptcl_pft(ip)
        fo, go = O.gencorr_grad3(g, t, refs[ir - 1], pft, irot, O.ctfmat(g, t, cp), O.dctfmat_ddf(g, t, cp),
                                 [sx, sy], False)
        # the oracle reads dfx+ddf through float32 parameters: compare at that precision
        assert abs(f[n] - fo) < 2e-5
        assert np.max(np.abs(g3[n] - go)) < 2e-4 * max(1.0, np.max(np.abs(go)))


def test_masked_particles_and_errors(pkg, O):
    w = pkg.synth.config0(nrefs=2, nptcls=6)
    mask = [1, 0, 1, 1, 0, 1]
    pc, refs, parts = setup(pkg, w, mask=mask)
    assert pc.get_nptcls() == 4
    with pytest.raises(pkg.PftccError) as e:
        pc.gencorrs(1, 2)          # masked particle: pinds(2) == 0
    assert e.value.status == 2
    with pytest.raises(pkg.PftccError) as e:
        pc.gencorrs(3, 1)          # iref out of range
    assert e.value.status == 2
    with pytest.raises(pkg.PftccError) as e:
        pc.gencorr_for_rot_8(1, 1, [0.0, 0.0], w.nrots + 1)
    assert e.value.status == 2
    # slot 2 holds global particle 4
    cc = pc.gencorrs(1, 4)
    assert cc.shape == (w.nrots,)


def test_ctf_state_error(pkg):
    w = pkg.synth.config0(nrefs=1, nptcls=1)
    pc = pkg.polarft_corrcalc()
    pc.new(1, (1, 1), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True)
    with pytest.raises(pkg.PftccError) as e:
        pc.gencorrs(1, 1)
    assert e.value.status == 3


def test_getters_and_setters(pkg):
    pc = pkg.polarft_corrcalc()
    pc.new(3, (10, 14), box=64, nrots=128, kfromto=(2, 20), ctf=False)
    assert pc.get_nrots() == 128 and pc.get_pftsz() == 64 and pc.get_pdim() == [64, 2, 20]
    assert pc.get_box() == 64 and pc.get_nrefs() == 3 and pc.get_nptcls() == 5
    assert pc.get_rot(1) == 0.0 and abs(pc.get_rot(33) - 90.0) < 1e-4
    assert pc.get_roind(359.0) == 1 and pc.get_roind(90.2) == 33
    xy = pc.get_coord(33, 10)
    assert abs(xy[0] - 10.0) < 1e-5 and abs(xy[1]) < 1e-5
    rng = np.random.default_rng(0)
    a = (rng.standard_normal((19, 64)) + 1j * rng.standard_normal((19, 64))).astype(np.complex64)
    pc.set_ref_pft(2, a, True)
    assert np.array_equal(pc.get_ref_pft(2, True), a)
    pc.cp_even2odd_ref(2)
    assert np.array_equal(pc.get_ref_pft(2, False), a)
    pc.set_ref_fcomp(2, 5, 7, 3 + 4j, True)
    assert pc.get_ref_pft(2, True)[7 - 2, 4] == np.complex64(3 + 4j)
    pc.cp_even_ref2ptcl(2, 12)
    assert np.array_equal(pc.get_ptcl_pft(12), pc.get_ref_pft(2, True))
    assert abs(pc.get_sqsum_ptcl(12) - np.sum(np.abs(pc.get_ref_pft(2, True)) ** 2)) < 1e-2
    # self correlation KAT through the device: irot 1, cc 1
    cc = pc.gencorrs(2, 12)
    assert cc.argmax() == 0 and abs(cc[0] - 1) < 1e-5
    pc.set_eo(12, False)
    assert not pc.ptcl_iseven(12)
    pc.swap_ptclsevenodd()
    assert pc.ptcl_iseven(12)
    pc.reallocate_ptcls(2, [20, 25])
    assert pc.get_nptcls() == 2
    with pytest.raises(pkg.PftccError):
        pc.get_ptcl_pft(12)
    pc.kill()
    assert not pc.exists()
