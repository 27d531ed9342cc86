"""GPU parity tests of the Euclidean objective through the C ABI against the FP64 oracle:
gencorrs_euclid_1/_2, gencorr_euclid_for_rot(_8), gencorr_euclid_grad(_only)_for_rot_8,
gencorr_sigma_contrib (single and batched), the cc_objfun dispatch of gencorrs /
gencorr_for_rot_8 / gencorr_grad_for_rot_8 and the exact batched searches, and the error
codes.

Tolerances.  The library evaluates with its FP32 |CTF| matrices (the reference's
create_polar_absctfmats is single precision) while the oracle takes the CTF in FP64, so the
operands differ by ~1e-7 relative.  The Euclidean objective subtracts the square sums of
both operands from twice their correlation, so its error is measured against the size of
those terms: |got - want| / max_rot |want| < 1e-5 for the FP32 outputs, 2e-6 for the FP64 ones."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def setup(pkg, O, w, kstop=None, eo=None, seed=0):
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    refs = refs.numpy()
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), kstop=kstop, ctf=True,
           ctf_frame="ref", eoarr=eo)
    pc.set_refs(1, refs, True)
    pc.set_refs(1, (refs * np.complex64(0.9 - 0.1j)).astype(np.complex64), False)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    K = w.kto - w.kfrom + 1
    # noise power falling with resolution, as the group spectra of euclid_sigma2 do
    rng = np.random.default_rng(seed)
    sig = (rng.uniform(0.5, 2.0, (w.nptcls, K)) * np.linspace(4.0, 0.5, K)).astype(np.float32)
    pc.assign_sigma2_noise(sig)
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box, kstop=kstop)
    t = O.tables(g)
    return pc, refs, parts, sig, g, t


def ctf_of(O, w, g, t, parts, i):
    return O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                     float(parts.angast[i])))


def scaled_err(got, want):
    want = np.asarray(want, np.float64)
    return np.max(np.abs(np.asarray(got, np.float64) - want)) / np.max(np.abs(want))


@pytest.mark.parametrize("cfgname", ["config0", "config1"])
def test_gencorrs_euclid_matches_oracle(pkg, O, cfgname):
    w = getattr(pkg.synth, cfgname)(nrefs=2, nptcls=4)
    pc, refs, parts, sig, g, t = setup(pkg, O, w, eo=[0, 1, 0, 1])
    odd = (refs * np.complex64(0.9 - 0.1j)).astype(np.complex64)
    for i in range(4):
        c = ctf_of(O, w, g, t, parts, i)
        pft = pc.get_ptcl_pft(i + 1)
        r = refs[1] if i % 2 == 0 else odd[1]
        for sh in (None, [0.75, -1.25]):
            want = O.gencorrs_euclid(g, t, r, pft, sig[i].astype(np.float64), c, sh)
            got = pc.gencorrs_euclid(2, i + 1, sh)
            assert scaled_err(got, want) < 1e-5
            assert got.argmax() == want.argmax() or abs(want[got.argmax()] - want.max()) < 1e-5 * np.abs(want).max()
    # cc_objfun dispatch: gencorrs serves gencorrs_euclid_1/_2
    pc.set_objfun(pkg._lib.OBJFUN_EUCLID)
    assert np.array_equal(pc.gencorrs(1, 3), pc.gencorrs_euclid(1, 3))
    assert np.array_equal(pc.gencorrs(1, 3, [0.5, 0.5]), pc.gencorrs_euclid(1, 3, [0.5, 0.5]))
    pc.set_objfun(pkg._lib.OBJFUN_CC)
    assert abs(pc.gencorrs(1, 3).max()) <= 1.0
    pc.kill()


def test_euclid_for_rot_and_gradient(pkg, O):
    w = pkg.synth.config0(nrefs=2, nptcls=3)
    pc, refs, parts, sig, g, t = setup(pkg, O, w, kstop=20, seed=1)
    for i in range(3):
        c = ctf_of(O, w, g, t, parts, i)
        pft = pc.get_ptcl_pft(i + 1)
        scale = np.abs(O.gencorrs_euclid(g, t, refs[0], pft, sig[i].astype(np.float64), c, None)).max()
        for irot in (1, 40, 64, 65, 128):
            sh = np.array([0.7, -0.3])
            fo, go = O.gencorr_euclid_grad_for_rot(g, t, refs[0], pft, irot, sig[i].astype(np.float64), c, sh)
            f8 = pc.gencorr_euclid_for_rot_8(1, i + 1, sh, irot)
            assert abs(f8 - fo) < 2e-6 * abs(fo) + 1e-9 * scale
            assert abs(pc.gencorr_euclid_for_rot(1, i + 1, sh, irot) - fo) < 1e-5 * abs(fo)
            f, gr = pc.gencorr_euclid_grad_for_rot_8(1, i + 1, sh, irot)
            assert f == f8
            assert np.max(np.abs(gr - go)) < 2e-6 * max(1.0, np.max(np.abs(go)), abs(fo))
            assert np.array_equal(pc.gencorr_euclid_grad_only_for_rot_8(1, i + 1, sh, irot), gr)
    # cc_objfun dispatch of the single-rotation correlators
    pc.set_objfun(pkg._lib.OBJFUN_EUCLID)
    sh = np.array([0.2, 0.4])
    assert pc.gencorr_for_rot_8(2, 2, sh, 17) == pc.gencorr_euclid_for_rot_8(2, 2, sh, 17)
    f, gr = pc.gencorr_grad_for_rot_8(2, 2, sh, 17)
    fe, ge = pc.gencorr_euclid_grad_for_rot_8(2, 2, sh, 17)
    assert f == fe and np.array_equal(gr, ge)
    pc.kill()


def test_sigma_contrib(pkg, O):
    w = pkg.synth.config0(nrefs=2, nptcls=3)
    pc, refs, parts, sig, g, t = setup(pkg, O, w, kstop=18, seed=2)
    reqs = [(1, 1, 1, 0.0, 0.0), (2, 2, 50, 0.5, -1.0), (1, 3, 128, -1.5, 0.25)]
    ir, ip, ro, sx, sy = (np.array(v) for v in zip(*reqs))
    sc_b, ps_b, rs_b = pc.sigma_contrib_batch(ir, ip, ro, np.stack([sx, sy], 1))
    for n, (r, i, irot, x, y) in enumerate(reqs):
        c = ctf_of(O, w, g, t, parts, i - 1)
        pft = pc.get_ptcl_pft(i)
        sc, ps, rs = O.sigma_contrib(g, t, refs[r - 1], pft, irot, c, (x, y))
        assert sc.shape == (g.K,)   # every shell kfrom..kto, beyond kstop too
        got = pc.gencorr_sigma_contrib(r, i, [x, y], irot)
        for a, b in zip(got, (sc, ps, rs)):
            assert np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-3 * np.abs(b).max())) < 1e-5
        assert np.array_equal(got[0], sc_b[n]) and np.array_equal(got[1], ps_b[n]) and np.array_equal(got[2], rs_b[n])
    pc.kill()


def test_euclid_batched_exact_search(pkg, O):
    """corr_all / search_best (exact) under OBJFUN_EUCLID equal the per-pair gencorrs_euclid
    and their maxloc; in the reference frame the FP32 / BF16 m-domain paths refuse it"""
    w = pkg.synth.config0(nrefs=4, nptcls=5)
    pc, refs, parts, sig, g, t = setup(pkg, O, w, seed=3)
    pc.set_objfun(pkg._lib.OBJFUN_EUCLID)
    shifts = np.array([[0, 0], [0.5, -1.0]], np.float32)
    cc = pc.corr_all(shifts)
    for i in range(5):
        for r in range(4):
            for s in range(2):
                assert np.array_equal(cc[i, r, s], pc.gencorrs_euclid(r + 1, i + 1, shifts[s]))
    best = pc.search_best(shifts, "exact")
    flat = cc.reshape(5, -1)
    for i in range(5):
        j = int(np.argmax(flat[i]))
        r, s, rot = np.unravel_index(j, (4, 2, w.nrots))
        assert (best["iref"][i], best["ishift"][i], best["irot"][i]) == (r + 1, s, rot + 1)
        assert best["corr"][i] == flat[i, j]
    with pytest.raises(pkg.PftccError) as e:
        pc.search_best(shifts, "fp32")
    assert e.value.status == pkg._lib.ERR_UNSUPPORTED
    pc.kill()


def test_euclid_state_errors(pkg, O):
    w = pkg.synth.config0(nrefs=1, nptcls=3)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    pc = pkg.polarft_corrcalc()
    pc.new(1, (1, 3), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=False, ctf_frame="ref")
    pc.set_refs(1, refs.numpy(), True)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    # no sigma2 yet
    with pytest.raises(pkg.PftccError) as e:
        pc.gencorrs_euclid(1, 1)
    assert e.value.status == pkg._lib.ERR_STATE
    pc.set_objfun(pkg._lib.OBJFUN_EUCLID)
    with pytest.raises(pkg.PftccError) as e:
        pc.gencorrs(1, 1)
    assert e.value.status == pkg._lib.ERR_STATE
    K = w.kto - w.kfrom + 1
    # a range that misses particle 3
    pc.assign_sigma2_noise(np.ones((2, K), np.float32))
    with pytest.raises(pkg.PftccError) as e:
        pc.gencorrs(1, 1)
    assert e.value.status == pkg._lib.ERR_STATE
    pc.assign_sigma2_noise(np.ones((3, K), np.float32))
    a = pc.gencorrs(1, 2)
    assert np.all(np.isfinite(a)) and a.max() <= 0.0
    # sigma_contrib needs no sigma2, the Euclidean objective needs the reference frame
    pc.kill()
    # in the particle frame the Euclidean objective is the m-domain search's: the exact calls refuse
    pc = pkg.polarft_corrcalc()
    pc.new(1, (1, 3), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=False, ctf_frame="ptcl")
    pc.set_refs(1, refs.numpy(), True)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    pc.set_objfun(pkg._lib.OBJFUN_EUCLID)
    pc.assign_sigma2_noise(np.ones((3, K), np.float32))
    for call in (lambda: pc.gencorrs(1, 1), lambda: pc.search_best(None, "exact"), lambda: pc.corr_all(None)):
        with pytest.raises(pkg.PftccError) as e:
            call()
        assert e.value.status == pkg._lib.ERR_UNSUPPORTED
    pc.kill()


def test_mdomain_euclid_matches_oracle(pkg, O):
    """the m-domain search under OBJFUN_EUCLID (particle CTF frame: shell weights on the particle
    spectra and the CTF^2 spectra, the additive normaliser): every value of corr_all_prec against
    the oracle's particle-frame objective (2e-5 of the row's largest magnitude in FP32, 2e-4 with
    the BF16 hi+lo products), and search_best with the FP32 re-score of the top 8 at the argmax"""
    w = pkg.synth.config0(nrefs=4, nptcls=6)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    refs = refs.numpy()
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame="ptcl")
    try:
        pc.set_refs(1, refs, True)
        pc.set_refs(1, refs, False)
        pc.polarize_ptcls(0, parts.cmat.numpy())
        pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                       dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
        K = w.kto - w.kfrom + 1
        rng = np.random.default_rng(5)
        sig = (rng.uniform(0.5, 2.0, (w.nptcls, K)) * np.linspace(4.0, 0.5, K)).astype(np.float32)
        pc.assign_sigma2_noise(sig)
        pc.set_objfun(pkg._lib.OBJFUN_EUCLID)
        shifts = np.array([[0, 0], [0.5, -1.0], [-1.5, 1.0]], np.float32)
        g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
        t = O.tables(g)
        want = np.zeros((w.nptcls, w.nrefs, len(shifts), w.nrots))
        for i in range(w.nptcls):
            c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(parts.dfx[i]), float(parts.dfy[i]),
                                          float(parts.angast[i])))
            pft = pc.get_ptcl_pft(i + 1)
            for r in range(w.nrefs):
                for s in range(len(shifts)):
                    want[i, r, s] = O.gencorrs_euclid_ptclframe(g, t, refs[r], pft, sig[i].astype(np.float64), c,
                                                                shifts[s].astype(np.float64))
        for prec, tol in (("fp32", 2e-5), ("bf16x3", 2e-4)):
            got = pc.corr_all_prec(shifts, prec)
            err = np.max(np.abs(got - want), axis=-1) / np.max(np.abs(want), axis=-1)
            print(f"m-domain Euclid {prec}: max error {err.max():.2e} of the row's scale")
            assert err.max() < tol
            best = pc.search_best(shifts, prec, ntop=8)
            for i in range(w.nptcls):
                flat = want[i].ravel()
                got_v = want[i, best["iref"][i] - 1, best["ishift"][i], best["irot"][i] - 1]
                assert got_v >= flat.max() - 1e-5 * np.abs(flat).max()
                assert abs(best["corr"][i] - got_v) < 2e-5 * np.abs(flat).max()
    finally:
        pc.kill()
