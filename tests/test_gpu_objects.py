"""GPU tests of the object's remaining procedures through the C ABI: cp_refs (:491-495),
set_ptcl_fcomp (:471-476), calc_ptcl_pspec (:897-904), assign_pinds (:706-710) and
calc_roinv_corrmat (:2207-2231), the last against the per-pair gencorrs maxloc it is defined by."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def rand_pfts(rng, n, K, P):
    return (rng.standard_normal((n, K, P)) + 1j * rng.standard_normal((n, K, P))).astype(np.complex64)


def test_cp_refs_fcomp_pspec_pinds(pkg):
    K, P = 13, 32
    rng = np.random.default_rng(0)
    a, b = pkg.polarft_corrcalc(), pkg.polarft_corrcalc()
    a.new(3, (5, 7), box=64, nrots=2 * P, kfromto=(2, 14), ctf=False, ptcl_mask=[1, 0, 1])
    b.new(3, (1, 2), box=64, nrots=2 * P, kfromto=(2, 14), ctf=False)
    try:
        refs = rand_pfts(rng, 3, K, P)
        a.set_refs(1, refs, True)
        a.set_refs(1, (refs * 0.5).astype(np.complex64), False)
        b.cp_refs(a)
        for r in range(3):
            assert np.array_equal(b.get_ref_pft(r + 1, True), refs[r])
            assert np.array_equal(b.get_ref_pft(r + 1, False), (refs[r] * 0.5).astype(np.complex64))
        assert list(a.assign_pinds()) == [1, 0, 2]
        p = rand_pfts(rng, 1, K, P)[0]
        a.set_ptcl_pft(7, p)
        sq = a.get_sqsum_ptcl(7)
        a.set_ptcl_fcomp(7, 5, 3, 2.5 - 1.5j)
        got = a.get_ptcl_pft(7)
        assert got[3 - 2, 5 - 1] == np.complex64(2.5 - 1.5j)
        assert np.array_equal(np.delete(got.ravel(), (3 - 2) * P + 4), np.delete(p.ravel(), (3 - 2) * P + 4))
        assert a.get_sqsum_ptcl(7) == sq     # not refreshed, as in the reference
        want = np.mean(np.abs(got.astype(np.complex128)) ** 2, axis=1)
        assert np.allclose(a.calc_ptcl_pspec(7), want, rtol=1e-6)
        with pytest.raises(pkg.PftccError) as e:
            a.set_ptcl_fcomp(7, P + 1, 3, 1.0)
        assert e.value.status == pkg._lib.ERR_INDEX
    finally:
        a.kill()
        b.kill()


def test_calc_roinv_corrmat(pkg):
    w = pkg.synth.config0(nrefs=5, nptcls=5)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    pc = pkg.polarft_corrcalc()
    pc.new(5, (1, 5), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=False)
    try:
        pc.set_refs(1, refs.numpy(), True)
        pc.set_refs(1, refs.numpy(), False)
        pc.polarize_ptcls(0, parts.cmat.numpy())
        m = pc.calc_roinv_corrmat()
        assert np.array_equal(m, m.T) and np.all(np.diag(m) == 1.0)
        for i in range(5):
            for j in range(i + 1, 5):
                assert m[i, j] == pc.gencorrs(i + 1, j + 1).max()
    finally:
        pc.kill()
    pc = pkg.polarft_corrcalc()
    pc.new(2, (1, 3), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=False)
    with pytest.raises(pkg.PftccError) as e:
        pc.calc_roinv_corrmat()
    assert e.value.status == pkg._lib.ERR_ARG
    pc.kill()
