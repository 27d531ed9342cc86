"""CPU tests of the oracle's Euclidean objective (cc_objfun = OBJFUN_EUCLID,
simple_polarft_corrcalc.f90: gencorrs_euclid_1/_2 :1536-1592, calc_euclid_for_rot_8 :1308-1334,
gencorr_euclid_grad_for_rot_8 :2071-2109, gencorr_sigma_contrib :2150-2188,
setup_pxls_p_shell :879-893).

Each routine is checked against an independent numpy restatement of the reference's
formula (the difference form sum |ref_prep - ptcl~|^2 that calc_euclid_for_rot evaluates),
against the other routines (the expanded correlation form of gencorrs_euclid equals the
difference form; sigma_contrib reproduces gencorrs_euclid), and the gradient against
central differences of f."""
import numpy as np
import pytest

GEOMS = [(128, 2, 20, 64, 16), (360, 2, 40, 128, 40)]


def rand_pft(rng, K, P):
    return (rng.standard_normal((K, P)) + 1j * rng.standard_normal((K, P))).astype(np.complex64)


def setup(O, geom, seed=0):
    g = O.geom(*geom[:4], kstop=geom[4])
    t = O.tables(g)
    rng = np.random.default_rng(seed)
    ref = rand_pft(rng, g.K, g.pftsz)
    ptcl = (0.5 * ref + 0.8 * rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=2.1, dfy=1.9, angast=25.0))
    sigma2 = rng.uniform(0.5, 3.0, g.K)
    return g, t, ref, ptcl, ctf, sigma2


def prepared(O, g, t, ref, ctf, shvec):
    a = ref.astype(np.complex128) * ctf
    if shvec is not None:
        a = a * O.shmat(g, t, *shvec)
    return a


def diffsq(g, a, ptcl, irot):
    """per-shell sum_n |a(n) - ptcl~(n + irot - 1)|^2, ptcl~ the conjugate-extended particle"""
    full = np.concatenate([ptcl, np.conj(ptcl)], axis=1).astype(np.complex128)
    q = np.roll(full, -(irot - 1), axis=1)[:, :g.pftsz]
    return np.sum(np.abs(a - q) ** 2, axis=1)


def test_pxls_p_shell_counts(O):
    g = O.geom(128, 2, 40, 128)
    want = np.zeros(g.K)
    for h in range(1, g.kto + 1):
        for k in range(1, g.kto + 1):
            sh = int(np.floor(np.sqrt(h * h + k * k) + 0.5))
            if g.kfrom <= sh <= g.kto:
                want[sh - g.kfrom] += 1
    assert np.array_equal(O.pxls_p_shell(g), want)
    # a quarter annulus of radius k holds about pi k / 2 pixels
    k = np.arange(g.kfrom, g.kto + 1)
    assert np.all(np.abs(want[5:] / (np.pi * k[5:] / 2) - 1) < 0.2)


@pytest.mark.parametrize("geom", GEOMS)
@pytest.mark.parametrize("shvec", [None, (0.8, -1.3)])
def test_gencorrs_euclid_is_weighted_distance(O, geom, shvec):
    """gencorrs_euclid(irot) = -sum_{k<=kstop} pxls(k)/P |ref_prep - ptcl~_irot|^2 / (2 sigma2(k))"""
    g, t, ref, ptcl, ctf, sigma2 = setup(O, geom)
    got = O.gencorrs_euclid(g, t, ref, ptcl, sigma2, ctf, shvec)
    a = prepared(O, g, t, ref, ctf, shvec)
    w = O.pxls_p_shell(g)[:g.Ks] / g.pftsz / (2 * sigma2[:g.Ks])
    for irot in (1, 2, 17, g.pftsz, g.pftsz + 1, g.pftsz + 5, g.nrots):
        want = -np.sum(w * diffsq(g, a, ptcl, irot)[:g.Ks])
        assert abs(got[irot - 1] - want) <= 1e-10 * abs(want)


@pytest.mark.parametrize("geom", GEOMS)
def test_euclid_for_rot_and_gradient(O, geom):
    """f = -sum k pxls/P |d|^2/(2 sigma2) over k <= kstop; grad equals central differences"""
    g, t, ref, ptcl, ctf, sigma2 = setup(O, geom, seed=1)
    pxls = O.pxls_p_shell(g)
    k = np.arange(g.kfrom, g.kto + 1)
    sh = np.array([0.6, -0.9])
    for irot in (1, 9, g.pftsz + 3):
        f, gr = O.gencorr_euclid_grad_for_rot(g, t, ref, ptcl, irot, sigma2, ctf, sh)
        a = prepared(O, g, t, ref, ctf, sh)
        want = -np.sum((k * pxls / g.pftsz * diffsq(g, a, ptcl, irot) / (2 * sigma2))[:g.Ks])
        assert abs(f - want) <= 1e-10 * abs(want)
        h = 1e-5
        for d in range(2):
            e = np.zeros(2)
            e[d] = h
            fp, _ = O.gencorr_euclid_grad_for_rot(g, t, ref, ptcl, irot, sigma2, ctf, sh + e)
            fm, _ = O.gencorr_euclid_grad_for_rot(g, t, ref, ptcl, irot, sigma2, ctf, sh - e)
            fd = (fp - fm) / (2 * h)
            assert abs(gr[d] - fd) <= 1e-5 * max(1.0, abs(fd))


@pytest.mark.parametrize("geom", GEOMS)
def test_sigma_contrib(O, geom):
    """sigma_contrib(k) = |d|^2/(2P) over all shells; -sum_{k<=kstop} pxls/sigma2 * sigma_contrib
    reproduces gencorrs_euclid at that rotation"""
    g, t, ref, ptcl, ctf, sigma2 = setup(O, geom, seed=2)
    sh = (1.1, 0.4)
    for irot in (1, 33, g.pftsz + 1, g.nrots):
        sc, ps, rs = O.sigma_contrib(g, t, ref, ptcl, irot, ctf, sh)
        a = prepared(O, g, t, ref, ctf, sh)
        assert np.allclose(sc, 0.5 * diffsq(g, a, ptcl, irot) / g.pftsz, rtol=1e-12)
        assert np.allclose(ps, np.sum(np.abs(ptcl.astype(np.complex128)) ** 2, axis=1), rtol=1e-12)
        assert np.allclose(rs, np.sum(np.abs(a) ** 2, axis=1), rtol=1e-12)
        eu = O.gencorrs_euclid(g, t, ref, ptcl, sigma2, ctf, sh)[irot - 1]
        via = -np.sum((O.pxls_p_shell(g) / sigma2 * sc)[:g.Ks])
        assert abs(eu - via) <= 1e-10 * abs(eu)


@pytest.mark.parametrize("j", [0, 7, 70, 200])
def test_euclid_recovers_rotation_and_shift(O, j):
    """a noisy copy of the reference rotated by j samples and shifted peaks at irot = j + 1
    when the reference is prepared with the opposite shift"""
    g = O.geom(360, 2, 40, 128)
    t = O.tables(g)
    rng = np.random.default_rng(10 + j)
    P, N = g.pftsz, g.nrots
    ref = rand_pft(rng, g.K, P)
    sh = np.array([1.5, -0.75])
    moved = (ref.astype(np.complex128) * O.shmat(g, t, *sh))
    full = np.concatenate([moved, np.conj(moved)], axis=1)
    ptcl = (np.roll(full, j % N, axis=1)[:, :P] + 0.3 * rand_pft(rng, g.K, P)).astype(np.complex64)
    sigma2 = np.full(g.K, 0.09)
    eu = O.gencorrs_euclid(g, t, ref, ptcl, sigma2, None, sh)
    assert eu.argmax() == j % N
    assert eu.max() <= 0.0


@pytest.mark.parametrize("geom", GEOMS)
def test_particle_frame_euclid(O, geom):
    """the particle-frame objective equals gencorrs_euclid_2 for an isotropic CTF and without
    CTF, equals its expanded form sum_k w_k (corr_k - (E_ref,k(rot) + E_ptcl,k) / 2) with the
    reference energy taken at the particle's CTF, and differs from the reference frame for an
    astigmatic CTF"""
    g, t, ref, ptcl, ctf, sigma2 = setup(O, geom, seed=4)
    sh = (0.6, -0.4)
    iso = O.ctfmat(g, t, O.make_ctf(dfx=2.0, dfy=2.0))
    # an isotropic CTF on the polar grid varies with the angle only through the FP32 grid
    # coordinates (k^2 = x^2 + y^2 to rounding): agreement to that level
    for c, tol in ((None, 1e-10), (iso, 1e-6)):
        a = O.gencorrs_euclid_ptclframe(g, t, ref, ptcl, sigma2, c, sh)
        b = O.gencorrs_euclid(g, t, ref, ptcl, sigma2, c, sh)
        assert np.max(np.abs(a - b)) < tol * np.max(np.abs(b))
    got = O.gencorrs_euclid_ptclframe(g, t, ref, ptcl, sigma2, ctf, sh)
    P, N = g.pftsz, g.nrots
    A = ref.astype(np.complex128) * O.shmat(g, t, *sh)
    full = np.concatenate([ptcl, np.conj(ptcl)], axis=1).astype(np.complex128)
    cfull = np.concatenate([ctf, ctf], axis=1)
    w = O.pxls_p_shell(g) / P / sigma2
    for s in (0, 5, P, N - 1):
        q = np.roll(full, -s, axis=1)[:, :P]
        c = np.roll(cfull, -s, axis=1)[:, :P]
        corr = np.sum((A * c * np.conj(q)).real, axis=1)
        eref = np.sum(np.abs(ref.astype(np.complex128)) ** 2 * c ** 2, axis=1)
        eptcl = np.sum(np.abs(ptcl.astype(np.complex128)) ** 2, axis=1)
        want = np.sum((w * (corr - 0.5 * (eref + eptcl)))[:g.Ks])
        assert abs(got[s] - want) < 1e-10 * abs(want)
    ref_frame = O.gencorrs_euclid(g, t, ref, ptcl, sigma2, ctf, sh)
    assert np.max(np.abs(got - ref_frame)) > 1e-6 * np.max(np.abs(ref_frame))
