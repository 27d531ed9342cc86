"""CPU tests of the oracle's matched-filter mode (params_glob%l_match_filt,
simple_polarft_corrcalc.f90: shellnorm_and_filter_ref(_8) :756-807, prep_matchfilt :987-1095;
SavitzkyGolay_filter, simple_math.f90:3511-3588): the smoothing coefficients against the least
squares normal equations that define them, the filter's exactness on quartics, the shell
normalisation's unit power, and prep_matchfilt against an independent numpy restatement."""
import numpy as np
import pytest


def rand_pft(rng, K, P):
    return (rng.standard_normal((K, P)) + 1j * rng.standard_normal((K, P))).astype(np.complex64)


def test_savgol_coefficients_and_quartics(O):
    # the least-squares quartic through 7 equally spaced points, value at the centre
    k = np.arange(-3, 4, dtype=np.float64)
    V = np.vander(k, 5, increasing=True)
    c = np.linalg.pinv(V)[0]
    y = np.zeros(20)
    y[10] = 1.0                       # the impulse response reads the coefficients back
    out = O.savgol7(y)
    assert np.allclose(out[7:14], c[::-1], atol=1e-14)
    # a quartic is reproduced away from both ends
    x = np.arange(30, dtype=np.float64)
    q = 0.3 + 0.1 * x - 0.02 * x ** 2 + 1e-3 * x ** 3 - 2e-5 * x ** 4
    f = O.savgol7(q)
    assert np.allclose(f[3:27], q[3:27], rtol=1e-10)
    assert np.array_equal(f[27:], q[27:])            # the last three points untouched
    # the left border omits the missing points (no renormalisation)
    ones = O.savgol7(np.ones(10))
    assert abs(ones[0] - (131 + 75 - 30 + 5) / 231) < 1e-14


def test_shellnorm_unit_power(O):
    g = O.geom(128, 2, 20, 64, kstop=16)
    rng = np.random.default_rng(0)
    ref = rand_pft(rng, g.K, g.pftsz)
    opt = rng.uniform(0.2, 1.0, g.Ks).astype(np.float32)
    s = O.shellnorm_factors(g, ref, opt)
    pw = np.mean(np.abs((ref[:g.Ks].astype(np.complex128) * s[:, None])) ** 2, axis=1)
    assert np.allclose(pw, opt.astype(np.float64) ** 2, rtol=1e-6)
    z = ref.copy()
    z[3] = 0
    assert O.shellnorm_factors(g, z, opt)[3] == pytest.approx(float(opt[3]))   # pw <= 1e-12: optlp alone


def matchfilt_numpy(g, ref, ptcl, irot, ctf, optlp):
    P, N, Ks = g.pftsz, g.nrots, g.Ks
    o = np.ones(Ks) if optlp is None else optlp.astype(np.float64)
    r = ref[:Ks].astype(np.complex128) * (1.0 if ctf is None else ctf[:Ks])
    q = ptcl[:Ks].astype(np.complex128)
    norm = lambda a: np.where((np.mean(np.abs(a) ** 2, axis=1) > 1e-12)[:, None],
                              a * (o / np.sqrt(np.maximum(np.mean(np.abs(a) ** 2, axis=1), 1e-300)))[:, None],
                              a * o[:, None])
    q, r = norm(q), norm(r)
    full = np.concatenate([q, np.conj(q)], axis=1)
    qs = np.roll(full, -(irot - 1), axis=1)[:, :P]
    diff = np.mean(np.abs(r - qs) ** 2, axis=1)
    c = np.array([5, -30, 75, 131, 75, -30, 5]) / 231.0
    fit = diff.copy()
    for i in range(Ks - 3):
        fit[i] = sum(c[k + 3] * diff[i + k] for k in range(-3, 4) if i + k >= 0)
    fit = np.where(fit <= 0, diff, fit)
    fit[:3] = diff[:3]
    pwq, pwr = np.mean(np.abs(q) ** 2, axis=1), np.mean(np.abs(r) ** 2, axis=1)
    w = np.where(pwq > 1e-12, 1 / np.sqrt(pwq), 1.0)
    ss = pwr / np.where(fit > 1e-12, fit, 1.0)
    w = np.where(fit > 1e-12, w * np.sqrt(ss / (ss + 1)), w)
    out = ptcl.astype(np.complex128).copy()
    out[:Ks] = q * w[:, None]
    return out


@pytest.mark.parametrize("irot", [1, 5, 65, 128])
def test_prep_matchfilt_matches_numpy(O, irot):
    g = O.geom(128, 2, 20, 64, kstop=16)
    t = O.tables(g)
    rng = np.random.default_rng(irot)
    ref = rand_pft(rng, g.K, g.pftsz)
    ptcl = (0.6 * ref + 0.5 * rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=1.8, dfy=1.6, angast=30.0))
    opt = rng.uniform(0.3, 1.0, g.Ks).astype(np.float32)
    got = O.prep_matchfilt(g, ref, ptcl, irot, ctf, opt)
    want = matchfilt_numpy(g, ref, ptcl, irot, ctf, opt)
    assert np.max(np.abs(got - want)) < 1e-6 * np.max(np.abs(want))
    assert np.array_equal(got[g.Ks:], ptcl[g.Ks:])   # shells beyond kstop untouched


def test_prep_matchfilt_identical_pair(O):
    """a particle equal to its reference has no difference power: the filter reduces to the
    shell normalisation (unit power per shell)"""
    g = O.geom(128, 2, 20, 64)
    ref = rand_pft(np.random.default_rng(9), g.K, g.pftsz)
    got = O.prep_matchfilt(g, ref, ref, 1)
    assert np.allclose(np.mean(np.abs(got.astype(np.complex128)) ** 2, axis=1), 1.0, rtol=1e-5)


def test_pssnr_factors_and_particle_weights(O):
    """the l_pssnr branches (shellnorm_and_filter_ref :763-770; prep_matchfilt :999-1019): the
    reference's shell k scaled to power ssnr k (ssnr = ref_optlp(k)); the particle's shell k to
    power k times sqrt(1 + ssnr |CTF|^2) sample by sample"""
    g = O.geom(128, 2, 20, 64, kstop=17)
    t = O.tables(g)
    rng = np.random.default_rng(3)
    ref = rand_pft(rng, g.K, g.pftsz)
    ssnr = rng.uniform(0.1, 3.0, g.Ks).astype(np.float32)
    s = O.shellnorm_factors(g, ref, ssnr, pssnr=True)
    k = np.arange(g.kfrom, g.kstop + 1)
    pw = np.mean(np.abs(ref[:g.Ks].astype(np.complex128) * s[:, None]) ** 2, axis=1)
    assert np.allclose(pw, ssnr.astype(np.float64) * k, rtol=1e-6)
    z = ref.copy()
    z[2] = 0
    assert O.shellnorm_factors(g, z, ssnr, pssnr=True)[2] == pytest.approx(float(np.sqrt(float(ssnr[2]) * k[2])))
    ptcl = rand_pft(rng, g.K, g.pftsz)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=1.8, dfy=1.7, angast=10.0))
    got = O.prep_matchfilt_pssnr(g, ptcl, ctf, ssnr)
    q = ptcl[:g.Ks].astype(np.complex128)
    w = np.sqrt(k) / np.sqrt(np.mean(np.abs(q) ** 2, axis=1))
    want = q * w[:, None] * np.sqrt(1.0 + ssnr.astype(np.float64)[:, None] * ctf[:g.Ks] ** 2)
    assert np.allclose(got[:g.Ks], want, rtol=1e-6, atol=1e-6 * np.abs(want).max())
    assert np.array_equal(got[g.Ks:], ptcl[g.Ks:])                 # shells beyond kstop untouched
