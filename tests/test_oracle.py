"""CPU tests of the oracle: known-answer tests derived from the reference's formulas.

The reference ships no golden vectors for this path and cannot be compiled here,
so the oracle is pinned by properties the reference's code implies (see the
citations in oracle/pftcc_oracle.c)."""
import math

import numpy as np
import pytest

GEOMS = [(128, 2, 20, 64), (360, 2, 40, 128)]


def rand_pft(rng, K, P):
    return (rng.standard_normal((K, P)) + 1j * rng.standard_normal((K, P))).astype(np.complex64)


@pytest.mark.parametrize("n", [2, 3, 4, 5, 12, 64, 180, 300, 360, 600, 7 * 11])
def test_fft_matches_numpy(O, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    assert np.allclose(O.cfft(x, -1), np.fft.fft(x), atol=1e-11 * n)
    assert np.allclose(O.cfft(x, +1), np.fft.ifft(x) * n, atol=1e-11 * n)


@pytest.mark.parametrize("geom", GEOMS)
def test_fft_path_equals_direct_sums(O, geom):
    """calc_corrs_over_k (FFT path, FP32) == calc_corr_for_rot_8 sums (FP64) for every rotation"""
    g = O.geom(*geom)
    t = O.tables(g)
    rng = np.random.default_rng(1)
    ref = rand_pft(rng, g.K, g.pftsz)
    ptcl = (0.4 * ref + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=2.05, dfy=1.95, angast=30.0))
    for sh in ([0.0, 0.0], [0.7, -1.2]):
        want = O.gencorrs(g, t, ref, ptcl, ctf, sh)
        got = O.FFTPath(g).gencorrs(ref, ptcl, ctf, sh)
        assert np.max(np.abs(got - want) / np.maximum(np.abs(want), 1e-3)) < 1e-4
        assert np.max(np.abs(got - want)) < 1e-6


@pytest.mark.parametrize("geom", GEOMS)
def test_self_correlation_is_one_at_zero_rotation(O, geom):
    """gencorrs(ref, ref) without CTF or shift: argmax irot = 1 and cc = 1 (normalisation :1499)"""
    g = O.geom(*geom)
    t = O.tables(g)
    ref = rand_pft(np.random.default_rng(2), g.K, g.pftsz)
    cc = O.gencorrs(g, t, ref, ref)
    assert cc.argmax() == 0
    assert abs(cc[0] - 1.0) < 1e-12


@pytest.mark.parametrize("geom", GEOMS)
@pytest.mark.parametrize("j", [1, 5, 63, 64, 100])
def test_rotation_moves_argmax(O, geom, j):
    """a particle rotated by j samples (ptcl~(n) = ref~(n - j), conj wrap at P) peaks at irot = j + 1"""
    g = O.geom(*geom)
    t = O.tables(g)
    P, N = g.pftsz, g.nrots
    ref = rand_pft(np.random.default_rng(3), g.K, P)
    full = np.concatenate([ref, np.conj(ref)], axis=1)
    ptcl = np.roll(full, j % N, axis=1)[:, :P]
    cc = O.gencorrs(g, t, ref, ptcl)
    assert cc.argmax() == j % N
    assert abs(cc.max() - 1.0) < 1e-6


def test_isotropic_ctf_frames_agree(O):
    """with dfx == dfy the particle-frame objective equals gencorrs_cc_2 to rounding"""
    g = O.geom(360, 2, 40, 128)
    t = O.tables(g)
    rng = np.random.default_rng(4)
    ref = rand_pft(rng, g.K, g.pftsz)
    ptcl = (0.3 * ref + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=2.0, dfy=2.0))
    a = O.gencorrs(g, t, ref, ptcl, ctf, [0.5, 1.5])
    b = O.gencorrs_ptclframe(g, t, ref, ptcl, ctf, [0.5, 1.5])
    assert np.max(np.abs(a - b)) < 1e-6


def test_shift_gradient_matches_finite_differences(O):
    """gencorr_cc_grad_for_rot_8 (both branches) against central differences, step 1e-4 px"""
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    rng = np.random.default_rng(5)
    ref = rand_pft(rng, g.K, g.pftsz)
    ptcl = (0.5 * ref + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=2.05, dfy=1.95, angast=30.0))
    h = 1e-4
    for mf in (False, True):
        for irot in (1, 7, 70):
            sh = np.array([0.3, -0.8])
            f, g3 = O.gencorr_grad3(g, t, ref, ptcl, irot, ctf, None, sh, mf)
            assert abs(f - O.gencorr_for_rot(g, t, ref, ptcl, irot, ctf, sh, mf)) < 1e-13
            for d in range(2):
                e = np.zeros(2)
                e[d] = h
                fd = (O.gencorr_for_rot(g, t, ref, ptcl, irot, ctf, sh + e, mf)
                      - O.gencorr_for_rot(g, t, ref, ptcl, irot, ctf, sh - e, mf)) / (2 * h)
                assert abs(fd - g3[d]) < 1e-6 * max(1.0, abs(fd))


def test_defocus_gradient_matches_finite_differences(O):
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    rng = np.random.default_rng(6)
    ref = rand_pft(rng, g.K, g.pftsz)
    ptcl = (0.5 * ref + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
    c = O.make_ctf(dfx=2.25, dfy=1.75, angast=30.0)   # exactly representable in float32
    ctf, dctf = O.ctfmat(g, t, c), O.dctfmat_ddf(g, t, c)
    h = 2.0 ** -12
    cp = O.ctfmat(g, t, O.make_ctf(dfx=2.25 + h, dfy=1.75 + h, angast=30.0))
    cm = O.ctfmat(g, t, O.make_ctf(dfx=2.25 - h, dfy=1.75 - h, angast=30.0))
    for mf in (False, True):
        f, g3 = O.gencorr_grad3(g, t, ref, ptcl, 9, ctf, dctf, [0.2, 0.1], mf)
        fd = (O.gencorr_for_rot(g, t, ref, ptcl, 9, cp, [0.2, 0.1], mf)
              - O.gencorr_for_rot(g, t, ref, ptcl, 9, cm, [0.2, 0.1], mf)) / (2 * h)
        assert abs(fd - g3[2]) < 2e-3 * max(1.0, abs(fd))


def test_kweighted_equals_unweighted_for_one_shell(O):
    """the two branches of gencorr_cc_for_rot_8 agree when K = 1 (the shell weight cancels)"""
    g = O.geom(128, 7, 7, 64)
    t = O.tables(g)
    rng = np.random.default_rng(7)
    ref, ptcl = rand_pft(rng, 1, 64), rand_pft(rng, 1, 64)
    for irot in (1, 33, 100):
        a = O.gencorr_for_rot(g, t, ref, ptcl, irot, None, [0.4, 0.1], True)
        b = O.gencorr_for_rot(g, t, ref, ptcl, irot, None, [0.4, 0.1], False)
        assert abs(a - b) < 1e-12


def test_for_rot_matchfilt_equals_gencorrs(O):
    g = O.geom(360, 2, 40, 128)
    t = O.tables(g)
    rng = np.random.default_rng(8)
    ref, ptcl = rand_pft(rng, g.K, g.pftsz), rand_pft(rng, g.K, g.pftsz)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=1.5, dfy=1.4, angast=10.0))
    cc = O.gencorrs(g, t, ref, ptcl, ctf, [1.0, 0.5])
    for irot in (1, 91, 181, 300):
        assert abs(O.gencorr_for_rot(g, t, ref, ptcl, irot, ctf, [1.0, 0.5], True) - cc[irot - 1]) < 1e-12


def test_shmat_recurrence_matches_analytic(O):
    """gen_shmat_8's de Moivre recurrence equals exp(i*(argtransf_x*sx + argtransf_y*sy))"""
    g = O.geom(360, 2, 40, 128)
    t = O.tables(g)
    sx, sy = 1.7, -2.3
    sh = O.shmat(g, t, sx, sy)
    P = g.pftsz
    arg = t.argtransf[:, :P] * sx + t.argtransf[:, P:] * sy
    assert np.max(np.abs(sh - np.exp(1j * arg))) < 1e-6


def test_kb_weights_and_plane_wave(O, pkg):
    """KB window: symmetric, zero outside the half-width, normalised taps reproduce a
    constant and a slowly varying plane wave at the polar nodes (init_polarizer :87)"""
    assert O.kb_apod(1.6) == 0.0 and O.kb_apod(-1.6) == 0.0
    assert abs(O.kb_apod(0.3) - O.kb_apod(-0.3)) < 1e-15
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    box = 64
    cmat = np.ones((box, box // 2 + 1), np.complex64)
    pft = O.polarize(g, t, cmat)
    assert np.max(np.abs(pft - 1.0)) < 1e-12
    # slowly varying field F(h,k) = exp(i*0.05*(h + 2k)), Hermitian by construction
    hh = np.arange(box // 2 + 1)
    kk = np.arange(box)
    kk = np.where(kk >= box // 2, kk - box, kk)
    H, Kc = np.meshgrid(hh, kk)
    cmat = np.exp(1j * 0.05 * (H + 2 * Kc)).astype(np.complex64)
    pft = O.polarize(g, t, cmat)
    x, y = pkg.synth.polar_tables(pkg.synth.config0())
    want = np.exp(1j * 0.05 * (x + 2 * y))
    assert np.max(np.abs(pft - want)) < 5e-3


def test_generator_kat_rotation_and_shift(O, pkg):
    """noise- and CTF-free particles polarized by the oracle peak at the generating
    in-plane angle when the reference is shifted by -(R(-psi) t)"""
    w = pkg.synth.config0(nrefs=3, nptcls=4)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R, noise=False, ctf=False)
    g = O.geom(w.nrots, w.kfrom, w.kto, w.box)
    t = O.tables(g)
    for i in range(w.nptcls):
        pft = O.polarize(g, t, parts.cmat[i].numpy()).astype(np.complex64)
        psi = math.radians(parts.psi[i])
        tx, ty = parts.shift[i]
        sh = [-(math.cos(psi) * tx + math.sin(psi) * ty), -(-math.sin(psi) * tx + math.cos(psi) * ty)]
        cc = O.gencorrs(g, t, refs[parts.ref[i]].numpy(), pft, None, sh)
        expect = parts.psi[i] * w.nrots / 360.0
        d = abs(cc.argmax() - expect)
        assert min(d, w.nrots - d) <= 1.0
        assert cc.max() > 0.8


def test_cpu_search_finds_best(O):
    """the OpenMP FFT-path search returns the maxloc over refs x shifts x rotations of gencorrs"""
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    rng = np.random.default_rng(9)
    refs = np.stack([rand_pft(rng, g.K, g.pftsz) for _ in range(3)])
    ptcls = np.stack([(0.5 * refs[i % 3] + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64) for i in range(4)])
    ctfs = np.stack([O.ctfmat(g, t, O.make_ctf(dfx=1.5 + 0.1 * i, dfy=1.45 + 0.1 * i, angast=20.0)) for i in range(4)])
    shifts = np.array([[0, 0], [0.5, 0], [0, -0.5]], np.float32)
    br, bro, bs, bcc, used = O.cpu_search(g, refs, ptcls, ctfs, shifts, nthreads=2)
    assert used >= 1
    for i in range(4):
        allcc = np.array([[O.gencorrs(g, t, refs[r], ptcls[i], ctfs[i], shifts[s].astype(np.float64))
                           for s in range(3)] for r in range(3)])
        r, s, rot = np.unravel_index(np.argmax(allcc), allcc.shape)
        assert (br[i], bs[i], bro[i]) == (r, s, rot + 1)
        assert abs(bcc[i] - allcc.max()) < 1e-5


@pytest.mark.parametrize("geom", GEOMS)
def test_specscore_self_is_one(O, geom):
    """genfrc of a reference with itself at irot = 1: every shell FRC is 1, specscore 1"""
    g = O.geom(*geom)
    t = O.tables(g)
    ref = rand_pft(np.random.default_rng(21), g.K, g.pftsz)
    frc = O.genfrc(g, t, ref, ref, 1)
    assert np.allclose(frc, 1.0, atol=1e-12)
    assert abs(O.specscore(g, t, ref, ref, 1) - 1.0) < 1e-12


@pytest.mark.parametrize("geom", GEOMS)
def test_genfrc_shells_recombine_to_gencorrs(O, geom):
    """sum_k frc_k sqrt(|p_k|^2 |r_k|^2) / sqrt(sum|p|^2 sum|r|^2) = gencorrs at that rotation
    (both are the same per-shell sums, calc_k_corrs / calc_corrs_over_k), with CTF and shift"""
    g = O.geom(*geom)
    t = O.tables(g)
    rng = np.random.default_rng(22)
    ref = rand_pft(rng, g.K, g.pftsz)
    ptcl = (0.5 * ref + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=1.9, dfy=1.7, angast=10.0))
    sh = [0.6, -0.9]
    cc = O.gencorrs(g, t, ref, ptcl, ctf, sh)
    prep = ref.astype(np.complex128) * ctf * O.shmat(g, t, *sh)
    sp = np.sum(np.abs(ptcl.astype(np.complex128)) ** 2, axis=1)
    sr = np.sum(np.abs(prep) ** 2, axis=1)
    for irot in (1, 7, g.nrots // 2 + 3):
        frc = O.genfrc(g, t, ref, ptcl, irot, ctf, sh)
        rec = np.sum(frc * np.sqrt(sp * sr)) / math.sqrt(sp.sum() * sr.sum())
        assert abs(rec - cc[irot - 1]) < 1e-12


@pytest.mark.parametrize("kto", [20, 21])
def test_specscore_is_clamped_median(O, kto):
    """odd and even shell counts: the middle value / the mean of the two middle values
    (median_nocopy), clamped at zero"""
    g = O.geom(128, 2, kto, 64)
    t = O.tables(g)
    rng = np.random.default_rng(23 + kto)
    ref = rand_pft(rng, g.K, g.pftsz)
    for mix in (0.8, 0.0):
        ptcl = (mix * ref + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
        for irot in (1, 40):
            frc = O.genfrc(g, t, ref, ptcl, irot)
            assert abs(O.specscore(g, t, ref, ptcl, irot) - max(0.0, float(np.median(frc)))) < 1e-14


def test_snhc_first_improvement_and_greedy_fallback(O):
    """srch_snhc + shcloc: with prev_corr below everything the first visited (non-empty)
    reference improves and its rotation is the draw's pick among all rotations; with
    prev_corr above everything no reference improves and the greedy best over the first
    nrefs_bound visited references is kept; empty classes count against the bound"""
    rng = np.random.default_rng(31)
    nrefs, nrots = 12, 40
    corrs = rng.uniform(-0.2, 0.9, (nrefs, nrots)).astype(np.float32)
    order = rng.permutation(nrefs) + 1
    iref, irot, found, neval, cc = O.snhc_select(corrs, order, -1.0, 6, 7, 5)
    k = int(O.snhc_uniform(7, 5, 1) * nrots)
    assert (iref, irot, found, neval) == (order[0], k + 1, 1, 1) and cc == corrs[order[0] - 1, k]
    iref, irot, found, neval, cc = O.snhc_select(corrs, order, 2.0, 6, 7, 5)
    sub = corrs[order[:6] - 1]
    best_row = int(np.argmax(sub.max(1)))
    assert (iref, irot, found, neval) == (order[best_row], int(np.argmax(sub[best_row])) + 1, 0, 7)
    pops = np.ones(nrefs, np.int32)
    pops[order[0] - 1] = 0
    iref, irot, found, neval, cc = O.snhc_select(corrs, order, -1.0, 6, 7, 5, pops)
    k = int(O.snhc_uniform(7, 5, 2) * nrots)
    assert (iref, irot, found, neval) == (order[1], k + 1, 1, 2)


def test_snhc_pick_is_uniform_over_improving_rotations(O):
    """shcloc draws uniformly among the rotations with corr >= prev_corr"""
    nrots = 20
    corrs = np.full((1, nrots), 0.1, np.float32)
    good = [2, 5, 11, 17]
    corrs[0, good] = 0.5
    counts = np.zeros(nrots, int)
    for seed in range(4000):
        iref, irot, found, neval, cc = O.snhc_select(corrs, [1], 0.3, 1, seed, 3)
        assert found == 1 and cc == np.float32(0.5)
        counts[irot - 1] += 1
    assert set(np.flatnonzero(counts)) == set(good)
    assert np.all(np.abs(counts[good] - 1000) < 120)


@pytest.mark.parametrize("geom", GEOMS)
@pytest.mark.parametrize("frame", ["ref", "ptcl"])
def test_batched_fp64_correlations_equal_direct_sums(O, geom, frame):
    """the FFT-evaluated FP64 batch (iter_allcorrs64) equals the direct FP64 sums of
    gencorrs_cc_2 / the particle frame for every (particle, reference, shift, rotation)"""
    g = O.geom(*geom)
    t = O.tables(g)
    rng = np.random.default_rng(7)
    refs = np.stack([rand_pft(rng, g.K, g.pftsz) for _ in range(3)])
    ptcls = np.stack([(0.3 * refs[i % 3] + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64) for i in range(2)])
    ctfs = np.stack([O.ctfmat(g, t, O.make_ctf(dfx=1.6 + 0.4 * i, dfy=1.5 + 0.4 * i, angast=25.0 + 40 * i))
                     for i in range(2)])
    shifts = np.array([[0.0, 0.0], [0.7, -1.2], [-2.0, 1.5]])
    got = O.allcorrs64(g, t, refs, ptcls, ctfs, shifts, frame=frame, ref_chunk=2)
    fn = O.gencorrs if frame == "ref" else O.gencorrs_ptclframe
    for p in range(2):
        for r in range(3):
            for s in range(3):
                want = fn(g, t, refs[r], ptcls[p], ctfs[p], shifts[s])
                assert np.max(np.abs(got[p, r, s] - want)) < 1e-12
    # without shifts: gencorrs_cc_1 (reference square sum over kfrom..kstop)
    g2 = O.geom(geom[0], geom[1], geom[2], geom[3], kstop=geom[2] - 3)
    t2 = O.tables(g2)
    got1 = O.allcorrs64(g2, t2, refs, ptcls, ctfs, None, frame=frame)
    fn(g2, t2, refs[1], ptcls[0], ctfs[0], None)
    assert np.max(np.abs(got1[0, 1, 0] - fn(g2, t2, refs[1], ptcls[0], ctfs[0], None))) < 1e-12


def test_batched_fft_loop_equals_single_calls(O):
    """fftpath_allcorrs (OpenMP over pairs) gives each pair's FFT-loop result (the particle
    square sum is accumulated in a different order, hence the FP32 tolerance)"""
    g = O.geom(128, 2, 20, 64)
    t = O.tables(g)
    rng = np.random.default_rng(8)
    refs = np.stack([rand_pft(rng, g.K, g.pftsz) for _ in range(3)])
    ptcl = (0.5 * refs[0] + rand_pft(rng, g.K, g.pftsz)).astype(np.complex64)
    ctf = O.ctfmat(g, t, O.make_ctf(dfx=2.1, dfy=1.9, angast=10.0))
    shifts = np.array([[0.0, 0.0], [0.5, -1.0]], np.float32)
    got, used = O.fftpath_allcorrs(g, refs, ptcl, ctf, shifts, nthreads=2)
    assert used >= 1
    fp = O.FFTPath(g)
    for r in range(3):
        for s in range(2):
            want = fp.gencorrs(refs[r], ptcl, ctf, shifts[s])
            assert np.max(np.abs(got[r, s] - want)) < 1e-6 * np.abs(want).max()
