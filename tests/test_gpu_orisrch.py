"""GPU parity of the orientation-gradient path against the oracle: pftcc_fdf_project_polar
(fdf_project_polar / fdf_interp_fcomp, simple_projector.f90:245-267, :338-400) writes the
sections and their Euler-angle derivatives; pftcc_gencorr_cont_shift_grad_cc_for_rot_8 /
pftcc_gencorr_cont_grad_cc_for_rot_8 / pftcc_cont_shift_grad_batch
(simple_polarft_corrcalc.f90:1735-1847) correlate them with particles; argument and state
checks.  Tolerances: the sections and derivatives are FP64 sums rounded to FP32
(1e-5 of each array's largest value); the correlator runs in FP64 on FP32 operands with the
library's FP32 |CTF| against the oracle's FP64 one (1e-6)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _vol(box, seed):
    rng = np.random.default_rng(seed)
    shape = (box, box, box // 2 + 1)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def _euls(n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(0, 360, n), rng.uniform(0, 180, n), rng.uniform(0, 360, n)], 1)


@pytest.mark.parametrize("box,nrots,kto", [(32, 64, 14), (64, 128, 30)])
def test_fdf_project_polar_matches_oracle(pkg, O, box, nrots, kto):
    g = O.geom(nrots, 2, kto, box)
    t = O.tables(g)
    vol = _vol(box, 3)
    ex = O.expand_cmat3d(vol, box)
    n = 4
    euls = _euls(n, 5)
    pc = pkg.polarft_corrcalc()
    pc.new(2 * n, (1, 1), box=box, nrots=nrots, kfromto=(2, kto), ctf=False)
    try:
        pc.set_volume_ft(vol)
        pc.fdf_project_polar(1, euls, iseven=False)
        pc.fproject_polar(n + 1, euls.astype(np.float32), iseven=False)
        for r in range(n):
            want, dwant = O.fdf_project_polar(g, t, ex, box, euls[r])
            got = pc.get_ref_pft(r + 1, False)
            dgot = pc.get_dref_pft(r + 1, False)
            assert np.max(np.abs(got - want)) < 1e-5 * np.max(np.abs(want))
            for j in range(3):
                assert np.max(np.abs(dgot[j] - dwant[j])) < 1e-5 * np.max(np.abs(dwant[j]))
            # the sections are interp_fcomp_norm's, as fproject_polar writes them (its angles in FP32)
            proj = pc.get_ref_pft(n + r + 1, False)
            assert np.max(np.abs(proj - got)) < 1e-4 * np.max(np.abs(got))
    finally:
        pc.kill()


def test_cont_shift_grad_matches_oracle(pkg, O):
    w = pkg.synth.config0(nrefs=3, nptcls=4)
    box, nrots = w.box, w.nrots
    g = O.geom(nrots, w.kfrom, w.kto, box, kstop=w.kto - 4)
    t = O.tables(g)
    vol = _vol(box, 9)
    euls = _euls(3, 13)
    pc = pkg.polarft_corrcalc()
    pc.new(3, (1, 4), box=box, nrots=nrots, kfromto=(w.kfrom, w.kto), kstop=w.kto - 4, ctf=True, ctf_frame="ref",
           eoarr=[0, 1, 0, 1])
    try:
        pc.set_volume_ft(vol)
        pc.fdf_project_polar(1, euls, iseven=True)
        pc.fdf_project_polar(1, euls[::-1].copy(), iseven=False)
        rng = np.random.default_rng(1)
        for i in range(4):
            base = pc.get_ref_pft(1 + i % 3, i % 2 == 0)
            noise = rng.standard_normal(base.shape) + 1j * rng.standard_normal(base.shape)
            pc.set_ptcl_pft(i + 1, (0.7 * base + 0.2 * np.abs(base).mean() * noise).astype(np.complex64))
        dfx = np.array([1.5, 2.0, 2.5, 1.8])
        pc.create_polar_absctfmats(pkg.ctfparams_array(4, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca, dfx=dfx,
                                                       dfy=dfx - 0.1, angast=[10.0, 50.0, 90.0, 130.0]))
        reqs = [(1, 1, 1, 0.0, 0.0), (2, 2, 17, 0.5, -0.3), (3, 3, 100, -1.0, 0.75), (1, 4, 128, 0.2, 0.2)]
        fb, gb = pc.cont_shift_grad_batch(*[np.array(v) for v in zip(*reqs)])
        for n, (ir, ip, irot, sx, sy) in enumerate(reqs):
            ev = ip % 2 == 1
            ref = pc.get_ref_pft(ir, ev)
            dref = pc.get_dref_pft(ir, ev)
            ptcl = pc.get_ptcl_pft(ip)
            c = O.ctfmat(g, t, O.make_ctf(w.smpd, w.kv, w.cs, w.fraca, float(dfx[ip - 1]), float(dfx[ip - 1] - 0.1),
                                          [10.0, 50.0, 90.0, 130.0][ip - 1]))
            fo, go = O.gencorr_cont_shift_grad(g, t, ref, dref, ptcl, irot, c, (sx, sy))
            f, gr = pc.gencorr_cont_shift_grad_cc_for_rot_8(ir, ip, [sx, sy], irot)
            assert abs(f - fo) < 1e-6
            assert np.max(np.abs(gr - go)) < 1e-6 * max(1.0, np.max(np.abs(go)))
            assert f == fb[n] and np.array_equal(gr, gb[n])
            cc, dcc = pc.gencorr_cont_grad_cc_for_rot_8(ir, ip, [sx, sy], irot)
            assert cc == f and np.array_equal(dcc, gr[:3])
            # the value is gencorr_cc_for_rot_8's unweighted (match_filt) branch
            assert abs(f - O.gencorr_for_rot(g, t, ref, ptcl, irot, c, [sx, sy], match_filt=True)) < 1e-6
    finally:
        pc.kill()


def test_orisrch_state_errors(pkg):
    pc = pkg.polarft_corrcalc()
    pc.new(2, (1, 2), box=32, nrots=64, kfromto=(2, 14), ctf=False, ctf_frame="ref")
    try:
        with pytest.raises(pkg.PftccError) as e:
            pc.fdf_project_polar(1, [[10.0, 20.0, 30.0]])
        assert e.value.status == pkg._lib.ERR_STATE
        with pytest.raises(pkg.PftccError) as e:
            pc.gencorr_cont_shift_grad_cc_for_rot_8(1, 1, [0.0, 0.0], 1)
        assert e.value.status == pkg._lib.ERR_STATE
        pc.set_volume_ft(_vol(32, 1))
        with pytest.raises(pkg.PftccError) as e:
            pc.fdf_project_polar(1, [[10.0, np.nan, 30.0]])
        assert e.value.status == pkg._lib.ERR_ARG
        with pytest.raises(pkg.PftccError) as e:
            pc.fdf_project_polar(2, [[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]])
        assert e.value.status == pkg._lib.ERR_INDEX
        pc.fdf_project_polar(1, [[10.0, 20.0, 30.0], [40.0, 50.0, 60.0]])
        with pytest.raises(pkg.PftccError) as e:
            pc.gencorr_cont_shift_grad_cc_for_rot_8(1, 1, [0.0, 0.0], 65)
        assert e.value.status == pkg._lib.ERR_INDEX
    finally:
        pc.kill()


def _smooth_vol(box, seed, sigma=5.0):
    """a random volume FT under a Gaussian low-pass: broad correlation peaks in angle"""
    v = _vol(box, seed)
    f = np.fft.fftfreq(box) * box
    h = np.arange(box // 2 + 1)
    r2 = f[:, None, None] ** 2 + f[None, :, None] ** 2 + h[None, None, :] ** 2
    return (v * np.exp(-r2 / (2 * sigma ** 2))).astype(np.complex64)


def test_orisrch_batch_recovers_orientation(pkg):
    """particles made as sections of the volume at known angles (zero shifts), searched from
    perturbed starts: the search improves the correlation, moves the angles towards the truth,
    and its reported correlation is the correlator's value at the reported point"""
    box, nrots, kto, n = 64, 128, 14, 5
    vol = _smooth_vol(box, 21)
    rng = np.random.default_rng(4)
    truth = np.stack([rng.uniform(20, 340, n), rng.uniform(30, 150, n), rng.uniform(20, 340, n)], 1)
    pc = pkg.polarft_corrcalc()
    pc.new(n + 1, (1, n), box=box, nrots=nrots, kfromto=(2, kto), ctf=False, ctf_frame="ref")
    try:
        pc.set_volume_ft(vol)
        pc.fproject_polar(1, truth.astype(np.float32), iseven=True)
        for i in range(n):
            pc.set_ptcl_pft(i + 1, pc.get_ref_pft(i + 1, True))
        start = truth + rng.uniform(-2.0, 2.0, (n, 3))
        res = pc.orisrch_batch(np.arange(1, n + 1), start, angerr_deg=6.0, maxhwshift=2.0, maxits=60)
        for i, r in enumerate(res):
            assert r["found_better"] and r["corr"] > r["corr_init"]
            assert np.max(np.abs(r["e"] - truth[i])) < np.max(np.abs(start[i] - truth[i]))
            assert r["corr"] > 0.99
            # the reported value is the correlator's at the reported point: undo rotmat2d(e3)
            a = np.radians(r["e"][2])
            M = np.array([[np.cos(a), np.sin(a)], [-np.sin(a), np.cos(a)]])
            x45 = r["shift"] @ M.T
            pc.fdf_project_polar(n + 1, r["e"][None], iseven=True)
            f, _ = pc.gencorr_cont_shift_grad_cc_for_rot_8(n + 1, i + 1, x45, 1)
            assert abs(f - r["corr"]) < 1e-9
        # a search started at the truth cannot improve beyond rounding
        res0 = pc.orisrch_batch([1], truth[:1], angerr_deg=6.0, maxhwshift=2.0)
        assert res0[0]["corr"] - res0[0]["corr_init"] < 1e-6
    finally:
        pc.kill()
