"""GPU parity of the polar projector (pftcc_set_volume_ft + pftcc_fproject_polar:
expand_cmat, fproject_polar and interp_fcomp of simple_projector.f90) against the
oracle's restatement: random volume FTs at random orientations, both interpolation
normalisations, a shell mask, the even and the odd reference sets; the projected
references then serve a search like references set directly; and the argument
checks (no volume yet, non-finite angles, out-of-range references)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _vol(box, seed):
    rng = np.random.default_rng(seed)
    shape = (box, box, box // 2 + 1)
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(np.complex64)


def _euls(n, seed):
    rng = np.random.default_rng(seed)
    return np.stack([rng.uniform(0, 360, n), rng.uniform(0, 180, n), rng.uniform(0, 360, n)], 1).astype(np.float32)


@pytest.mark.parametrize("box,nrots,kto", [(32, 64, 14), (64, 128, 30)])
def test_fproject_polar_matches_oracle(pkg, O, box, nrots, kto):
    g = O.geom(nrots, 2, kto, box)
    t = O.tables(g)
    vol = _vol(box, 7)
    ex = O.expand_cmat3d(vol, box)
    n = 6
    euls = _euls(n, 11)
    mask = np.ones(g.K, bool)
    mask[4:7] = False
    pc = pkg.polarft_corrcalc()
    pc.new(n, (1, 1), box=box, nrots=nrots, kfromto=(2, kto), ctf=False)
    try:
        pc.set_volume_ft(vol)
        worst = 0.0
        for griddev in (False, True):
            for iseven in (True, False):
                m = None if iseven else mask
                pc.fproject_polar(1, euls, iseven=iseven, mask=m, griddev=griddev)
                for r in range(n):
                    got = pc.get_ref_pft(r + 1, iseven)
                    want = O.fproject_polar(g, t, ex, box, euls[r].astype(np.float64),
                                            mask=None if m is None else m.astype(np.int32), griddev=griddev)
                    worst = max(worst, float(np.max(np.abs(got - want)) / np.max(np.abs(want))))
                    if m is not None:
                        assert np.all(got[~m] == 0)
        print(f"fproject_polar box {box}: max relative error vs the oracle {worst:.2e}")
        assert worst < 1e-5
    finally:
        pc.kill()


def test_search_over_projected_references(pkg):
    """references from the projector serve the search exactly like the same arrays set
    directly (the projection writes the reference sets in place)"""
    w = pkg.synth.config0(nrefs=6, nptcls=20)
    box, nrots, kto = w.box, w.nrots, w.kto
    vol = _vol(box, 5)
    euls = _euls(w.nrefs, 9)
    parts = pkg.synth.make_particles(w, pkg.synth.random_rotations(w.nrefs, np.random.default_rng(1)))
    shifts = np.array([[0.0, 0.0], [1.0, -0.5]], np.float32)
    res = []
    for mode in ("project", "set"):
        pc = pkg.polarft_corrcalc()
        pc.new(w.nrefs, (1, w.nptcls), box=box, nrots=nrots, kfromto=(w.kfrom, kto), ctf=False)
        try:
            if mode == "project":
                pc.set_volume_ft(vol)
                pc.fproject_polar(1, euls, iseven=True)
                pc.fproject_polar(1, euls, iseven=False)
                refs = np.stack([pc.get_ref_pft(r + 1, True) for r in range(w.nrefs)])
            else:
                pc.set_refs(1, refs, True)
                pc.set_refs(1, refs, False)
            pc.polarize_ptcls(0, parts.cmat.numpy())
            res.append(pc.search_best(shifts, "exact"))
        finally:
            pc.kill()
    assert np.array_equal(res[0]["iref"], res[1]["iref"]) and np.array_equal(res[0]["irot"], res[1]["irot"])
    assert np.array_equal(res[0]["corr"], res[1]["corr"])


def test_fproject_polar_argument_checks(pkg):
    pc = pkg.polarft_corrcalc()
    pc.new(2, (1, 1), box=32, nrots=64, kfromto=(2, 14), ctf=False)
    try:
        with pytest.raises(Exception):
            pc.fproject_polar(1, _euls(2, 3))                    # no volume yet
        pc.set_volume_ft(_vol(32, 1))
        with pytest.raises(Exception):
            pc.fproject_polar(2, _euls(2, 3))                    # references 2..3 of 2
        bad = _euls(1, 3)
        bad[0, 1] = np.nan
        with pytest.raises(Exception):
            pc.fproject_polar(1, bad)                            # non-finite angle
        pc.fproject_polar(1, _euls(2, 3))                        # still usable
    finally:
        pc.kill()
