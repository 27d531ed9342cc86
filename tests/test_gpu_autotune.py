"""GPU test of the search's wave / tile tuning and its autotuner (pftcc_set_tuning,
pftcc_autotune): the sizes only change how the work is cut, so every tuning gives
bit-identical search results; the autotuner keeps a timed candidate, writes a wisdom line and
reads it back on the next call without timing."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def build(pkg, w):
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame="ptcl")
    pc.set_refs(1, refs.numpy(), True)
    pc.set_refs(1, refs.numpy(), False)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    return pc


@pytest.mark.parametrize("cfgname", ["config0", "config1"])
def test_tunings_give_identical_results(pkg, cfgname):
    w = getattr(pkg.synth, cfgname)(nrefs=40, nptcls=700)
    pc = build(pkg, w)
    shifts = np.array(pkg.synth.shift_grid(1.0, 0.5), np.float32)
    ref = pc.search_best(shifts, "bf16x3", ntop=8)
    ref32 = pc.search_best(shifts, "fp32", ntop=8)
    for t in ((64, 128, 2), (128, 256, 3), (192, 512, 4), (4096, 4096, 0)):
        pc.set_tuning(*t)
        got = pc.search_best(shifts, "bf16x3", ntop=8)
        assert np.array_equal(got.view(np.int32), ref.view(np.int32)), t
        got32 = pc.search_best(shifts, "fp32", ntop=8)
        assert np.array_equal(got32.view(np.int32), ref32.view(np.int32)), t
    pc.kill()


def test_autotune_and_wisdom(pkg, tmp_path):
    w = pkg.synth.config0(nrefs=30, nptcls=600)
    pc = build(pkg, w)
    shifts = np.array(pkg.synth.shift_grid(1.0, 0.5), np.float32)
    ref = pc.search_best(shifts, "bf16x3", ntop=8)
    wis = str(tmp_path / "wisdom.txt")
    t = pc.autotune(shifts, "bf16x3", 8, wisdom=wis)
    assert not t["from_wisdom"]
    lines = open(wis).read().splitlines()
    assert len(lines) == 1 and "nrots=128" in lines[0] and " -> w_rows=" in lines[0]
    assert np.array_equal(pc.search_best(shifts, "bf16x3", ntop=8).view(np.int32), ref.view(np.int32))
    pc.set_tuning(0, 0, 0)
    t2 = pc.autotune(shifts, "bf16x3", 8, wisdom=wis)
    assert t2["from_wisdom"] and {k: t2[k] for k in ("w_rows", "w_cols", "s1_stages")} == \
        {k: t[k] for k in ("w_rows", "w_cols", "s1_stages")}
    assert len(open(wis).read().splitlines()) == 1
    # another shape is another line
    pc.autotune(None, "bf16x3", 4, wisdom=wis)
    assert len(open(wis).read().splitlines()) == 2
    pc.kill()
