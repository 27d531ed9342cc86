"""GPU tests of the stochastic reference search (pftcc_search_snhc: strategy2D_snhc's
srch_snhc with shcloc) through the C ABI.  The selection must be exactly the oracle's
restatement replayed over the same correlations (the library's own corr_all in the same
precision), particle by particle: chosen reference and rotation, whether an improving
reference was found, the number of visits counted, and the correlation."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make(pkg, w, frame):
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame=frame)
    pc.set_refs(1, refs.numpy(), True)
    pc.set_refs(1, refs.numpy(), False)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    return pc


@pytest.mark.parametrize("frame,precision", [("ref", "exact"), ("ptcl", "fp32"), ("ptcl", "bf16x3")])
def test_snhc_matches_oracle_replay(pkg, O, frame, precision):
    w = pkg.synth.config0(nrefs=20, nptcls=24)
    pc = make(pkg, w, frame)
    cc = pc.corr_all() if precision == "exact" else pc.corr_all_prec(None, precision)
    cc = cc[:, :, 0, :]                                   # (nptcls, nrefs, nrots)
    rng = np.random.default_rng(17)
    order = np.stack([rng.permutation(w.nrefs) + 1 for _ in range(w.nptcls)]).astype(np.int32)
    best = cc.max(axis=(1, 2))
    # a third improve easily, a third only sometimes, a third never (greedy fallback)
    sel = np.arange(w.nptcls) % 3
    prev = np.where(sel == 0, best - 0.3, np.where(sel == 1, best - 0.002, best + 0.1)).astype(np.float32)
    pops = np.ones(w.nrefs, np.int32)
    pops[[3, 11]] = 0
    seed = 0x5EED1234ABCDEF
    for cls_pops, bound in ((None, 14), (pops, 20)):
        got = pc.search_snhc(order, prev, bound, seed, cls_pops=cls_pops, precision=precision)
        for i in range(w.nptcls):
            iref, irot, found, neval, corr = O.snhc_select(cc[i], order[i], float(prev[i]), bound, seed, i + 1,
                                                           cls_pops)
            g = got[i]
            assert (g["iref"], g["irot"], g["found_better"], g["nrefs_eval"]) == (iref, irot, found, neval), (i, bound)
            assert g["corr"] == np.float32(corr)
        assert got["found_better"][0::3].all() and not got["found_better"][2::3].any()
    pc.kill()


def test_snhc_rejects_bad_input(pkg):
    w = pkg.synth.config0(nrefs=4, nptcls=3)
    pc = make(pkg, w, "ref")
    order = np.tile(np.arange(1, 5, dtype=np.int32), (3, 1))
    bad = order.copy()
    bad[1, 2] = 5
    with pytest.raises(pkg.PftccError):
        pc.search_snhc(bad, np.zeros(3), 4, 1)
    with pytest.raises(pkg.PftccError):
        pc.search_snhc(order, np.zeros(3), 4, 1, precision="fp32")    # m-domain needs the particle frame
    pc.kill()
