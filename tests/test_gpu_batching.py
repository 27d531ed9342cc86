"""GPU tests of the chunk queue (simple3.0_b200/batching.py): chunks of the three batching
geometries, of uneven sizes, run through two worker streams, or as grouped searches (one handle
and one pftcc_search_groups call per geometry), must give per chunk exactly the result of
searching that chunk alone (BF16-split search with the FP32 re-score of the top 8)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_queue_results_equal_each_chunk_alone(pkg):
    b = pkg.batching
    spec = [("A", 14, 70), ("B", 9, 33), ("C", 5, 21), ("A", 23, 48), ("B", 6, 57), ("C", 7, 12)]
    chunks = [b.synthetic_chunk(g, nr, npt, seed=i) for i, (g, nr, npt) in enumerate(spec)]
    got = b.SearchQueue(workers=2).run(chunks)
    for ch, res in zip(chunks, got):
        alone = b.search_chunk(ch)
        assert res.shape == (ch.nptcls,)
        for f in ("iref", "irot", "ishift"):
            assert np.array_equal(res[f], alone[f])
        assert np.array_equal(res["corr"].view(np.int32), alone["corr"].view(np.int32))
        assert np.all(res["iref"] >= 1) and np.all(res["iref"] <= ch.nrefs)


def _same(res, alone):
    for f in ("iref", "irot", "ishift"):
        assert np.array_equal(res[f], alone[f]), f
    assert np.array_equal(res["corr"].view(np.int32), alone["corr"].view(np.int32))


@pytest.mark.parametrize("precision", ["bf16x3", "fp32"])
def test_grouped_search_equals_each_chunk_alone(pkg, precision):
    """pftcc_search_groups over a queue of uneven chunks of the three batching geometries (one
    handle per geometry, one persistent stage-1 launch and one stage-2 launch over all of a
    geometry's chunks): every chunk's result is bit for bit its result searched alone."""
    b = pkg.batching
    spec = [("A", 14, 70), ("B", 9, 33), ("C", 5, 21), ("A", 23, 148), ("B", 6, 257), ("C", 7, 12), ("A", 3, 40)]
    chunks = [b.synthetic_chunk(g, nr, npt, seed=i) for i, (g, nr, npt) in enumerate(spec)]
    got = b.search_grouped(chunks, precision=precision)
    for ch, res in zip(chunks, got):
        alone = b.search_chunk(ch, precision=precision)
        assert res.shape == (ch.nptcls,)
        _same(res, alone)
        assert np.all(res["iref"] >= 1) and np.all(res["iref"] <= ch.nrefs)


def test_grouped_search_with_shifts_and_unsearched_slots(pkg):
    """with a shift grid (rows = references x shifts, group rows not tile aligned) the grouped
    search equals each chunk alone; slots outside every group come back unsearched"""
    b = pkg.batching
    sh = np.array([[0.0, 0.0], [0.5, -0.5], [-1.0, 0.5]], np.float32)
    chunks = []
    for i, (nr, npt) in enumerate([(11, 150), (7, 61), (13, 130)]):
        ch = b.synthetic_chunk("B", nr, npt, seed=40 + i)
        ch.shifts = sh
        chunks.append(ch)
    got = b.search_grouped(chunks)
    for ch, res in zip(chunks, got):
        _same(res, b.search_chunk(ch))
    # one handle, two of three chunks grouped: the third chunk's slots are left out
    ch = chunks
    pc = pkg.polarft_corrcalc()
    nrefs, nptcls = sum(c.nrefs for c in ch), sum(c.nptcls for c in ch)
    pc.new(nrefs, (1, nptcls), box=ch[0].box, nrots=ch[0].nrots, kfromto=(ch[0].kfrom, ch[0].kto), ctf=True,
           ctf_frame="ptcl")
    refs = np.concatenate([c.refs for c in ch])
    pc.set_refs(1, refs, True)
    pc.set_refs(1, refs, False)
    s = 0
    for c in ch:
        pc.polarize_ptcls_dev(s, c.nptcls, c.cmats.contiguous().data_ptr())
        s += c.nptcls
    pc.create_polar_absctfmats(pkg.ctfparams_array(nptcls, smpd=ch[0].smpd, kv=ch[0].kv, cs=ch[0].cs, fraca=ch[0].fraca,
                                                   dfx=np.concatenate([c.dfx for c in ch]),
                                                   dfy=np.concatenate([c.dfy for c in ch]),
                                                   angast=np.concatenate([c.angast for c in ch])))
    g0 = (1, ch[0].nrefs, 1, ch[0].nptcls)
    g2 = (ch[0].nrefs + ch[1].nrefs + 1, ch[2].nrefs, ch[0].nptcls + ch[1].nptcls + 1, ch[2].nptcls)
    out = pc.search_groups([g0, g2], sh, "bf16x3", 8)
    mid = out[ch[0].nptcls:ch[0].nptcls + ch[1].nptcls]
    assert np.all(mid["iref"] == 0) and np.all(np.isneginf(mid["corr"]))
    a0 = out[:ch[0].nptcls]
    assert np.all((a0["iref"] >= 1) & (a0["iref"] <= ch[0].nrefs))
    a2 = out[ch[0].nptcls + ch[1].nptcls:]
    assert np.all((a2["iref"] > ch[0].nrefs + ch[1].nrefs) & (a2["iref"] <= nrefs))
    with pytest.raises(pkg.PftccError):
        pc.search_groups([g0, (1, 2, 3, 5)], sh, "bf16x3", 8)     # groups sharing particle slots
    pc.kill()


def test_grouped_search_captured_in_a_graph(pkg):
    """pftcc_search_groups_dev: after one call outside capture, the same call captured into a CUDA
    graph on the handle's stream replays to the uncaptured call's result, bit for bit, every time
    (the outputs cleared in between); the bounded waits report no error; a first call inside a
    capture (nothing sized yet) is refused with PFTCC_ERR_STATE"""
    import torch
    b = pkg.batching
    chunks = [b.synthetic_chunk("B", nr, npt, seed=70 + i) for i, (nr, npt) in enumerate([(9, 150), (12, 70), (5, 200)])]
    side = torch.cuda.Stream()
    pc, groups = b.grouped_handle(chunks, stream=side.cuda_stream)
    try:
        n = sum(ch.nptcls for ch in chunks)
        out = torch.zeros((n, 4), dtype=torch.int32, device="cuda")
        with torch.cuda.stream(side):
            pc.search_groups_dev(groups, None, "bf16x3", 8, out.data_ptr())
        torch.cuda.synchronize()
        pc.search_check()
        want = out.clone()
        host = pc.search_groups(groups, None, "bf16x3", 8)
        assert np.array_equal(want.cpu().numpy().view(np.int32).reshape(-1), host.view(np.int32).reshape(-1))
        g = torch.cuda.CUDAGraph()
        out.zero_()
        torch.cuda.synchronize()
        with torch.cuda.graph(g, stream=side):
            pc.search_groups_dev(groups, None, "bf16x3", 8, out.data_ptr())
        for _ in range(2):
            out.zero_()
            torch.cuda.synchronize()
            g.replay()
            torch.cuda.synchronize()
            assert torch.equal(out, want)
        pc.search_check()
        del g
    finally:
        pc.kill()
    # nothing sized: refused inside the capture, with the capture then abandoned by the caller
    pc2, groups2 = b.grouped_handle(chunks[:1], stream=side.cuda_stream)
    try:
        out2 = torch.zeros((chunks[0].nptcls, 4), dtype=torch.int32, device="cuda")
        g2 = torch.cuda.CUDAGraph()
        with pytest.raises(pkg.PftccError) as e:
            with torch.cuda.graph(g2, stream=side):
                pc2.search_groups_dev(groups2, None, "bf16x3", 8, out2.data_ptr())
        assert e.value.status == 3      # PFTCC_ERR_STATE
    finally:
        torch.cuda.synchronize()
        pc2.kill()
