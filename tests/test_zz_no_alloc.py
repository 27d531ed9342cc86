"""GPU test of pftcc_gencorrs_noalloc, the gencorrs batch that allocates no device
memory (for callers that hand all device memory to their own pool at start-up, or
that must keep a fixed device footprint, and so cannot let a library call
cudaMalloc).  Called through the C ABI, its output must equal the allocating
pftcc_gencorrs within the exact path's tolerance on two calls in a row (the second
call reuses the shared fixed scratch), and the device's free memory must not change
across a call.  The file is named to be collected last."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_gencorrs_noalloc_matches_gencorrs(pkg):
    import torch
    w = pkg.synth.config0(nrefs=4, nptcls=6)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True)
    pc.set_refs(1, refs.numpy(), True)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    rng = np.random.default_rng(4)
    n = 24
    iref = rng.integers(1, w.nrefs + 1, n).astype(np.int32)
    iptcl = rng.integers(1, w.nptcls + 1, n).astype(np.int32)
    shifts = rng.uniform(-2, 2, (n, 2)).astype(np.float32)
    want = np.stack([pc.gencorrs(int(iref[i]), int(iptcl[i]), shifts[i]) for i in range(n)])
    want1 = np.stack([pc.gencorrs(int(iref[i]), int(iptcl[i])) for i in range(n)])
    outs = [torch.full((n, w.nrots), float("nan"), dtype=torch.float32, device="cuda:0") for _ in range(2)]
    for call in range(2):
        out = outs[call]
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(0)[0]
        pc.gencorrs_noalloc(iref, iptcl, shifts, out.data_ptr())
        torch.cuda.synchronize()
        if call == 1:   # the first call may load the library's device code; later calls allocate nothing
            assert torch.cuda.mem_get_info(0)[0] == free0
        got = out.cpu().numpy()
        assert np.max(np.abs(got - want)) < 1e-6, call
        out1 = torch.full((n, w.nrots), float("nan"), dtype=torch.float32, device="cuda:0")
        pc.gencorrs_noalloc(iref, iptcl, None, out1.data_ptr())
        torch.cuda.synchronize()
        assert np.max(np.abs(out1.cpu().numpy() - want1)) < 1e-6, call
    with pytest.raises(pkg.PftccError) as e:
        pc.gencorrs_noalloc(np.ones(7000, np.int32), np.ones(7000, np.int32), None, out.data_ptr())
    assert e.value.status == 1
    pc.kill()
