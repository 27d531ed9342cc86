"""GPU test of the tensor-core kernel's bounded waits, without a GPU fault: with the
pipeline-wait limit set to one poll (pftcc_set_wait_limit) the tcgen05 stage 1 gives up on
its first barrier wait, records the error word, drains the copies and MMAs it issued, frees
its tensor memory and returns; the call reports PFTCC_ERR_TIMEOUT.  With the default limit
restored the same handle searches again and agrees with the exact search (which a leaked
tensor-memory allocation or a stuck barrier would prevent).  The grouped search into device
memory reads nothing back: an expired wait in one of its calls stays in the error word, through
later good calls, until pftcc_search_check reports it and clears it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _handle(pkg):
    w = pkg.synth.config0(nrefs=8, nptcls=300)
    refs, R = pkg.synth.make_refs(w)
    parts = pkg.synth.make_particles(w, R)
    pc = pkg.polarft_corrcalc()
    pc.new(w.nrefs, (1, w.nptcls), box=w.box, nrots=w.nrots, kfromto=(w.kfrom, w.kto), ctf=True, ctf_frame="ptcl")
    pc.set_refs(1, refs.numpy(), True)
    pc.set_refs(1, refs.numpy(), False)
    pc.polarize_ptcls(0, parts.cmat.numpy())
    pc.create_polar_absctfmats(pkg.ctfparams_array(w.nptcls, smpd=w.smpd, kv=w.kv, cs=w.cs, fraca=w.fraca,
                                                   dfx=parts.dfx, dfy=parts.dfy, angast=parts.angast))
    return w, pc


def test_stage1_wait_runs_out_then_recovers(pkg):
    w, pc = _handle(pkg)
    shifts = np.array([[0.0, 0.0], [0.5, -0.5]], np.float32)
    ex = pc.search_best(shifts, "exact")
    pc.set_wait_limit(1)
    with pytest.raises(pkg.PftccError) as e:
        pc.search_best(shifts, "bf16x3", ntop=8)
    assert e.value.status == 6          # PFTCC_ERR_TIMEOUT
    pc.set_wait_limit(0)
    for _ in range(2):
        bf = pc.search_best(shifts, "bf16x3", ntop=8)
        assert np.max(np.abs(bf["corr"] - ex["corr"])) < 1e-5
    pc.kill()


def test_device_search_timeout_held_until_checked(pkg):
    import torch
    w, pc = _handle(pkg)
    shifts = np.array([[0.0, 0.0], [0.5, -0.5]], np.float32)
    groups = [(1, w.nrefs, 1, w.nptcls)]
    host = pc.search_groups(groups, shifts, "bf16x3", 8)
    out = torch.zeros((w.nptcls, 4), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    pc.set_wait_limit(1)
    pc.search_groups_dev(groups, shifts, "bf16x3", 8, out.data_ptr())    # its stage 1 gives up
    pc.set_wait_limit(0)
    pc.search_groups_dev(groups, shifts, "bf16x3", 8, out.data_ptr())    # a good call after it
    with pytest.raises(pkg.PftccError) as e:
        pc.search_check()
    assert e.value.status == 6          # PFTCC_ERR_TIMEOUT, kept through the good call
    pc.search_check()                   # reported once: the check cleared it
    assert np.array_equal(out.cpu().numpy().view(np.int32).reshape(-1, 4), host.view(np.int32).reshape(-1, 4))
    pc.search_groups_dev(groups, shifts, "bf16x3", 8, out.data_ptr())
    pc.search_check()
    pc.kill()
