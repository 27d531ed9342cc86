"""CPU tests of the C ABI: the library builds, loads and exports every symbol the
public header declares; without a GPU, construction fails loudly (no fallback)."""
import ctypes as C
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "pftcc_b200.h")


def declared_symbols():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(pftcc_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_reference_surface():
    names = declared_symbols()
    for must in ("pftcc_new", "pftcc_set_ref_pft", "pftcc_set_ptcl_pft", "pftcc_gencorrs", "pftcc_gencorr_for_rot",
                 "pftcc_gencorr_for_rot_8", "pftcc_gencorr_grad_for_rot_8", "pftcc_kill", "pftcc_search_best",
                 "pftcc_grad_batch", "pftcc_create_polar_absctfmats", "pftcc_polarize_ptcls"):
        assert must in names


def test_library_exports_every_declared_symbol(pkg):
    L = pkg.load_library()
    missing = [s for s in declared_symbols() if not hasattr(L, s)]
    assert not missing, missing
    # and the ctypes binding covers the same set
    from simple3_0_b200 import _lib
    assert sorted(_lib.SIGNATURES) == declared_symbols()


def test_library_is_sm100a(pkg):
    """the shared library carries an sm_100a cubin (checked through the build flags)"""
    assert "arch=compute_100a,code=sm_100a" in " ".join(pkg.build.ARCH)
    assert os.path.exists(pkg.build.LIB)


def test_strerror(pkg):
    L = pkg.load_library()
    assert L.pftcc_strerror(0) == b"ok"
    assert L.pftcc_strerror(7).startswith(b"no usable")


def test_new_without_gpu_fails_loudly(pkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    pc = pkg.polarft_corrcalc()
    with pytest.raises(pkg.PftccError) as e:
        pc.new(4, (1, 4), box=64, nrots=128, kfromto=(2, 20))
    assert e.value.status == 7


def test_new_rejects_bad_geometry(pkg):
    """argument checks of new :227-243 happen before any device call"""
    pc = pkg.polarft_corrcalc()
    bad = [dict(box=63, nrots=128, kfromto=(2, 20)), dict(box=64, nrots=127, kfromto=(2, 20)),
           dict(box=64, nrots=128, kfromto=(20, 2)), dict(box=64, nrots=128, kfromto=(2, 40))]
    for kw in bad:
        with pytest.raises(pkg.PftccError) as e:
            pc.new(4, (1, 4), **kw)
        assert e.value.status == 1
    with pytest.raises(pkg.PftccError):
        pc.new(0, (1, 4), box=64, nrots=128, kfromto=(2, 20))
    with pytest.raises(pkg.PftccError):
        pc.new(4, (5, 4), box=64, nrots=128, kfromto=(2, 20))


def test_oracle_builds_with_its_makefile(O):
    r = subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
