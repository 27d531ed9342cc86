"""GPU parity of particle ingestion (pftcc_prep_ptcls: prepimg4align fused with polarize,
simple_strategy2D3D_common.f90:316-366 / :353-376) against the oracle: the oracle's
prepimg4align of each image gridded by the oracle's polarize, compared with the polar FTs and
square sums the library holds afterwards; shifts, the three CTF flags, clipping to boxmatch,
a batch larger than one cuFFT batch is not needed here (the chunking is the polarize path's);
and the argument checks.  Tolerance: three FP32 transforms (cuFFT) on noise-normalised
images, 2e-5 of the largest polar component."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def particles(n, B, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:B, 0:B]
    out = []
    for i in range(n):
        cx, cy = B / 2 + rng.uniform(-4, 4), B / 2 + rng.uniform(-4, 4)
        blob = np.exp(-((xx - cx) ** 2 + (yy - cy) ** 2) / (2 * (B / 9) ** 2))
        out.append(2.0 + 4.0 * blob + 0.8 * rng.standard_normal((B, B)))
    return np.array(out, np.float32)


@pytest.mark.parametrize("B,Bm,msk,nrots,kto", [(64, 64, 26.0, 128, 24), (100, 80, 32.0, 128, 30)])
def test_prep_ptcls_matches_oracle(pkg, O, B, Bm, msk, nrots, kto):
    n = 6
    imgs = particles(n, B, B + Bm)
    rng = np.random.default_rng(1)
    xy = rng.uniform(-3, 3, (n, 2)).astype(np.float32)
    xy[0] = 0.0                                        # below SHTHRESH: no shift
    flags = np.array([0, 1, 2, 1, 1, 0], np.int32)     # no, yes, flip (nothing to do), ...
    dfx = rng.uniform(1.0, 2.5, n)
    dfy = dfx - rng.uniform(0.0, 0.3, n)
    ang = rng.uniform(0, 180, n)
    smpd = 2.2
    ctfp = pkg.ctfparams_array(n, smpd=smpd, dfx=dfx, dfy=dfy, angast=ang)
    pc = pkg.polarft_corrcalc()
    pc.new(1, (1, n), box=Bm, nrots=nrots, kfromto=(2, kto), ctf=False)
    try:
        pc.prep_ptcls(0, imgs, xy, flags, ctfp, msk)
        g = O.geom(nrots, 2, kto, Bm)
        t = O.tables(g)
        worst = 0.0
        for i in range(n):
            c = None
            if flags[i] == 1:
                c = O.make_ctf(smpd=smpd, dfx=float(np.float32(dfx[i])), dfy=float(np.float32(dfy[i])),
                               angast=float(np.float32(ang[i])))
            cm = O.prepimg4align(imgs[i], Bm, msk, float(xy[i, 0]), float(xy[i, 1]), c)
            want = O.polarize(g, t, cm)
            got = pc.get_ptcl_pft(i + 1)
            worst = max(worst, float(np.max(np.abs(got - want)) / np.max(np.abs(want))))
            sq = np.sum(np.abs(want[: g.Ks]) ** 2)
            assert abs(pc.get_sqsum_ptcl(i + 1) - sq) < 1e-4 * sq
        print(f"prep_ptcls B {B} -> {Bm}: max error {worst:.2e} of the largest component")
        assert worst < 2e-5
    finally:
        pc.kill()


@pytest.mark.parametrize("inner,width,focusmsk,griddev", [
    (10.0, 0.0, 0.0, False), (12.0, 4.0, 0.0, True), (0.0, 0.0, 18.0, False), (0.0, 0.0, 0.0, True)])
def test_prep_ptcls_mask_modes_match_oracle(pkg, O, inner, width, focusmsk, griddev):
    """the inner mask, the focus mask and griddev 'yes' (pftcc_prep_ptcls_opts) against the oracle:
    prepimg4align in the same mode, gridded with normalised or (griddev) raw weights"""
    n, B, Bm, msk, nrots, kto = 4, 80, 64, 26.0, 128, 24
    imgs = particles(n, B, 77)
    rng = np.random.default_rng(2)
    xy = rng.uniform(-2, 2, (n, 2)).astype(np.float32)
    flags = np.array([1, 0, 1, 2], np.int32)
    dfx = rng.uniform(1.0, 2.5, n)
    dfy = dfx - rng.uniform(0.0, 0.3, n)
    ang = rng.uniform(0, 180, n)
    ctfp = pkg.ctfparams_array(n, smpd=2.0, dfx=dfx, dfy=dfy, angast=ang)
    pc = pkg.polarft_corrcalc()
    pc.new(1, (1, n), box=Bm, nrots=nrots, kfromto=(2, kto), ctf=False)
    try:
        pc.prep_ptcls(0, imgs, xy, flags, ctfp, msk, inner=inner, width=width, focusmsk=focusmsk, griddev=griddev)
        g = O.geom(nrots, 2, kto, Bm)
        t = O.tables(g)
        worst = 0.0
        for i in range(n):
            c = None
            if flags[i] == 1:
                c = O.make_ctf(smpd=2.0, dfx=float(np.float32(dfx[i])), dfy=float(np.float32(dfy[i])),
                               angast=float(np.float32(ang[i])))
            cm = O.prepimg4align_opts(imgs[i], Bm, msk, inner, width, focusmsk, griddev, float(xy[i, 0]),
                                      float(xy[i, 1]), c)
            want = O.polarize(g, t, cm, griddev=griddev)
            got = pc.get_ptcl_pft(i + 1)
            worst = max(worst, float(np.max(np.abs(got - want)) / np.max(np.abs(want))))
        print(f"prep_ptcls inner {inner} width {width} focusmsk {focusmsk} griddev {griddev}: max error {worst:.2e}")
        assert worst < 2e-5
    finally:
        pc.kill()


def test_prep_ptcls_errors(pkg):
    pc = pkg.polarft_corrcalc()
    pc.new(1, (1, 2), box=64, nrots=128, kfromto=(2, 24), ctf=False)
    imgs = particles(2, 64, 0)
    try:
        for kw, st in ((dict(msk=40.0), pkg._lib.ERR_ARG),
                       (dict(ctfflag=[1, 0], msk=20.0), pkg._lib.ERR_ARG),      # YES without parameters
                       (dict(ctfflag=[3, 0], msk=20.0), pkg._lib.ERR_ARG)):
            with pytest.raises(pkg.PftccError) as e:
                pc.prep_ptcls(0, imgs, **kw)
            assert e.value.status == st
        with pytest.raises(pkg.PftccError) as e:
            pc.prep_ptcls(0, particles(2, 48, 1), msk=20.0)                    # box_in < boxmatch
        assert e.value.status == pkg._lib.ERR_ARG
        with pytest.raises(pkg.PftccError) as e:
            pc.prep_ptcls(1, imgs, msk=20.0)                                    # slots 1..2 of 2
        assert e.value.status == pkg._lib.ERR_INDEX
    finally:
        pc.kill()
