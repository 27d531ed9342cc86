"""CPU tests of the oracle's particle ingestion (prepimg4align,
simple_strategy2D3D_common.f90:316-366): the C restatement against an independent numpy
restatement of the same chain (noise_norm, fft with the phase-origin swap, shift2Dserial,
the CTF phase flip, ifft, clip, zero_background + cosine-edge mask, fft and the box factor;
numpy's FFTs in place of the C oracle's own), and properties of the chain: noise
normalisation makes the image's intensity scale and offset irrelevant, and the flip's sign
convention (identity where the CTF is positive, negation where it is negative)."""
import math

import numpy as np
import pytest


def _ctf_chi(c, s2, ang):
    kv = c.kv * 1000.0
    wl = 12.26 / math.sqrt(kv + 0.9784 * kv * kv / 1.0e6) / c.smpd
    cs = c.cs * 1.0e7 / c.smpd
    ampc = math.atan(c.fraca / math.sqrt(1.0 - c.fraca * c.fraca))
    sc = 1.0e4 / c.smpd
    dfx, dfy = c.dfx * sc, c.dfy * sc
    angast = c.angast / 180.0 * math.pi
    df = 0.5 * (dfx + dfy + np.cos(2.0 * (ang - angast)) * (dfx - dfy))
    return math.pi * wl * s2 * (df - 0.5 * wl * wl * s2 * cs) + c.phshift + ampc


def instr_numpy(x):
    """kbinterpol%instr for W = 3, beta = 7.4: sinh(y) / y, y = sqrt(beta^2 - (pi W x)^2)"""
    piW = float(np.float32(np.float32(math.pi) * np.float32(3.0)))
    betasq = float(np.float32(np.float32(7.4) * np.float32(7.4)))
    yv = np.sqrt(betasq - (piW * x) ** 2)
    return np.sinh(yv) / yv


def prep_numpy(img, Bm, msk, x=0.0, y=0.0, ctf=None, inner=0.0, iwidth=0.0, focusmsk=0.0, griddev=False):
    r = np.asarray(img, np.float64).copy()
    B = r.shape[0]
    c = B // 2 + 1
    ii = np.arange(1, B + 1)
    dist = np.sqrt((ii[None, :] - c) ** 2 + (ii[:, None] - c) ** 2)
    bg = ~(dist <= msk)
    n = bg.sum()
    ave = r[bg].sum() / n
    if abs(ave) > 1e-10:
        r -= ave
    ep, var = r[bg].sum(), (r[bg] ** 2).sum()
    var = (var - ep * ep / n) / (n - 1)
    if var > 0:
        r /= math.sqrt(var)
    Z = np.fft.rfft2(np.fft.fftshift(r)) / (B * B)            # [k][h]
    h = np.arange(B // 2 + 1)[None, :].astype(np.float64)
    k = (np.fft.fftfreq(B) * B)[:, None]
    F = np.ones(Z.shape, np.complex128)
    if abs(x) > 0.001 or abs(y) > 0.001:
        shconst = np.float32(math.pi) / np.float32(B // 2)
        sh1 = float(np.float32(-x) * shconst)
        sh2 = float(np.float32(-y) * shconst)
        a = h * sh1 + k * sh2
        F = np.cos(a).astype(np.float32) + 1j * np.sin(a).astype(np.float32)
    if ctf is not None:
        s2 = (h / B) ** 2 + (k / B) ** 2
        t = np.sin(_ctf_chi(ctf, s2, np.arctan2(k + 0 * h, h)))
        F = F * np.where(t >= 0, 1.0, -1.0)
    r2 = np.fft.fftshift(np.fft.irfft2(Z * F, s=(B, B)) * (B * B))
    st = (B - Bm) // 2
    m = r2[st:st + Bm, st:st + Bm].copy()
    med = np.mean([np.sort(v)[Bm // 2 - 1] for v in (m[:, 0], m[:, Bm - 1], m[0, :], m[Bm - 1, :])])
    if abs(med) > 1e-10:
        m -= med
    mrad = msk if inner > 0 else (focusmsk if focusmsk > 0 else msk)
    iw = iwidth if iwidth > 0 else 10.0
    minlen = min(int(math.floor(2 * (mrad + 6.0) + 0.5)), Bm)
    maxrad = float(minlen // 2)
    width = 2.0 * (maxrad - mrad)
    for i in range(1, Bm // 2 + 1):
        for j in range(1, Bm // 2 + 1):
            cx, cy = -Bm / 2 + (i - 1), -Bm / 2 + (j - 1)
            rad = math.sqrt(cx * cx + cy * cy)
            e = 1.0
            if rad >= maxrad:
                e = 0.0
            elif rad >= maxrad - width:
                e = (math.cos(((rad - (maxrad - width)) / width) * math.pi) + 1.0) / 2.0
            if inner > 0:
                e *= 0.0 if rad < inner - iw else (1.0 if rad > inner else
                                                   (1.0 + math.cos(math.pi * (inner - rad) / iw)) / 2.0)
            if e > 0.9999:
                continue
            for jj in (j, Bm + 1 - j):
                for ii_ in (i, Bm + 1 - i):
                    m[jj - 1, ii_ - 1] *= e
    if griddev:
        xs = np.array([float(np.float32(np.float32(i - (Bm // 2 + 1)) / np.float32(Bm))) for i in range(1, Bm + 1)])
        w = instr_numpy(xs)
        m /= w[None, :] * w[:, None]
    return np.fft.rfft2(np.fft.fftshift(m)) / (B * B)


def particle(B, seed):
    rng = np.random.default_rng(seed)
    yy, xx = np.mgrid[0:B, 0:B]
    blob = np.exp(-((xx - B / 2 - 3.0) ** 2 + (yy - B / 2 + 2.0) ** 2) / (2 * (B / 10) ** 2))
    return (3.0 + 5.0 * blob + 0.7 * rng.standard_normal((B, B))).astype(np.float32)


@pytest.mark.parametrize("B,Bm,msk,x,y,with_ctf", [
    (64, 64, 24.0, 0.0, 0.0, False),
    (64, 64, 24.0, 1.7, -2.3, False),
    (64, 48, 18.0, -0.6, 0.9, True),
    (100, 80, 30.5, 2.0, 3.0, True),
])
def test_prepimg4align_matches_numpy(O, B, Bm, msk, x, y, with_ctf):
    img = particle(B, B + Bm)
    ctf = O.make_ctf(smpd=2.1, dfx=1.9, dfy=1.5, angast=35.0) if with_ctf else None
    got = O.prepimg4align(img, Bm, msk, x, y, ctf)
    want = prep_numpy(img, Bm, msk, x, y, ctf)
    assert got.shape == (Bm, Bm // 2 + 1)
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))


@pytest.mark.parametrize("inner,iwidth,focusmsk,griddev", [
    (10.0, 0.0, 0.0, False),      # inner mask, the default width 10
    (12.0, 4.0, 0.0, True),       # inner mask of width 4, griddev 'yes'
    (0.0, 0.0, 16.0, False),      # focus mask
    (0.0, 0.0, 0.0, True),        # griddev alone
])
def test_prepimg4align_mask_modes(O, inner, iwidth, focusmsk, griddev):
    """l_innermsk, l_focusmsk and griddev 'yes' (prepimg4align :349-362) against the numpy chain"""
    img = particle(64, 9)
    ctf = O.make_ctf(smpd=2.1, dfx=1.9, dfy=1.5, angast=35.0)
    got = O.prepimg4align_opts(img, 56, 24.0, inner, iwidth, focusmsk, griddev, 0.7, -1.2, ctf)
    want = prep_numpy(img, 56, 24.0, 0.7, -1.2, ctf, inner, iwidth, focusmsk, griddev)
    assert np.max(np.abs(got - want)) < 1e-12 * np.max(np.abs(want))
    plain = O.prepimg4align(img, 56, 24.0, 0.7, -1.2, ctf)
    assert np.max(np.abs(got - plain)) > 1e-3 * np.max(np.abs(plain))     # the mode changes the output


def test_instrument_function_values(O):
    """the instrument function is 1 at the centre only in ratio: w(x) / w(0) falls towards the
    edges (the window's transform), symmetric, and is the sinh form of I0's transform"""
    x = np.linspace(-0.5, 0.5, 11)
    w = instr_numpy(x)
    assert np.allclose(w, w[::-1])
    assert np.all(np.diff(w[:6]) > 0)
    # sinh(y)/y is the continuous transform of the Kaiser-Bessel window I0(beta sqrt(1 - (2u/W)^2))
    # over |u| <= W/2 up to a constant: check at x = 0.3 by quadrature
    from scipy.special import i0
    u = np.linspace(-1.5, 1.5, 200001)
    kb = i0(7.4 * np.sqrt(np.clip(1 - (2 * u / 3.0) ** 2, 0, None)))
    ft = lambda xx: np.trapezoid(kb * np.cos(2 * np.pi * u * xx), u)
    assert abs(ft(0.3) / ft(0.0) - instr_numpy(0.3) / instr_numpy(0.0)) < 1e-4


def test_noise_norm_makes_intensity_scale_irrelevant(O):
    """noise_norm divides out the background's mean and deviation, so a * img + b (a > 0) gives
    the same output as img"""
    img = particle(64, 5)
    a = O.prepimg4align(img, 64, 22.0, 0.8, -1.1)
    b = O.prepimg4align((2.5 * img + 7.0).astype(np.float32), 64, 22.0, 0.8, -1.1)
    assert np.max(np.abs(a - b)) < 1e-5 * np.max(np.abs(a))


def test_flip_sign_convention(O):
    """with Cs = 0 and a small defocus the CTF argument stays in (0, pi) over the whole
    transform, so the flip is the identity; a phase shift of pi (added by apply_serial whatever
    the phase-plate flag) puts it in (pi, 2 pi) and the flip negates every component"""
    img = particle(64, 6)
    ref = O.prepimg4align(img, 64, 22.0, 0.4, 0.3)
    pos = O.prepimg4align(img, 64, 22.0, 0.4, 0.3, O.make_ctf(smpd=2.0, cs=0.0, dfx=0.01, dfy=0.01))
    neg = O.prepimg4align(img, 64, 22.0, 0.4, 0.3, O.make_ctf(smpd=2.0, cs=0.0, dfx=0.01, dfy=0.01,
                                                              phshift=math.pi))
    assert np.max(np.abs(pos - ref)) < 1e-12 * np.max(np.abs(ref))
    # negation is exact up to zero_background's constant: the lower median of the negated border
    # is not the negated lower median, so neg + ref is a constant times the mask's own transform
    B, msk = 64, 22.0
    minlen = min(int(math.floor(2 * (msk + 6.0) + 0.5)), B)
    maxrad, E = float(minlen // 2), np.ones((B, B))
    width = 2.0 * (maxrad - msk)
    for i in range(1, B // 2 + 1):
        for j in range(1, B // 2 + 1):
            rad = math.hypot(-B / 2 + i - 1, -B / 2 + j - 1)
            e = 0.0 if rad >= maxrad else (1.0 if rad < maxrad - width else
                                           (math.cos((rad - (maxrad - width)) / width * math.pi) + 1) / 2)
            if e <= 0.9999:
                for jj in (j, B + 1 - j):
                    for ii in (i, B + 1 - i):
                        E[jj - 1, ii - 1] = e
    fe = np.fft.rfft2(np.fft.fftshift(E)) / (B * B)
    d = neg + ref
    c = np.vdot(fe.ravel(), d.ravel()) / np.vdot(fe.ravel(), fe.ravel())
    assert np.max(np.abs(d - c * fe)) < 1e-10 * np.max(np.abs(ref))
