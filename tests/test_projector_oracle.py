"""CPU tests of the oracle's polar projector (expand_cmat + fproject_polar +
euler2m, simple_projector.f90:66-132 / :218-239 / :269-307, simple_ori.f90:1275):
its identity-orientation projection of a volume constant along the third axis
equals the (separately pinned) 2-D Kaiser-Bessel gridding of the slice, its
rotation matrices follow the reference's z-y-z convention, and projections of a
centred Gaussian volume reproduce the volume's analytic central sections."""
import math

import numpy as np


def _gauss_half(box, sigma):
    """half FT [m][k][h] of a centred 3-D Gaussian with per-axis std sigma = (sx, sy, sz) px
    (x along h, y along k, z along m): real, positive, anisotropic"""
    sx, sy, sz = (sigma, sigma, sigma) if np.isscalar(sigma) else sigma
    f = np.fft.fftfreq(box)
    h = np.arange(box // 2 + 1) / box
    arg = sz ** 2 * f[:, None, None] ** 2 + sy ** 2 * f[None, :, None] ** 2 + sx ** 2 * h[None, None, :] ** 2
    amp = (2 * math.pi) ** 1.5 * sx * sy * sz
    return (amp * np.exp(-2 * math.pi ** 2 * arg)).astype(np.complex64)


def test_identity_projection_equals_2d_gridding(O):
    box = 32
    g = O.geom(64, 2, 12, box)
    t = O.tables(g)
    rng = np.random.default_rng(3)
    half2d = (rng.standard_normal((box, box // 2 + 1)) + 1j * rng.standard_normal((box, box // 2 + 1))).astype(np.complex64)
    vol = np.repeat(half2d[None], box, axis=0)          # constant along m
    ex = O.expand_cmat3d(vol, box)
    # the z weights at loc_z = 0: normalised away, or a common factor without the normalisation
    zsum = sum(O.kb_apod(float(l)) for l in (-1, 0, 1))
    for griddev, factor in ((False, 1.0), (True, zsum)):
        p3 = O.fproject_polar(g, t, ex, box, [0.0, 0.0, 0.0], griddev=griddev)
        p2 = factor * O.polarize(g, t, half2d, griddev=griddev)
        assert np.max(np.abs(p3 - p2)) < 1e-12 * np.max(np.abs(p2))


def test_euler2m_convention(O):
    R = O.euler2m([31.0, 47.0, 113.0])
    assert np.max(np.abs(R @ R.T - np.eye(3))) < 1e-14 and abs(np.linalg.det(R) - 1.0) < 1e-14
    # rotmat(ang, 3) is the negative rotation about z: (1, 0, 0) -> (cos, sin, 0) as a row vector times R
    a = math.radians(30.0)
    Rz = O.euler2m([30.0, 0.0, 0.0])
    assert np.allclose(np.array([1.0, 0.0, 0.0]) @ Rz, [math.cos(a), math.sin(a), 0.0])
    # the tilt: (0, 0, 1) R2 = (sin, 0, cos)
    Ry = O.euler2m([0.0, 30.0, 0.0])
    assert np.allclose(np.array([0.0, 0.0, 1.0]) @ Ry, [math.sin(a), 0.0, math.cos(a)])
    # product order r3 r2 r1
    R3, R2, R1 = O.euler2m([0, 0, 113.0]), O.euler2m([0, 47.0, 0]), O.euler2m([31.0, 0, 0])
    assert np.allclose(R, R3 @ R2 @ R1)


def test_projection_of_gaussian_matches_central_sections(O):
    """the KB interpolation of a smooth, anisotropic (centred) volume FT at
    loc = (x, y, 0) R agrees with the analytic FT at that point, for every orientation
    (a wrong rotation convention would not)"""
    box, sig = 64, (1.0, 1.5, 2.0)
    g = O.geom(96, 2, 14, box)
    t = O.tables(g)
    ex = O.expand_cmat3d(_gauss_half(box, sig), box)
    N, P, K = g.nrots, g.pftsz, g.K
    pol = np.asarray(t.polar).reshape(K, 2 * N)
    x, y = pol[:, :P].astype(np.float64), pol[:, N:N + P].astype(np.float64)
    amp = (2 * math.pi) ** 1.5 * sig[0] * sig[1] * sig[2]
    for eul in ([0.0, 0.0, 0.0], [20.0, 50.0, 140.0], [250.0, 110.0, 10.0]):
        R = O.euler2m(eul)
        lx, ly, lz = (x * R[0, j] + y * R[1, j] for j in range(3))
        want = amp * np.exp(-2 * math.pi ** 2 * (sig[0] ** 2 * lx ** 2 + sig[1] ** 2 * ly ** 2 + sig[2] ** 2 * lz ** 2) / box ** 2)
        got = O.fproject_polar(g, t, ex, box, eul)
        err = np.max(np.abs(got - want)) / np.max(np.abs(want))
        assert err < 2e-2, (eul, err)
        assert np.max(np.abs(got.imag)) < 1e-6 * np.max(np.abs(want))
        # the transposed rotation would be far off
        lx2, ly2, lz2 = (x * R.T[0, j] + y * R.T[1, j] for j in range(3))
        wrong = amp * np.exp(-2 * math.pi ** 2 * (sig[0] ** 2 * lx2 ** 2 + sig[1] ** 2 * ly2 ** 2 + sig[2] ** 2 * lz2 ** 2) / box ** 2)
        if eul != [0.0, 0.0, 0.0]:
            assert np.max(np.abs(got - wrong)) / np.max(np.abs(want)) > 0.1


def test_mask_zeroes_shells(O):
    box = 32
    g = O.geom(64, 2, 12, box)
    t = O.tables(g)
    ex = O.expand_cmat3d(_gauss_half(box, 2.0), box)
    mask = np.ones(g.K, np.int32)
    mask[3:6] = 0
    p = O.fproject_polar(g, t, ex, box, [10.0, 20.0, 30.0], mask=mask)
    full = O.fproject_polar(g, t, ex, box, [10.0, 20.0, 30.0])
    assert np.all(p[3:6] == 0) and np.array_equal(p[mask == 1], full[mask == 1])
