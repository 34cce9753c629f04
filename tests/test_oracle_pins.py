"""The oracle pinned by the reference's own known-answer tests, restated (not copied):
sh.zig:441-606, lambert.zig:66-85, geometry.zig:195-235, master.zig:811-850 (on a synthetic
master), and the sphere/correlation path checked against the quadrature integral."""
import math

import numpy as np

from oracle import geometry, lambert, rot, sh, spherical


def test_gauss_legendre_integrates_polynomials():
    # sh.zig:441-454
    x, w = sh.gauss_legendre(12)
    assert abs(w.sum() - 2) < 1e-13
    assert abs((w * x ** 22).sum() - 2.0 / 23.0) < 1e-13
    assert x[0] > x[11]


def test_analysis_inverts_synthesis_and_parseval():
    # sh.zig:456-482
    L = 12
    g = sh.Grid(L, 16, 32)
    rng = np.random.default_rng(7)
    ms, _ = sh.pair_table(L)
    coef = (rng.random(len(ms)) - 0.5) + 1j * np.where(ms == 0, 0.0, rng.random(len(ms)) - 0.5)
    s = g.synthesize(coef)
    back = g.analyze(s)
    assert np.abs(back - coef).max() < 1e-12
    e = (g.w[:, None] * (2 * math.pi / 32) * s.reshape(16, 32) ** 2).sum()
    assert abs(sh.power(L, coef) - e) < 1e-11


def test_wigner_half_pi_matches_general_formula_and_factorizes():
    # sh.zig:484-519
    L = 9
    tab = sh.wigner_half_pi(L)
    for l in range(L):
        for k in range(-l, l + 1):
            for m in range(-l, l + 1):
                assert abs(sh.wigner_small_d(l, k, m, math.pi / 2) - sh.d_half_pi(tab, l, k, m)) < 1e-11
    beta = 0.83
    l = 5
    for mp in range(-l, l + 1):
        for m in range(-l, l + 1):
            acc = 0j
            for k in range(-l, l + 1):
                dd = sh.d_half_pi(tab, 5, k, mp) * sh.d_half_pi(tab, 5, k, m)
                acc += dd * complex(math.cos(k * beta), -math.sin(k * beta))
            acc *= sh.ipow(mp - m)
            assert abs(sh.wigner_small_d(l, mp, m, beta) - acc.real) < 1e-11
            assert abs(acc.imag) < 1e-11


def _ylm(L, l, m, v):
    p = sh.legendre_all(L, v[2])
    am = abs(m)
    phi = math.atan2(v[1], v[0])
    val = p[sh.pair(L, am, l)]
    s = 1.0 if (m >= 0 or am % 2 == 0) else -1.0
    return s * val * complex(math.cos(m * phi), math.sin(m * phi))


def test_harmonics_rotate_by_d():
    # sh.zig:521-548
    L = 6
    a, b, c = 0.7, 1.1, -0.4
    S = rot.from_zyz(a, b, c)
    x = np.array([0.3, -0.5, 0.6])
    x /= np.linalg.norm(x)
    xr = rot.qapply(rot.qconj(S), x)
    l = 4
    for m in range(-4, 5):
        lhs = _ylm(L, l, m, xr)
        rhs = 0j
        for mp in range(-4, 5):
            ang = -(mp * a + m * c)
            dv = sh.wigner_small_d(4, mp, m, b)
            rhs += dv * complex(math.cos(ang), math.sin(ang)) * _ylm(L, l, mp, x)
        assert abs(lhs - rhs) < 1e-12


def test_correlation_formula_equals_integral():
    # sh.zig:550-594
    L = 6
    tab = sh.wigner_half_pi(L)
    rng = np.random.default_rng(3)
    ms, _ = sh.pair_table(L)
    f = (rng.random(len(ms)) - 0.5) + 1j * np.where(ms == 0, 0, rng.random(len(ms)) - 0.5)
    g = (rng.random(len(ms)) - 0.5) + 1j * np.where(ms == 0, 0, rng.random(len(ms)) - 0.5)
    grid = sh.Grid(L, 24, 48)
    gs = grid.synthesize(g)
    a, b, c = 0.9, 0.6, 2.2
    R = rot.qconj(rot.from_zyz(a, b, c))
    dirs = grid.directions().reshape(-1, 3)
    v = rot.qapply(R, dirs)
    fgrid = sh.Grid(L, 2, 2)  # only for its pair layout
    p = sh.legendre_all(L, v[:, 2])
    phi = np.arctan2(v[:, 1], v[:, 0])
    fv = np.zeros(len(v))
    for idx, (m, l) in enumerate(zip(*sh.pair_table(L))):
        k = 1.0 if m == 0 else 2.0
        fv += k * p[idx] * (f[idx].real * np.cos(m * phi) - f[idx].imag * np.sin(m * phi))
    w = np.repeat(grid.w, 48) * (2 * math.pi / 48)
    integral = (w * gs * fv).sum()
    assert abs(integral - sh.correlation_at(L, tab, f, g, a, b, c)) < 1e-10
    del fgrid


def test_rules_are_read_from_coefficients():
    # sh.zig:596-606
    L = 8
    coef = np.zeros(sh.pair_count(L), complex)
    for m in range(L):
        for l in range(m, L):
            if m % 4 == 0 and l % 2 == 0:
                coef[sh.pair(L, m, l)] = 1 + 0.5j
    r = sh.Rules.detect(L, coef, 1e-6)
    assert r.n_fold == 4 and r.mirror and r.inversion
    assert r.allows(4, 4) and not r.allows(5, 4) and not r.allows(4, 2)


def test_lambert_inverts_with_equal_area():
    # lambert.zig:66-85
    pts = [(0.3, -0.7), (-0.9, 0.2), (0.0, 0.5), (1.0, 1.0), (-0.01, 0.01)]
    for x, y in pts:
        for south in (False, True):
            v = lambert.square_to_sphere(x, y, south)
            assert abs(np.linalg.norm(v) - 1) < 1e-13
            assert (v[2] <= 1e-12) == south or abs(v[2]) < 1e-12
            q = lambert.sphere_to_square(v)
            assert abs(q[0] - x) < 1e-10 and abs(q[1] - y) < 1e-10
    h = 1e-6
    for x, y in pts[:3]:
        dx = (lambert.square_to_sphere(x + h, y, False) - lambert.square_to_sphere(x - h, y, False)) / (2 * h)
        dy = (lambert.square_to_sphere(x, y + h, False) - lambert.square_to_sphere(x, y - h, False)) / (2 * h)
        assert abs(np.linalg.norm(np.cross(dx, dy)) - math.pi / 2) < 1e-6


def test_pattern_centre_and_pose_are_two_views():
    # geometry.zig:195-221
    g = geometry.Geometry(pc=(0.42, 0.21, 0.5), rot_vec=(0.01, -0.02, 0.005))
    R = g.rotation()
    t = g.translation(60, 80)
    pc = geometry.Geometry.pc_of(R, t, 60, 80)
    assert np.abs(pc - g.pc).max() < 1e-13
    n = R[:, 2]
    assert abs(np.dot(n, t) - 0.5 * 60.0) < 1e-10
    h = geometry.Geometry(rot_vec=(0, math.radians(3.0), 0))
    tilted = geometry.Geometry(detector_tilt_deg=3)
    assert np.abs(h.rotation() - tilted.rotation()).max() < 1e-12
    g.rot = np.zeros(3)
    t0 = g.translation(60, 60)
    a = math.radians(-70.0)
    assert abs(0.21 * 60 * math.sin(a) + 0.5 * 60 * math.cos(a) - math.sin(a) / 2.0 - t0[0]) < 1e-10
    assert abs(-60.0 * 0.42 + 0.5 - t0[1]) < 1e-10
    assert abs(0.21 * 60 * math.cos(a) - 0.5 * 60 * math.sin(a) - math.cos(a) / 2.0 - t0[2]) < 1e-10
    tr = g.translation(61.0 / 2.5, 61.0 / 2.5)
    back = geometry.Geometry.pc_of(g.rotation(), tr, 61.0 / 2.5, 61.0 / 2.5)
    assert np.abs(back - g.pc).max() < 1e-13


def test_beam_travel_matches_kikuchipy_extrapolation():
    # geometry.zig:223-235
    g = geometry.Geometry(pc=(0.42, 0.21, 0.5), px_um=70, step_x_um=1.5, step_y_um=1.5)
    R = g.rotation()
    t = g.translation(60, 60)
    s = g.scan_offset(1, 1, 0, 0, -1, -1, 8)
    pc = geometry.Geometry.pc_of(R, t - s, 60, 60)
    f = 1.5 / (70.0 * 8.0 * 60.0)
    alpha = math.radians(20.0)
    assert abs(0.42 - f - pc[0]) < 1e-12
    assert abs(0.21 - f * math.cos(alpha) - pc[1]) < 1e-12
    assert abs(0.5 + f * math.sin(alpha) - pc[2]) < 1e-12


def test_fft_size_and_grids():
    # spherical.zig:100-104: n is the next power of two ≥ 2L − 1, from 16
    assert [spherical.fft_size(L) for L in (8, 16, 32, 64, 128)] == [16, 32, 64, 128, 256]


def test_six_unknown_system_is_consistent():
    """The oracle's restatement of the six-unknown sums (detector.wgsl `sums`) and localOf
    (planefit.zig:176-200): its gradient is that of the NCC it reports up to the gradient table's
    discretization (a central difference a master pixel wide) — the same direction, a few percent
    apart — and its pivoted solve (planefit.zig:203-233) inverts a damped system; settle raises
    the NCC from a start 1° off."""
    import math

    import oracle.detector as od
    import oracle.geometry as og
    import oracle.rot as rot

    rng = np.random.default_rng(4)
    side = 101
    # a smooth master: a few low-order terms on the sheets' directions
    d = od.pixel_dirs(side)
    sheets = np.sin(3 * d[:, 0]) * np.cos(2 * d[:, 1]) + 0.5 * d[:, 2] ** 2 + 0.3 * np.sin(4 * d[:, 1] + d[:, 2])
    sheets = (sheets - sheets.mean()) / sheets.std()
    grad = od.gradient_table(sheets, side)
    geo = og.Geometry(pc=(0.5, 0.3, 0.6), sample_tilt_deg=70.0)
    fr, mask, t = geo.frame(), og.mask_of(40, 40), geo.translation(40, 40)
    q = rot.qstd(rng.normal(size=4))
    pat = od.project(sheets, side, fr, t, q, 40, 40)
    m_ = od.in_mask(40, 40, mask)
    pat = np.where(m_, pat - pat[m_].mean(), 0.0)
    pat /= np.linalg.norm(pat)
    q1 = rot.qmul(rot.so3_exp([0.004, -0.006, 0.005]), q)
    sh = np.array([0.2, -0.1, 0.3])
    ncc, g, H = od.local_of(od.sums6(grad, side, fr, t, q1, sh, pat, mask))

    def f(x):
        return od.local_of(od.sums6(grad, side, fr, t, rot.qmul(rot.so3_exp(x[3:]), q1), sh + x[:3], pat, mask))[0]

    fd = np.array([(f(np.eye(6)[i] * 1e-5) - f(-np.eye(6)[i] * 1e-5)) / 2e-5 for i in range(6)])
    cos = g @ fd / (np.linalg.norm(g) * np.linalg.norm(fd))
    assert cos > 0.99 and np.linalg.norm(g - fd) < 0.1 * np.linalg.norm(fd), (g, fd)
    A, b = od.damped(H, g, 1e-3)
    x = od.solve_pivot(A, b)
    assert np.allclose(A @ x, b, rtol=1e-10, atol=1e-12)
    q0 = rot.qmul(rot.so3_exp(np.radians([0.6, -0.5, 0.4])), q)
    start = od.local_of(od.sums6(grad, side, fr, t, q0, np.zeros(3), pat, mask))[0]
    qe, she, ncce, it = od.settle6(grad, side, fr, t, q0, pat, mask, trust=2.0, most=40)
    assert ncce > start and ncce > 0.99 and it >= 1
    assert math.degrees(2 * math.acos(min(1.0, abs(float(np.dot(rot.qstd(qe), rot.qstd(q))))))) < 0.2


def test_reduction_matches_reduce_zig_tests():
    """reduce.zig:151-215's assertions on the oracle's reduction: a whole factor is block
    binning (u8 6 × 8 by 2; 7 × 9 by 3 with the remainder dropped, u16 and f32 alike); any
    factor conserves the total (10 × 10 by 2.5), the first pixel by hand, a flat pattern stays flat."""
    import oracle.prep as op

    src = np.array([(i * 7 + 3) % 251 for i in range(48)], np.float64).reshape(6, 8)
    got = op.reduce(src, 2)
    want = src.reshape(3, 2, 4, 2).mean((1, 3))
    assert np.allclose(got, want, atol=1e-5)
    assert op.reduced_shape(7, 9, 2) == (3, 4)
    v = np.array([(i * 977 + 31) % 60000 for i in range(63)], np.float64).reshape(7, 9)
    a = op.reduce(v.astype(np.uint16), 3)
    b = op.reduce(v.astype(np.float32), 3)
    assert a.shape == (2, 3) and np.allclose(a, b, rtol=1e-6)
    s10 = np.array([(i * 37 + 11) % 1000 for i in range(100)], np.float64).reshape(10, 10)
    d = op.reduce(s10, 2.5)
    assert d.shape == (4, 4) and abs(d.sum() * 6.25 - s10.sum()) < 1e-5 * s10.sum()
    wr = np.array([1, 1, 0.5])
    assert abs(d[0, 0] - (wr[:, None] * wr[None, :] * s10[:3, :3]).sum() / 6.25) < 1e-5 * d[0, 0]
    flat = op.reduce(np.full((10, 10), 7.0), 3)
    assert flat.shape == (3, 3) and np.allclose(flat, 7.0)


def test_cubochoric_map_matches_rot_zig_tests():
    """rot.zig:330-355's assertions on the oracle's cubochoric and homochoric maps: a face centre
    lands on the ball's surface (radius (3π/4)^(1/3)); unit Jacobian determinant inside each
    pyramid; |h|³ = (3/4)(θ − sin θ)."""
    import oracle.dictionary as odict

    top = odict.cu_to_ho((0.0, 0.0, odict.CUBOCHORIC_HALF_EDGE))
    assert abs(top[2] - (0.75 * math.pi) ** (1 / 3)) < 1e-12
    for c in [(0.21, -0.33, 0.87), (-0.9, 0.2, 0.4), (0.1, 0.8, -0.35), (0.05, 0.02, 0.01)]:
        J = np.zeros((3, 3))
        for j in range(3):
            cp, cm = list(c), list(c)
            cp[j] += 1e-6
            cm[j] -= 1e-6
            J[:, j] = (np.array(odict.cu_to_ho(cp)) - np.array(odict.cu_to_ho(cm))) / 2e-6
        assert abs(np.linalg.det(J) - 1) < 1e-6
    q = odict.from_homochoric((0.3, 0.4, 0.5))
    th = 2 * math.acos(q[0])
    assert abs(0.75 * (th - math.sin(th)) - math.sqrt(0.5) ** 3) < 1e-12


def test_generators_match_published_vectors():
    """SplitMix64 from seed 0 and xoshiro256++ from the state (1, 2, 3, 4): the published first
    outputs of Vigna's reference implementations."""
    import oracle.dictionary as odict

    g = odict.SplitMix64(0)
    assert [g.next() for _ in range(3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]
    x = odict.Xoshiro256(0)
    x.s = [1, 2, 3, 4]
    assert [x.next() for _ in range(4)] == [41943041, 58720359, 3588806011781223, 3591011842654386]


def test_dictionary_grid_equals_its_restatement():
    """The package's vectorized dictionary (grid, zone, shuffle) is the oracle's entry for entry."""
    import oracle.dictionary as odict
    from zebsdsolve_b200 import dictionary as DI
    from zebsdsolve_b200 import rotations as R

    for g in ("o", "d6"):
        rots = R.group(g)
        for N in (3, 7):
            a = odict.dictionary(N, rots)
            b = DI.cubochoric_grid(N, rots)
            assert a.shape == b.shape and np.array_equal(a, b), (g, N)
