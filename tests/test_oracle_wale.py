"""Per-cell relaxation field and WALE LES of the oracle, pinned to the
reference's own tests (crates/lbm-core/tests/wale_les.rs: constant omega
field identical to the field off, WALE null for steady Couette and
Poiseuille, the null update leaves a laminar duct unchanged, unclipped WALE
equal to the raw formula, tau_eff clipping diagnostics and monotonicity)."""
import numpy as np

from oracle import oracle as o

CW = 0.325


def idx(dims, x, y, z):
    return (z * dims[1] + y) * dims[0] + x


def channel(ny, nu, force=(0.0, 0.0, 0.0), top_u=0.0):
    dims = (4, ny, 4)
    wu = np.zeros(18)
    wu[9] = top_u
    solid, wall = o.wall_rims(dims, [False, False, True, True, False, False], wu)
    return o.OracleSolver(dims, q=19, real_bits=64, nu=nu, periodic=(True, False, True), force=force, solid=solid,
                          wall_u=wall)


def run_to_steady(s, every=500, tol=1e-11, max_steps=200_000):
    prev = s.moments()[1]
    for _ in range(max_steps // every):
        s.step(every)
        cur = s.moments()[1]
        if np.abs(cur - prev).max() / max(np.abs(cur).max(), 1.0) <= tol:
            return
        prev = cur
    raise AssertionError("no steady state")


def init_fields(dims, fn):
    n = int(np.prod(dims))
    rho, u = np.zeros(n), np.zeros((n, 3))
    for z in range(dims[2]):
        for y in range(dims[1]):
            for x in range(dims[0]):
                r, v = fn(x, y, z)
                rho[idx(dims, x, y, z)] = r
                u[idx(dims, x, y, z)] = v
    return rho, u.ravel()


def test_constant_omega_field_is_identical_to_field_off():
    dims, nu = (12, 10, 8), 0.03

    def f(x, y, z):
        xf, yf, zf = x * 0.13, y * 0.17, z * 0.19
        return 1.0 + 1e-4 * np.sin(xf + yf), [0.02 * np.sin(xf) * np.cos(yf), -0.015 * np.sin(yf) * np.cos(zf),
                                              0.01 * np.sin(zf) * np.cos(xf)]
    rho, u = init_fields(dims, f)
    off = o.OracleSolver(dims, q=19, real_bits=64, nu=nu, periodic=(True, True, True))
    on = o.OracleSolver(dims, q=19, real_bits=64, nu=nu, periodic=(True, True, True))
    off.init_with(rho, u)
    on.init_with(rho, u)
    on.set_omega_field(np.full(off.n, 1.0 / (3.0 * nu + 0.5)))
    off.step(7)
    on.step(7)
    band = 5.0 * np.finfo(np.float64).eps
    assert np.abs(off.stage_out() - on.stage_out()).max() <= band
    for a, b in zip(off.moments(), on.moments()):
        assert np.abs(a - b).max() <= band


def test_wale_null_for_steady_couette_and_poiseuille():
    couette = channel(10, (1.0 - 0.5) / 3.0, top_u=0.1)
    run_to_steady(couette)
    nu_t, _ = couette.wale_update()
    assert nu_t.max() <= 1e-12
    pois = channel(10, 0.1, force=(1e-6, 0.0, 0.0))
    run_to_steady(pois)
    nu_t, _ = pois.wale_update()
    assert nu_t.max() <= 1e-12


def test_les_on_does_not_change_laminar_duct_after_null_update():
    off = channel(10, 0.1, force=(1e-6, 0.0, 0.0))
    on = channel(10, 0.1, force=(1e-6, 0.0, 0.0))
    run_to_steady(off)
    run_to_steady(on)
    on.wale_update()
    off.step(20)
    on.step(20)
    for a, b in zip(off.moments()[1:], on.moments()[1:]):
        assert np.abs(a - b).max() <= 1e-12


def multimode(n=12, nu=0.02, u0=0.04):
    k1, k2, k3 = 2 * np.pi / n, 4 * np.pi / n, 6 * np.pi / n

    def f(x, y, z):
        m1 = [np.sin(k1 * x) * np.cos(k1 * y) * np.cos(k1 * z), -np.cos(k1 * x) * np.sin(k1 * y) * np.cos(k1 * z),
              0.0]
        m2 = [0.0, np.sin(k2 * y) * np.cos(k2 * z) * np.cos(k2 * x), -np.cos(k2 * y) * np.sin(k2 * z) * np.cos(k2 * x)]
        m3 = [-np.cos(k3 * z) * np.sin(k3 * x) * np.cos(k3 * y), 0.0, np.sin(k3 * z) * np.cos(k3 * x) * np.cos(k3 * y)]
        return 1.0, [u0 * (m1[i] + m2[i] + m3[i]) for i in range(3)]
    dims = (n, n, n)
    s = o.OracleSolver(dims, q=19, real_bits=64, nu=nu, periodic=(True, True, True))
    rho, u = init_fields(dims, f)
    s.init_with(rho, u)
    return s


def raw_wale(g):
    s = 0.5 * (g + np.swapaxes(g, 1, 2))
    g2 = np.einsum("nik,nkj->nij", g, g)
    tr = np.trace(g2, axis1=1, axis2=2)
    sd = 0.5 * (g2 + np.swapaxes(g2, 1, 2)) - np.eye(3)[None] * (tr / 3.0)[:, None, None]
    ss = (s * s).sum(axis=(1, 2))
    sdsd = (sd * sd).sum(axis=(1, 2))
    den = ss ** 2.5 + sdsd ** 1.25
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(den > 0, CW * CW * sdsd ** 1.5 / den, 0.0)


def test_wale_unset_clipping_matches_raw_wale():
    s = multimode()
    expected = raw_wale(s.velocity_gradient())
    assert (expected > 0).any()
    nu_t, d = s.wale_update()
    assert np.abs(nu_t - expected).max() <= 1e-15 * expected.max()
    assert d["clipped_cells"] == 0 and d["clipped_fraction"] == 0.0
    assert abs(d["max_nu_t_before_clipping"] - expected.max()) <= 1e-15 * expected.max()
    assert d["tau_eff_max"] is None and d["nu_t_max"] is None


def test_wale_tau_eff_clipping_diagnostics_match_reference():
    nu = 0.02
    s = multimode(nu=nu)
    raw, _ = multimode(nu=nu).wale_update()
    cap = np.sort(raw)[raw.size // 4]
    tau_max = 0.5 + 3.0 * (nu + cap)
    nu_t, d = s.wale_update(tau_max)
    active = d["nu_t_max"]
    expected_clipped = int((raw > active).sum())
    assert expected_clipped > 0
    assert d["clipped_cells"] == expected_clipped
    assert d["clipped_fraction"] == expected_clipped / raw.size
    assert d["max_nu_t_before_clipping"] == raw.max()
    assert np.array_equal(nu_t, np.where(raw > active, active, raw))


def test_wale_clipping_count_is_monotone_with_bound():
    nu = 0.02
    raw, _ = multimode(nu=nu).wale_update()
    counts = []
    for frac in (0.25, 0.5, 0.75):
        _, d = multimode(nu=nu).wale_update(0.5 + 3.0 * (nu + frac * raw.max()))
        counts.append(d["clipped_cells"])
    assert counts[0] >= counts[1] >= counts[2]
