"""The adaptive kappa rule of the Dirac-3D current density on the oracle (CPU).

Reference: DiracSystem::compute_current_density (DiracSystem.cpp:271-331)
integrates kappa with split_integrate<100>(f, 0, kappa_max, n_kappa = 10,
threshold = 1e-3, elementwise error) from its author's library, which is not
available; ``oracle.adaptive_kappa`` restates the rule from that call (equal
splits, trapezoid halving until the elementwise change drops below the
threshold).  These tests pin the restatement by its defining properties:
exactness on linear integrands, convergence to the integral, refinement only
where the integrand needs it, and the symmetry of the Dirac current; its
first trapezoid is pinned to the reference's own fixed kappa rule
(sources/debug_output.cpp:69-95).
"""
import math

import numpy as np

from oracle import hhg_oracle as O


def _synthetic(g, kappa_max=1.0, n_kappa=4, threshold=1e-6, n_splits=4, max_halvings=12,
               n_samples=3):
    """adaptive_kappa on one slice with rows (0, kappa, 0, end factor) and
    contributions w g(kappa, sample)."""
    def rows_fn(z, a, H, L):
        panels = n_kappa << L
        h = H / panels
        idx = range(0, panels + 1) if L == 0 else range(1, panels, 2)
        out = []
        for i in idx:
            end = 0.5 if L == 0 and i in (0, panels) else 1.0
            out.append([0.0, a + i * h, 0.0, end, 0, 0, 0, 0])
        return np.array(out).reshape(-1, 8)

    def contrib(rows):
        k = rows[:, 1]
        return np.stack([rows[:, 3] * g(k, i) for i in range(n_samples)])

    return O.adaptive_kappa(contrib, [0.0], [kappa_max], n_kappa, threshold, n_splits,
                            max_halvings, 1.0, n_samples, rows_fn)


def test_linear_integrand_is_exact_after_one_halving():
    j, info = _synthetic(lambda k, i: (i + 1) * (2.0 * k - 0.25))
    exact = [(i + 1) * (1.0 - 0.25) for i in range(3)]
    assert np.allclose(j, exact, rtol=0, atol=1e-15)
    # the first trapezoid is already exact: one halving confirms it
    assert info["rounds"] == 2 and info["max_level"] == 1 and info["unconverged"] == 0
    assert info["trajectories"] == 4 * (4 + 1) + 4 * 4


def test_converges_to_the_integral():
    g = lambda k, i: np.sin((3 + i) * k) * np.exp(-k)
    exact = [((3 + i) - math.exp(-2) * ((3 + i) * math.cos(2 * (3 + i)) + math.sin(2 * (3 + i))))
             / (1 + (3 + i) ** 2) for i in range(3)]
    for thr in (1e-4, 1e-6, 1e-8):
        j, info = _synthetic(g, kappa_max=2.0, threshold=thr)
        assert info["unconverged"] == 0
        # the trapezoid error after the last halving is about a third of the
        # last change per split
        assert np.max(np.abs(j - exact)) <= 4 * thr, (thr, np.abs(j - exact))


def test_refines_only_the_splits_that_need_it():
    # a narrow bump inside the first of 8 splits
    g = lambda k, i: np.exp(-((k - 0.05) / 0.01) ** 2)
    j, info = _synthetic(g, kappa_max=1.0, threshold=1e-9, n_splits=8)
    assert info["unconverged"] == 0 and info["max_level"] >= 3
    # every split refined as deep as the bump's: 8 (5 + 4 (2^L - 1)) nodes
    uniform = 8 * (5 + 4 * ((1 << info["max_level"]) - 1))
    assert info["trajectories"] < uniform / 3
    assert abs(j[0] - 0.01 * math.sqrt(math.pi)) <= 1e-9


def test_halving_cap_reports_unconverged_splits():
    g = lambda k, i: np.sin(200 * k)
    j, info = _synthetic(g, threshold=1e-12, max_halvings=3)
    assert info["max_level"] == 3 and info["unconverged"] == 4


def _dirac_case(sign=1.0, beta=0.0, fermi=0.0):
    m = O.model(O.DIRAC3D, beta=beta, fermi_energy=fermi)
    p = O.Pulse(sign * 0.6, 1, 0.0)
    tc = O.time_config(0.0, 2 * math.pi, 96)
    return m, p, tc, O.solver(stepper=2)


def test_dirac_current_is_odd_in_the_field():
    # even n_z: the k_z slices are symmetric, and (k_z, A) -> (-k_z, -A) maps
    # S -> (-S_x, -S_y, S_z) for the T = 0 start (S_x = 0) while the weight
    # k_z kappa / |k| changes sign
    args = dict(max_k=2.5, n_z=6, n_kappa=3, threshold=1e-5, n_splits=3, max_halvings=6)
    jp, ip, rp = O.dirac_kappa_current(*_dirac_case(1.0), **args)
    jm, im, rm = O.dirac_kappa_current(*_dirac_case(-1.0), **args)
    assert rp == 0 and rm == 0
    assert ip == im
    assert np.max(np.abs(jp + jm)) <= 1e-12 * np.max(np.abs(jp))
    assert np.max(np.abs(jp)) > 1e-3
    # no field: the equilibrium is stationary, and the k_z-odd weight sums to 0
    m, p, tc, s = _dirac_case()
    j0, _, _ = O.dirac_kappa_current(m, O.Pulse(0.0, 1, 0.0), tc, s, **args)
    assert np.max(np.abs(j0)) <= 1e-12


def test_dirac_quadrature_converges_to_gauss_legendre():
    # each slice's kappa integral against a 200-point Gauss-Legendre rule of
    # the same trajectories
    m, p, tc, s = _dirac_case(beta=4.0, fermi=0.3)
    max_k, n_z = 2.0, 4
    j, info, rc = O.dirac_kappa_current(m, p, tc, s, max_k=max_k, n_z=n_z, n_kappa=4,
                                        threshold=1e-7, n_splits=2, max_halvings=10)
    assert rc == 0 and info["unconverged"] == 0
    dz = 2 * max_k / n_z
    x, w = np.polynomial.legendre.leggauss(200)
    ref = np.zeros(tc.n_measurements + 1)
    for z in range(1, n_z):
        if z == n_z // 2:
            continue
        kz = (z - n_z // 2) * dz
        km = math.sqrt(max_k * max_k - kz * kz)
        rows = []
        for xi, wi in zip(x, w):
            kap = 0.5 * km * (xi + 1)
            mk = math.hypot(kz, kap)
            rows.append([kz, kap, mk, 0.5 * km * wi * kz * kap / mk,
                         *O.initial_state(m, kz, kap, 0.0), 0.0])
        out, rc = O.k_resolved(m, p, tc, s, np.array(rows), 0)
        assert rc == 0
        ref += out[:, :, 2] @ np.array(rows)[:, 3]
    ref *= dz
    assert np.max(np.abs(j - ref)) <= 1e-5 * np.max(np.abs(ref)), np.max(np.abs(j - ref))


def test_first_trapezoid_matches_the_reference_fixed_rule():
    # the reference's fixed kappa trapezoid (sources/debug_output.cpp:69-95):
    # kappa = r dkappa, r = 1 .. n_kappa, weight (r == n_kappa ? 1/2 : 1)
    # dkappa dz k_z kappa / |k|, nothing at kappa = 0; one split's first
    # trapezoid of the adaptive rule (n_splits = 1) takes the same nodes and
    # weights
    m, p, tc, s = _dirac_case(beta=2.0, fermi=0.1)
    max_k, n_z, n_kappa = 2.0, 6, 7
    dz = 2 * max_k / n_z
    ref = np.zeros(tc.n_measurements + 1)
    ours = np.zeros(tc.n_measurements + 1)
    for z in range(1, n_z):
        k_z = (z - n_z // 2) * dz
        kmax = math.sqrt(max_k * max_k - k_z * k_z)
        dk = kmax / n_kappa
        rows = []
        for r in range(1, n_kappa + 1):
            kappa = r * dk
            mk = math.sqrt(k_z * k_z + kappa * kappa)
            w = (0.5 if r == n_kappa else 1.0) * dk * dz * (k_z * kappa / mk)
            rows.append([k_z, kappa, mk, w, *O.initial_state(m, k_z, kappa, 0.0), 0.0])
        out, rc = O.k_resolved(m, p, tc, s, np.array(rows), 0)
        assert rc == 0
        ref += out[:, :, 2] @ np.array(rows)[:, 3]
        if z == n_z // 2:
            continue  # weight 0 (k_z = 0): the adaptive rule skips the slice
        mine = O.kappa_rows(m, k_z, 0.0, kmax, 0, n_kappa)
        assert mine.shape[0] == n_kappa  # kappa = 0 left out
        assert np.allclose(mine[:, 1], np.array(rows)[:, 1], rtol=1e-15, atol=0)
        out, rc = O.k_resolved(m, p, tc, s, mine, 0)
        ours += (kmax / n_kappa) * (out[:, :, 2] @ mine[:, 3])
    ours *= dz
    assert np.max(np.abs(ours - ref)) <= 1e-13 * np.max(np.abs(ref))
