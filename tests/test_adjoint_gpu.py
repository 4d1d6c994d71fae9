"""Discrete adjoint (GPU): gradients of a gauge misfit with respect to the
element-mean Manning n and the bathymetry modes HB against central finite
differences of the same FP64 forward, on a smooth always-wet basin of
10,112 elements (no limiter, no WETDRY), 300 steps of 0.5 s with a short
tidal ramp so that the wave crosses the gauges (x within 2.5 km of the open
edge).
Observations: a forward run with Manning n 50 % larger.  Bar: 1e-4
relative."""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks
from dgswem_b200._abi import DgswemError
from dgswem_b200.adjoint import GaugeMisfitProblem, element_manning, locate_gauges

pytestmark = pytest.mark.gpu

RTOL_FD = 1e-4
NSTEPS = 300


@pytest.fixture(scope="module")
def problem(tmp_path_factory):
    from dgswem_b200 import build
    build.build_library()
    path = decks.smooth_basin(tmp_path_factory.mktemp("adj") / "basin", nsteps=NSTEPS, dt=0.5, dramp=0.002)
    deck = Deck(path)
    ne = deck.s.ne
    rng = np.random.default_rng(3)
    xy = np.column_stack([rng.uniform(300.0, 2500.0, 16), rng.uniform(300.0, 3700.0, 16)])
    elem, phi = locate_gauges(deck, xy)
    n0 = element_manning(deck)
    hb0 = deck.real_array("hb", 3 * ne).reshape(ne, 3)
    truth = GaugeMisfitProblem(deck, elem, phi, NSTEPS)
    truth.set_params(nbar=1.5 * n0)
    obs = truth.run()
    truth.close()
    prob = GaugeMisfitProblem(deck, elem, phi, NSTEPS, obs=obs)
    yield deck, prob, n0, hb0, elem
    prob.close()
    deck.close()


def misfit(prob, nbar, hb):
    prob.set_params(nbar, hb)
    return prob.forward()


def smooth_hb_direction(deck, seed):
    """A continuous bathymetry perturbation: a few random plane waves of 2 km
    scale at the nodes, projected to HB modes with the p=1 corner map.  (A
    per-element white-noise direction makes the LLF wave-speed maximum switch
    sides at edges within the FD step, where the flux is not differentiable,
    and the central difference stops converging to any derivative.)"""
    s = deck.s
    nm = deck.int_array("nm", 3 * s.ne).reshape(3, s.ne) - 1
    x, y = deck.real_array("x", s.np), deck.real_array("y", s.np)
    r = np.random.default_rng(seed)
    f = np.zeros(s.np)
    for _ in range(4):
        kx, ky = r.uniform(-np.pi / 1000.0, np.pi / 1000.0, 2)
        f += r.normal() * np.sin(kx * x + ky * y + r.uniform(0.0, 2 * np.pi))
    v1, v2, v3 = f[nm[0]], f[nm[1]], f[nm[2]]
    return np.stack([(v1 + v2 + v3) / 3.0, -(v1 + v2) / 6.0 + v3 / 3.0, (-v1 + v2) / 2.0], 1)


def test_gradient_matches_central_differences(problem):
    deck, prob, n0, hb0, _ = problem
    ne = deck.s.ne
    j0 = misfit(prob, n0, hb0)
    gn, ghb = prob.gradient()
    assert j0 > 0 and np.abs(gn).max() > 0 and np.abs(ghb).max() > 0
    rng = np.random.default_rng(11)
    dn = n0 * rng.standard_normal(ne)
    dh = smooth_hb_direction(deck, 7)
    cases = [("nbar", dn, np.zeros((ne, 3)), 1e-4), ("hb", np.zeros(ne), dh, 1e-4), ("both", dn, dh, 1e-4)]
    for name, dn, dh, eps in cases:
        jp = misfit(prob, n0 + eps * dn, hb0 + eps * dh)
        jm = misfit(prob, n0 - eps * dn, hb0 - eps * dh)
        fd = (jp - jm) / (2 * eps)
        ad = float(gn @ dn + np.sum(ghb * dh))
        print(f"{name}: adjoint {ad:.10e} central FD {fd:.10e} rel {abs(ad - fd) / abs(fd):.2e}")
        assert abs(ad - fd) <= RTOL_FD * abs(fd), name
    prob.set_params(n0, hb0)


def test_gradient_of_one_gauge_element(problem):
    """A single parameter: the Manning n of the element holding a gauge."""
    deck, prob, n0, hb0, elem = problem
    j0 = misfit(prob, n0, hb0)
    gn, _ = prob.gradient()
    e = int(elem[0]) - 1
    d = np.zeros_like(n0)
    d[e] = n0[e]
    eps = 1e-3
    fd = (misfit(prob, n0 + eps * d, hb0) - misfit(prob, n0 - eps * d, hb0)) / (2 * eps)
    ad = gn[e] * n0[e]
    print(f"element {e}: adjoint {ad:.10e} central FD {fd:.10e} J {j0:.6e}")
    assert abs(ad - fd) <= RTOL_FD * abs(fd)
    prob.set_params(n0, hb0)


def test_stepwise_entry_points_match_the_sweep(problem):
    """Step-wise driving (state slots, adjoint_seed / adjoint_step, each step
    recomputed) gives the sweep's gradient bit for bit."""
    deck, prob, n0, hb0, _ = problem
    misfit(prob, n0, hb0)
    gn, ghb = prob.gradient()
    gn2, ghb2 = prob.gradient_stepwise()
    np.testing.assert_array_equal(gn2, gn)
    np.testing.assert_array_equal(ghb2, ghb)


def test_torch_autograd_function(problem):
    import torch
    from dgswem_b200.adjoint import GaugeMisfit
    deck, prob, n0, hb0, _ = problem
    nb = torch.tensor(n0, dtype=torch.float64, requires_grad=True)
    hb = torch.tensor(hb0, dtype=torch.float64, requires_grad=True)
    j = GaugeMisfit.apply(nb, hb, prob)
    j.backward()
    gn, ghb = prob.gradient()
    assert float(j) == pytest.approx(misfit(prob, n0, hb0), rel=0, abs=0)
    np.testing.assert_array_equal(nb.grad.numpy(), gn)
    np.testing.assert_array_equal(hb.grad.numpy(), ghb)


def test_adjoint_rejects_barriers(built):
    """The wetdry golden deck has barrier edges, which the adjoint does not cover."""
    from conftest import golden_dir
    from dgswem_b200 import _abi
    with HydroStep(Deck(golden_dir("wetdry"))) as hs:
        with pytest.raises(DgswemError, match="barrier"):
            _abi.check(hs._lib.dgswem_cuda_adjoint_begin(hs._h))


@pytest.fixture(scope="module")
def limiter_problem(tmp_path_factory):
    """The basin with slope limiter 5 on: the limiter clamps at the extrema
    of the incoming wave, and its adjoint runs with the forward's branches
    frozen."""
    from dgswem_b200 import build
    build.build_library()
    n = 200
    path = decks.smooth_basin(tmp_path_factory.mktemp("adjlim") / "basin", nsteps=n, dt=0.5, dramp=0.002,
                              slopeflag=5)
    deck = Deck(path)
    rng = np.random.default_rng(5)
    elem, phi = locate_gauges(deck, np.column_stack([rng.uniform(300.0, 2000.0, 16), rng.uniform(300.0, 3700.0, 16)]))
    n0 = element_manning(deck)
    hb0 = deck.real_array("hb", 3 * deck.s.ne).reshape(deck.s.ne, 3)
    truth = GaugeMisfitProblem(deck, elem, phi, n)
    truth.set_params(nbar=1.5 * n0)
    obs = truth.run()
    truth.close()
    prob = GaugeMisfitProblem(deck, elem, phi, n, obs=obs)
    yield deck, prob, n0, hb0
    prob.close()
    deck.close()


def test_limiter_reverse_mode_dot_product(built, scratch):
    """The limiter's reverse mode (frozen branches) against central
    differences of the forward limiter itself, as a dot-product test:
    <(L(x + e d) - L(x - e d)) / 2e, mu> = <d, L^T mu>.  The limiter is
    piecewise linear, and its redistribution is discontinuous where a vertex
    difference changes sign (the divisor max(1, kdp) jumps), so the misfit of
    a limited run is not differentiable in the parameters and an end-to-end
    difference quotient does not converge; on one application at a seeded
    O(1) state (every element clamped somewhere, no ties) a step of 1e-7
    changes no branch."""
    from dgswem_b200 import _abi
    from dgswem_b200.adjoint import _dp
    path = decks.smooth_basin(scratch / "limvjp", nx=12, ny=4, nsteps=2, slopeflag=5)
    with HydroStep(Deck(path)) as hs:
        ne = hs.ne
        rng = np.random.default_rng(21)
        x = [np.ascontiguousarray(rng.standard_normal((ne, 3))) for _ in range(3)]
        wd = np.ones(ne, np.int32)
        mu = [np.ascontiguousarray(rng.standard_normal((ne, 3))) for _ in range(3)]
        d = [rng.standard_normal((ne, 3)) for _ in range(3)]
        g = [np.empty((ne, 3)) for _ in range(3)]
        hs.set_state(*x, wd)
        _abi.check(hs._lib.dgswem_cuda_limiter_vjp(hs._h, *[_dp(m) for m in mu], *[_dp(a) for a in g]))
        eps = 1e-7
        out = []
        for sgn in (1.0, -1.0):
            hs.set_state(*(np.ascontiguousarray(x[v] + sgn * eps * d[v]) for v in range(3)), wd)
            _abi.check(hs._lib.dgswem_cuda_limit_state(hs._h))
            out.append(hs.state()[:3])
        lhs = sum(float(np.sum((out[0][v] - out[1][v]) / (2 * eps) * mu[v])) for v in range(3))
        rhs = sum(float(np.sum(d[v] * g[v])) for v in range(3))
        print(f"limiter dot product: FD {lhs:.10e} reverse {rhs:.10e} rel {abs(lhs - rhs) / abs(rhs):.2e}")
        assert abs(lhs - rhs) <= 1e-6 * abs(rhs)
        # the limiter changed the state: clamps and sweeps are exercised
        hs.set_state(*x, wd)
        _abi.check(hs._lib.dgswem_cuda_limit_state(hs._h))
        assert max(np.abs(a - b).max() for a, b in zip(hs.state()[:3], x)) > 1e-3


def test_limiter_adjoint_stepwise_matches_sweep(limiter_problem):
    deck, prob, n0, hb0 = limiter_problem
    misfit(prob, n0, hb0)
    gn, ghb = prob.gradient()
    gn2, ghb2 = prob.gradient_stepwise()
    np.testing.assert_array_equal(gn2, gn)
    np.testing.assert_array_equal(ghb2, ghb)


def test_limiter_is_active(limiter_problem, tmp_path_factory):
    """Without the limiter the same run gives other gauge values: the test
    above exercises the limiter's reverse mode."""
    deck, prob, n0, hb0 = limiter_problem
    prob.set_params(n0, hb0)
    eta_lim = prob.run().copy()
    path = decks.smooth_basin(tmp_path_factory.mktemp("adjnolim") / "basin", nsteps=200, dt=0.5, dramp=0.002)
    d2 = Deck(path)
    p2 = GaugeMisfitProblem(d2, prob.elem, prob.phi, 200)
    eta = p2.run()
    p2.close()
    d2.close()
    assert np.abs(eta - eta_lim).max() > 1e-9


def test_wetdry_reverse_mode_dot_product(built, scratch):
    """WETDRY after the limiter (the stage path's limit_wetdry) against
    central differences of the forward, as the limiter's dot-product test, at
    a seeded state whose vertex depths straddle H0 on a sloping beach (all-wet,
    flattened and partially wet elements; random input flags)."""
    from dgswem_b200 import _abi
    from dgswem_b200.adjoint import _dp
    path = decks.sloping_beach(scratch / "wdvjp", nx=16, ny=4, lx=800.0, ly=200.0, nsteps=2)
    deck = Deck(path)
    ne, npn = deck.s.ne, deck.s.np
    nm = deck.int_array("nm", 3 * ne).reshape(3, ne) - 1
    dp = deck.real_array("dp", npn)
    with HydroStep(deck) as hs:
        rng = np.random.default_rng(31)
        dpe = (dp[nm[0]] + dp[nm[1]] + dp[nm[2]]) / 3.0
        ze = np.stack([-dpe + rng.uniform(-0.3, 0.6, ne), 0.1 * rng.standard_normal(ne),
                       0.1 * rng.standard_normal(ne)], 1)
        x = [np.ascontiguousarray(ze), np.ascontiguousarray(0.2 * rng.standard_normal((ne, 3))),
             np.ascontiguousarray(0.2 * rng.standard_normal((ne, 3)))]
        wd = rng.integers(0, 2, ne).astype(np.int32)
        mu = [np.ascontiguousarray(rng.standard_normal((ne, 3))) for _ in range(3)]
        d = [rng.standard_normal((ne, 3)) for _ in range(3)]
        g = [np.empty((ne, 3)) for _ in range(3)]
        hs.set_state(*x, wd)
        _abi.check(hs._lib.dgswem_cuda_limiter_vjp(hs._h, *[_dp(m) for m in mu], *[_dp(a) for a in g]))
        eps = 1e-6  # the ZE modes are ~20 m (-DP): a smaller step drowns in rounding
        out = []
        for sgn in (1.0, -1.0):
            hs.set_state(*(np.ascontiguousarray(x[v] + sgn * eps * d[v]) for v in range(3)), wd)
            _abi.check(hs._lib.dgswem_cuda_limit_state(hs._h))
            out.append(hs.state())
        assert np.array_equal(out[0][3], out[1][3])  # no flag flipped inside the step
        lhs = sum(float(np.sum((out[0][v] - out[1][v]) / (2 * eps) * mu[v])) for v in range(3))
        rhs = sum(float(np.sum(d[v] * g[v])) for v in range(3))
        print(f"wetdry dot product: FD {lhs:.10e} reverse {rhs:.10e} rel {abs(lhs - rhs) / abs(rhs):.2e}")
        assert abs(lhs - rhs) <= 1e-6 * abs(rhs)
        # WETDRY acted: some elements were flattened or wetted / dried
        hs.set_state(*x, wd)
        _abi.check(hs._lib.dgswem_cuda_limit_state(hs._h))
        y = hs.state()
        assert not np.array_equal(y[3], wd) and np.abs(y[1] - x[1]).max() > 1e-3
    deck.close()


@pytest.fixture(scope="module")
def wetdry_problem(tmp_path_factory):
    """The sloping beach (config 2 physics: WETDRY, limiter 5, nodal Manning n)
    at a state with moving fronts: a 1 m tide ramped over 0.002 days, 600
    steps from cold start (the wave reaches and runs up the shore), then a
    3-step misfit at gauges around the shoreline, observations from Manning
    n x 1.5."""
    from dgswem_b200 import _abi
    from dgswem_b200 import build
    build.build_library()
    path = decks.sloping_beach(tmp_path_factory.mktemp("adjwd") / "beach", nx=60, ny=12, lx=3000.0, ly=600.0,
                               nsteps=700, dt=0.5, dramp=0.002)
    deck = Deck(path)
    rng = np.random.default_rng(9)
    elem, phi = locate_gauges(deck, np.column_stack([rng.uniform(2300.0, 2800.0, 16), rng.uniform(50.0, 550.0, 16)]))
    n0 = element_manning(deck)
    hb0 = deck.real_array("hb", 3 * deck.s.ne).reshape(deck.s.ne, 3)

    def warmed(nbar):
        p = GaugeMisfitProblem(deck, elem, phi, 3, it0=601)
        p.set_params(nbar=nbar)
        p.hs.run(1, 600)
        _abi.check(p.hs._lib.dgswem_cuda_state_save(p.hs._h, 0))
        return p
    t = warmed(1.5 * n0)
    obs = t.run()
    t.close()
    prob = warmed(n0)
    prob.obs = obs
    yield deck, prob, n0, hb0
    prob.close()
    deck.close()


def test_wetdry_adjoint_matches_short_central_difference(wetdry_problem):
    """Gradient of the 3-step misfit through the whole wet/dry chain (dry
    elements' volume terms masked, dry-side edge rules, limiter, WETDRY, all
    frozen at the forward's branches) against a central difference of step
    1e-7 in a random Manning direction, small enough that no branch of the 3
    steps changes."""
    deck, prob, n0, hb0 = wetdry_problem
    prob.set_params(n0, hb0)
    prob.forward()
    gn, ghb = prob.gradient()
    dn = n0 * np.random.default_rng(3).standard_normal(deck.s.ne)
    eps = 1e-7
    fd = (misfit(prob, n0 + eps * dn, hb0) - misfit(prob, n0 - eps * dn, hb0)) / (2 * eps)
    ad = float(gn @ dn)
    print(f"wetdry 3 steps: adjoint {ad:.10e} central FD {fd:.10e} J {misfit(prob, n0, hb0):.3e}")
    assert fd != 0.0
    assert abs(ad - fd) <= 1e-5 * abs(fd)
    prob.set_params(n0, hb0)


def test_wetdry_adjoint_stepwise_matches_sweep(wetdry_problem):
    deck, prob, n0, hb0 = wetdry_problem
    prob.set_params(n0, hb0)
    prob.forward()
    gn, ghb = prob.gradient()
    gn2, ghb2 = prob.gradient_stepwise()
    np.testing.assert_array_equal(gn2, gn)
    np.testing.assert_array_equal(ghb2, ghb)
