"""The discrete adjoint's gradient against a full FP64 reference gradient:
every component of dJ/dnbar (one per element) and dJ/dHB (three modes per
element) by central finite differences of the strict FP64 forward, on a
200-element smooth always-wet basin (no limiter, no WETDRY), 100 steps of
5 s with a short tidal ramp, 8 gauges, observations from a forward run with
Manning n 30 % larger.

The finite differences use steps of 1e-6 of each parameter's scale (Manning
n, and 1 m for the bathymetry modes): small enough that the LLF wave-speed
maximum keeps its side at every edge point within the step on this smooth
solution, large enough that rounding stays far below the bar.  Bar: every
component within 1e-4 of the largest component of its group, and 1e-4
relative for the components above 1 % of it."""
import numpy as np
import pytest

from dgswem_b200 import Deck, decks
from dgswem_b200.adjoint import GaugeMisfitProblem, element_manning, locate_gauges

pytestmark = pytest.mark.gpu

NSTEPS = 100
RTOL = 1e-4


def test_full_gradient_against_central_differences(built, scratch):
    path = decks.smooth_basin(scratch / "adj_full_200", nx=20, ny=5, lx=20e3, ly=4e3, dt=5.0, nsteps=NSTEPS,
                              dramp=0.002)
    deck = Deck(path)
    ne = deck.s.ne
    assert ne == 200
    rng = np.random.default_rng(17)
    xy = np.column_stack([rng.uniform(500.0, 9000.0, 8), rng.uniform(300.0, 3700.0, 8)])
    elem, phi = locate_gauges(deck, xy)
    n0 = element_manning(deck)
    hb0 = deck.real_array("hb", 3 * ne).reshape(ne, 3)
    truth = GaugeMisfitProblem(deck, elem, phi, NSTEPS)
    truth.set_params(nbar=1.3 * n0)
    obs = truth.run()
    truth.close()
    prob = GaugeMisfitProblem(deck, elem, phi, NSTEPS, obs=obs)

    def misfit(nb, hb):
        prob.set_params(nb, hb)
        return prob.forward()

    j0 = misfit(n0, hb0)
    gn, ghb = prob.gradient()
    assert j0 > 0
    fn = np.empty(ne)
    for e in range(ne):
        h = 1e-6 * n0[e]
        d = np.zeros(ne)
        d[e] = h
        fn[e] = (misfit(n0 + d, hb0) - misfit(n0 - d, hb0)) / (2 * h)
    fh = np.empty((ne, 3))
    for e in range(ne):
        for k in range(3):
            h = 1e-6
            d = np.zeros((ne, 3))
            d[e, k] = h
            fh[e, k] = (misfit(n0, hb0 + d) - misfit(n0, hb0 - d)) / (2 * h)
    prob.set_params(n0, hb0)
    prob.close()
    deck.close()
    for name, ad, fd in (("nbar", gn, fn), ("hb", ghb.ravel(), fh.ravel())):
        scale = np.abs(fd).max()
        err = np.abs(ad - fd)
        big = np.abs(fd) > 1e-2 * scale
        rel_big = (err[big] / np.abs(fd[big])).max()
        print(f"{name}: {len(fd)} components, max |adjoint - FD| / max |FD| = {err.max() / scale:.2e}, "
              f"max relative over the {big.sum()} components above 1 % = {rel_big:.2e}")
        assert err.max() <= RTOL * scale, name
        assert rel_big <= RTOL, name
