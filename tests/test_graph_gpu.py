"""CUDA-graph replay of whole steps (dgswem_cuda_set_graph, GPU): the same
kernels and data as the launch-by-launch path, so the state after any mix of
graph chunks, remainders and single steps is bit-identical to it; the ramp
and forcing that change per stage come from device memory in the replays."""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks

pytestmark = pytest.mark.gpu


def run(path, graph, plan, met=None, mixed=False):
    with HydroStep(Deck(path), mixed=mixed) as hs:
        if met is not None:
            hs.set_met(*met)
        if graph:
            hs.set_graph(graph)
        it = 1
        for n in plan:
            if n == 1:
                hs.timestep(it)
            else:
                hs.run(it, n)
            it += n
        hs.synchronize()
        return hs.state(), hs.kernel_launches


def wind(path):
    d = Deck(path)
    npn = d.s.np
    d.close()
    t = 0.1 / 1000.0
    return np.full(npn, t * np.cos(0.5)), np.full(npn, t * np.sin(0.5)), np.full(npn, 1e-3)


# (name, deck, plan of run() lengths; 1 = a single timestep)
PLANS = [(8, [40]), (8, [37, 1, 13]), (4, [3, 17, 1, 9, 20])]


@pytest.mark.parametrize("graph,plan", PLANS)
def test_graph_matches_launches_wetdry_barriers(built, graph, plan):
    """wetdry golden deck: barriers (ramped weirs), hybrid friction, wet/dry,
    ocean forcing, SSP(5,2)."""
    from conftest import golden_dir
    a, la = run(golden_dir("wetdry"), 0, plan)
    b, lb = run(golden_dir("wetdry"), graph, plan)
    for x, y, name in zip(a, b, ("ZE", "QX", "QY", "WDFLG")):
        np.testing.assert_array_equal(x, y, err_msg=name)
    assert la == lb  # graph replays count their kernels


@pytest.mark.parametrize("mixed", [False, True])
def test_graph_matches_launches_wind_limiter(built, scratch, mixed):
    path = decks.quarter_annulus(scratch / "gr_wind", nr=8, nth=16, nsteps=60, nws=1, nolibf=1, cf=0.0025,
                                 slopeflag=5)
    met = wind(path)
    a, _ = run(path, 0, [25, 1, 34], met, mixed)
    b, _ = run(path, 6, [25, 1, 34], met, mixed)
    for x, y, name in zip(a, b, ("ZE", "QX", "QY", "WDFLG")):
        np.testing.assert_array_equal(x, y, err_msg=name)


def test_set_graph_rejects_odd_steps(built, scratch):
    from dgswem_b200._abi import DgswemError
    path = decks.quarter_annulus(scratch / "gr_odd", nr=4, nth=8, nsteps=2)
    with HydroStep(Deck(path)) as hs:
        with pytest.raises(DgswemError, match="even"):
            hs.set_graph(3)
