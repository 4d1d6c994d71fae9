"""Tile and block shapes, autotuner (GPU).

The stage kernel is compiled for several tile shapes (elements per tile,
threads per block) and limit_wetdry for several block sizes.  Every shape
gives the same state bit for bit: each edge point's flux is evaluated in the
reference's in/ex orientation whichever tile evaluates it, and each element's
sums keep the reference's order.  The autotuner times whole steps with each
shape from the handle's state, leaves that state as it was and keeps the
fastest shapes.
"""
import numpy as np
import pytest

from dgswem_b200 import Deck, Ensemble, HydroStep, decks
from dgswem_b200._abi import DgswemError
from dgswem_b200.ensemble import make_members

pytestmark = pytest.mark.gpu

NAMES = ("ZE", "QX", "QY", "WDFLG")


def _decks(scratch):
    from conftest import golden_dir
    return {
        # barriers (ramped weirs), hybrid friction, wet/dry, ocean forcing, SSP(5,2)
        "wetdry_golden": golden_dir("wetdry"),
        # flow and radiation boundaries, quadratic friction, slope limiter 5
        "qa_flow_radiation_limiter": decks.quarter_annulus(
            scratch / "sh_qa", nr=10, nth=20, nsteps=40, flow_amp=0.2, radiation=True, nolibf=1, cf=0.0025,
            slopeflag=5),
        # wet/dry beach, Manning n, slope limiter 5
        "beach_manning": decks.sloping_beach(scratch / "sh_beach", nx=60, ny=12, nsteps=40, slopeflag=5,
                                              dramp=0.002),
    }


def _run(path, variant, tile=-1, limiter=-1, nsteps=30, graph=0):
    kw = {"strict": variant == "strict", "mixed": variant == "mixed"}
    with HydroStep(Deck(path), **kw) as hs:
        hs.set_shapes(tile, limiter)
        if graph:
            hs.set_graph(graph)
        hs.run(1, nsteps)
        hs.synchronize()
        return hs.state(), hs.get_shapes()


@pytest.mark.parametrize("variant", ["fast", "strict", "mixed"])
def test_every_shape_bit_identical(built, scratch, variant):
    sh = HydroStep.shapes()
    assert sh["tile"][0] == (128, 384) and len(sh["tile"]) >= 2 and len(sh["limiter"]) >= 2
    for name, path in _decks(scratch).items():
        want, picked = _run(path, variant)
        assert picked == (0, 0)
        assert np.abs(want[1]).max() > 0, f"{name}: nothing moved"
        runs = [(t, -1) for t in range(1, len(sh["tile"]))] + [(-1, l) for l in range(1, len(sh["limiter"]))]
        for t, l in runs:
            got, picked = _run(path, variant, t, l)
            assert picked == (max(t, 0), max(l, 0))
            for a, b, n in zip(got, want, NAMES):
                np.testing.assert_array_equal(a, b, err_msg=f"{name}: tile shape {t}, limiter {l}: {n}")
    # the last tile and limiter shapes together, replayed as CUDA graphs
    path = _decks(scratch)["wetdry_golden"]
    want, _ = _run(path, variant)
    got, _ = _run(path, variant, len(sh["tile"]) - 1, len(sh["limiter"]) - 1, graph=6)
    for a, b, n in zip(got, want, NAMES):
        np.testing.assert_array_equal(a, b, err_msg=f"graphs, last shapes: {n}")


def test_autotune_keeps_state_and_picks_fastest(built, scratch):
    path = decks.sloping_beach(scratch / "tune_beach", nx=120, ny=24, nsteps=40, slopeflag=5, dramp=0.002)
    with HydroStep(Deck(path)) as ref:
        ref.run(1, 25)
        ref.synchronize()
        want = ref.state()
    with HydroStep(Deck(path)) as hs:
        hs.run(1, 5)
        hs.synchronize()
        before = hs.state()
        launches = hs.kernel_launches
        r = hs.autotune(it=6, steps=3, reps=2, cached=False)
        assert hs.kernel_launches > launches  # the timings ran on the device
        for a, b, n in zip(hs.state(), before, NAMES):
            np.testing.assert_array_equal(a, b, err_msg=f"state after autotune: {n}")
        timed = [m for m in r["ms_tile"] if m is not None]
        assert len(timed) == len(HydroStep.shapes()["tile"]) and all(m > 0 for m in timed)
        assert r["ms_tile"][r["tile"]] == min(timed)
        lim = [m for m in r["ms_limiter"] if m is not None]
        assert lim and r["ms_limiter"][r["limiter"]] == min(lim)
        assert hs.get_shapes() == (r["tile"], r["limiter"])
        hs.run(6, 20)
        hs.synchronize()
        for a, b, n in zip(hs.state(), want, NAMES):
            np.testing.assert_array_equal(a, b, err_msg=f"tuned run: {n}")
    # a second handle on the same mesh reuses the process's result
    with HydroStep(Deck(path)) as hs2:
        launches = hs2.kernel_launches
        r2 = hs2.autotune(it=1, steps=3, reps=2, cached=True)
        assert hs2.kernel_launches == launches  # nothing timed
        assert r2["ms_tile"] == r["ms_tile"] and (r2["tile"], r2["limiter"]) == (r["tile"], r["limiter"])
        assert hs2.get_shapes() == (r["tile"], r["limiter"])


def test_autotune_ensemble_matches_members(built, scratch):
    specs = decks.ensemble_specs(4, seed=9, ne_min=400, ne_max=3000)
    ds, met = make_members(scratch / "tune_ens", specs, nsteps=30)
    with Ensemble(ds) as ens:
        ens.set_met(*met)
        r = ens.autotune(it=1, steps=2, reps=1, cached=False)
        assert r["ms_tile"][r["tile"]] is not None
        ens.run(1, 30)
        ens.synchronize()
        got = ens.states()
    for i, d in enumerate(ds):
        with HydroStep(d, mixed=True) as hs:
            hs.set_met(met[0][i], met[1][i], met[2][i])
            hs.run(1, 30)
            want = hs.state()
        for a, b, n in zip(got[i], want, NAMES):
            np.testing.assert_array_equal(a, b, err_msg=f"member {i} {n}")


def test_set_shapes_rejects_bad_index(built, scratch):
    path = decks.quarter_annulus(scratch / "sh_bad", nr=4, nth=8, nsteps=2)
    with HydroStep(Deck(path)) as hs:
        with pytest.raises(DgswemError, match="out of range"):
            hs.set_shapes(len(HydroStep.shapes()["tile"]), -1)
        with pytest.raises(DgswemError, match="out of range"):
            hs.set_shapes(-1, 99)
        with pytest.raises(DgswemError, match=">= 1"):
            hs.autotune(it=1, steps=0)
        assert hs.get_shapes() == (0, 0)
