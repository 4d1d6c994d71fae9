"""The p=2 device path (GPU) against the oracle's p=2, which is checked by
its convergence order (test_oracle_p2_convergence.py): the strict variant
bit for bit, the fast one within 1e-10 relative, the mixed-precision one
within the mixed form's bars (1e-5 m elevation, 1e-9 relative volume); its
own convergence order; and the p=1-only features rejected on a p=2
handle."""
import math
import os

import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks
from dgswem_b200 import _abi
from dgswem_b200._abi import DgswemError
from oracle_lib import Oracle

import test_oracle_p2_convergence as sw

pytestmark = pytest.mark.gpu

P2 = {"extra": {"pl": 2, "ph": 2}}


def standing_wave_state(path, nx):
    """The basin deck and the L2 projection of the standing wave (oracle tables)."""
    x, y, elems = sw.basin(path, nx, 2)
    orc = Oracle(path)
    px, py, wphys, phi, wa = sw.area_points(orc, x, y, elems)
    minv = orc.real_table("M_INV")
    ze = (sw.A * np.cos(sw.K * px) * wa[None, :]) @ phi.T * minv[None, :]
    return orc, ze, np.zeros_like(ze), (px, wphys, phi)


def run_pair(path, nsteps, strict, state=None, met=None, mixed=False):
    orc = Oracle(path)
    with HydroStep(Deck(path), strict=None if mixed else strict, mixed=mixed) as hs:
        assert hs.dofh == 6
        # the p=2 tile kernel runs (its tiles fit shared memory) unless the pair is forced
        forced_pair = os.environ.get("DGSWEM_CUDA_P2_PAIR", "0") not in ("", "0")
        assert (hs.get_shapes()[0] < 0) == forced_pair
        if state is not None:
            wd = np.ones(hs.ne, np.int32)
            hs.set_state(state[0], state[1], state[1], wd)
            orc.set_state(state[0], state[1], state[1], wd)
        if met is not None:
            hs.set_met(*met)
            orc.set_met(*met)
        hs.run(1, nsteps)
        orc.run(1, nsteps)
        hs.synchronize()
        g, o = hs.state(), orc.state()
        gn, on = hs.modal2nodal(), orc.modal2nodal()
    orc.close()
    return g, o, gn, on


def decks_p2(scratch):
    basin = scratch / "p2_basin"
    orc, ze, zero, _ = standing_wave_state(basin, 16)
    orc.close()
    qa = decks.quarter_annulus(scratch / "p2_qa", nr=8, nth=16, nsteps=60, nolibf=1, cf=0.0025, **P2)
    qa_lin = decks.quarter_annulus(scratch / "p2_qa_lin", nr=8, nth=16, nsteps=60, nolifa=0, nolica=0, nolicat=0,
                                   nolibf=2, nws=1, **P2)
    return [("standing wave, linear, SSP(3,3)", basin, 150, (ze, zero), None),
            ("quarter annulus, tide, quadratic friction", qa, 60, None, None),
            ("quarter annulus, linear, hybrid friction, wind", qa_lin, 60, None, "wind")]


def wind(path):
    d = Deck(path)
    npn = d.s.np
    d.close()
    t = 0.1 / 1000.0
    return np.full(npn, t * math.cos(0.5)), np.full(npn, t * math.sin(0.5)), np.zeros(npn)


def test_p2_strict_bitwise_vs_oracle(built, scratch):
    for name, path, n, state, met in decks_p2(scratch):
        g, o, gn, on = run_pair(path, n, True, state, wind(path) if met else None)
        assert np.abs(g[0]).max() > 0, name
        for a, b, v in zip(g, o, ("ZE", "QX", "QY", "WDFLG")):
            np.testing.assert_array_equal(a, b, err_msg=f"{name}: {v}")
        for a, b, v in zip(gn, on, ("ETA2", "UU2", "VV2")):
            np.testing.assert_array_equal(a, b, err_msg=f"{name}: {v}")


def test_p2_fast_vs_oracle(built, scratch):
    for name, path, n, state, met in decks_p2(scratch):
        g, o, _, _ = run_pair(path, n, False, state, wind(path) if met else None)
        for a, b, v in zip(g[:3], o[:3], ("ZE", "QX", "QY")):
            scale = max(np.abs(b).max(), 1e-300)
            assert np.abs(a - b).max() / scale <= 1e-10, f"{name}: {v}"


def test_p2_mixed_vs_oracle(built, scratch):
    """Mixed precision at p=2 (FP32 traces, fluxes, volume terms and sums;
    FP64 state and SSP): nodal elevation within 1e-5 m of the FP64 oracle,
    element means within 1e-5 m, water volume within 1e-9 relative (the
    p=1 mixed form's bar: the FP32 right-hand side of the element means
    rounds the flux balance)."""
    for name, path, n, state, met in decks_p2(scratch):
        g, o, gn, on = run_pair(path, n, False, state, wind(path) if met else None, mixed=True)
        d = Deck(path)
        ne = d.s.ne
        nm = d.int_array("nm", 3 * ne).reshape(3, ne) - 1
        x, y = d.real_array("x", d.s.np), d.real_array("y", d.s.np)
        hb = d.real_array("hb", 6 * ne).reshape(ne, 6)
        a, b, c = nm
        area = 0.5 * ((x[a] - x[c]) * (y[b] - y[c]) + (x[c] - x[b]) * (y[a] - y[c]))
        d.close()
        eta = np.abs(gn[0] - on[0]).max()
        mean = np.abs(g[0][:, 0] - o[0][:, 0]).max()
        vg, vo = np.sum((g[0][:, 0] + hb[:, 0]) * area), np.sum((o[0][:, 0] + hb[:, 0]) * area)
        print(f"p=2 mixed, {name}: nodal eta {eta:.2e} m, mean {mean:.2e} m, volume {(vg - vo) / vo:.2e}")
        assert eta <= 1e-5 and mean <= 1e-5, name
        assert abs(vg - vo) <= 1e-9 * abs(vo), name


def test_p2_convergence_order_on_device(built, scratch):
    errs = []
    for nx in (8, 16, 32):
        path = scratch / f"p2_conv_{nx}"
        orc, ze, zero, (px, wphys, phi) = standing_wave_state(path, nx)
        orc.close()
        with HydroStep(Deck(path)) as hs:
            hs.set_state(ze, zero, zero, np.ones(hs.ne, np.int32))
            hs.run(1, sw.NSTEPS)
            z = hs.state()[0]
        eta = sw.A * np.cos(sw.K * px) * math.cos(sw.OMEGA * sw.DT * sw.NSTEPS)
        errs.append(math.sqrt(float(np.sum(wphys * (z @ phi - eta) ** 2))))
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    assert all(r > 2.6 for r in rates), (errs, rates)


def test_p2_rejects_p1_only_features(built, scratch):
    path = decks.quarter_annulus(scratch / "p2_rej", nr=4, nth=8, nsteps=2, **P2)
    with HydroStep(Deck(path)) as hs:
        for call in (lambda: hs.autotune(), lambda: hs.set_shapes(1, -1),
                     lambda: _abi.check(hs._lib.dgswem_cuda_state_save(hs._h, 0))):
            with pytest.raises(DgswemError, match="p=1 only"):
                call()
    lim = decks.quarter_annulus(scratch / "p2_lim", nr=4, nth=8, nsteps=2, slopeflag=5, **P2)
    with pytest.raises(DgswemError, match="p = 1 only"):
        Deck(lim)


def test_p2_ensemble_matches_members_alone(built, scratch):
    from dgswem_b200 import Ensemble
    paths = [decks.quarter_annulus(scratch / f"p2_ens_{i}", nr=4 + 2 * i, nth=8 + 4 * i, nsteps=40, nolibf=1,
                                   cf=0.0025, **P2) for i in range(3)]
    ds = [Deck(p) for p in paths]
    with Ensemble(ds, mixed=False) as ens:
        ens.run(1, 40)
        ens.synchronize()
        got = ens.states()
    for i, d in enumerate(ds):
        with HydroStep(d) as hs:
            hs.run(1, 40)
            want = hs.state()
        for a, b, v in zip(got[i], want, ("ZE", "QX", "QY", "WDFLG")):
            np.testing.assert_array_equal(a, b, err_msg=f"member {i} {v}")
        assert want[0].shape[1] == 6


def test_p2_graphs_match_launches(built, scratch):
    """Whole-step CUDA graphs at p=2 (the wind ramp read from device memory
    in the replays): bit-identical to launch-by-launch stepping."""
    path = decks.quarter_annulus(scratch / "p2_graph", nr=6, nth=12, nsteps=60, nolibf=1, cf=0.0025, nws=1,
                                 dramp=0.01, **P2)
    met = wind(path)
    out = []
    for graph in (0, 6):
        with HydroStep(Deck(path)) as hs:
            hs.set_met(*met)
            if graph:
                hs.set_graph(graph)
            hs.run(1, 25)
            hs.timestep(26)
            hs.run(27, 30)
            hs.synchronize()
            out.append(hs.state())
    for a, b, v in zip(out[0], out[1], ("ZE", "QX", "QY", "WDFLG")):
        np.testing.assert_array_equal(a, b, err_msg=v)


@pytest.mark.parametrize("variant", ["strict", "fast", "mixed"])
def test_p2_pair_matches_tile_kernel(built, scratch, monkeypatch, variant):
    """The edge + element kernel pair (DGSWEM_CUDA_P2_PAIR=1 at create, the
    fallback for tiles that do not fit shared memory) against the tile
    kernel on the same decks: the same bits in the strict build; within
    the variant's own bar in the fast (contractions placed by the compiler
    per kernel: 1e-10 of the field) and mixed (FP32 terms: 1e-5) builds."""
    kw = {"strict": {"strict": True}, "fast": {"fast": True}, "mixed": {"mixed": True}}[variant]
    for name, path, n, state, met in decks_p2(scratch):
        out = []
        for pair in ("0", "1"):
            monkeypatch.setenv("DGSWEM_CUDA_P2_PAIR", pair)
            with HydroStep(Deck(path), **kw) as hs:
                assert (hs.get_shapes()[0] < 0) == (pair == "1")
                if state is not None:
                    hs.set_state(state[0], state[1], state[1], np.ones(hs.ne, np.int32))
                if met is not None:
                    hs.set_met(*wind(path))
                hs.run(1, n)
                hs.synchronize()
                out.append(hs.state())
        qscale = max(np.abs(out[1][1]).max(), np.abs(out[1][2]).max(), 1e-300)  # momentum scale
        for a, b, v in zip(out[0][:3], out[1][:3], ("ZE", "QX", "QY")):
            if variant == "strict":
                np.testing.assert_array_equal(a, b, err_msg=f"{variant}, {name}: {v}")
            else:
                scale = max(np.abs(b).max(), 1e-300) if v == "ZE" else qscale
                bar = 1e-10 if variant == "fast" else 1e-5
                assert np.abs(a - b).max() <= bar * scale, f"{variant}, {name}: {v}"


def p2_rain_manning_deck(path):
    """A p=2 rectangular basin (20 x 6 km, 10 m to 4 m deep) with a tide on
    one short side, nodal Manning n (fort.13), rain (rainfall = 1) and
    SSP-RK(3,3): the tile kernel's rain, Manning and boundary-weight
    branches."""
    nx, ny = 20, 6
    xs, ys = np.linspace(0.0, 20e3, nx + 1), np.linspace(0.0, 6e3, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    dp = 10.0 - 6.0 * X / 20e3
    elems = decks._grid_triangles(nx, ny)
    nid = lambda i, j: i * (ny + 1) + j + 1  # noqa: E731
    ocean = [nid(0, j) for j in range(ny, -1, -1)]
    land = [nid(i, 0) for i in range(0, nx + 1)] + [nid(nx, j) for j in range(1, ny + 1)] + \
           [nid(i, ny) for i in range(nx - 1, -1, -1)]
    rng = np.random.default_rng(7)
    ctl = decks.Controls(title="p2 rain manning", nolibf=1, nolifa=1, cf=0.0025, dt=2.0, nsteps=100,
                         rk_stage=3, rk_order=3, slopeflag=0, h0=0.01, nramp=1, dramp=0.01, manning=True,
                         rainfall=1, extra={"pl": 2, "ph": 2})
    return decks.write_deck(path, X.ravel(), Y.ravel(), dp.ravel(), elems, [ocean], [(land, 0)], ctl,
                            emo=np.full(len(ocean), 0.5), efa=np.zeros(len(ocean)),
                            manning=0.025 * rng.uniform(0.8, 1.2, X.size))


@pytest.mark.parametrize("pair", ["0", "1"])
def test_p2_rain_manning_strict_bitwise(built, scratch, monkeypatch, pair):
    """Rain, nodal Manning n and SSP(3,3) at p=2: the strict tile kernel and
    the edge + element pair each bit-identical to the oracle."""
    monkeypatch.setenv("DGSWEM_CUDA_P2_PAIR", pair)
    path = p2_rain_manning_deck(scratch / "p2_rain_manning")
    g, o, gn, on = run_pair(path, 100, True)
    assert np.abs(g[0]).max() > 0
    for a, b, v in zip(g, o, ("ZE", "QX", "QY", "WDFLG")):
        np.testing.assert_array_equal(a, b, err_msg=v)
    for a, b, v in zip(gn, on, ("ETA2", "UU2", "VV2")):
        np.testing.assert_array_equal(a, b, err_msg=v)
