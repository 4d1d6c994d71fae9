"""CUDA hydro step vs the FP64 oracle (GPU).

Two kernel variants are checked:
* strict (the drop-in default: -fmad=false, the oracle's evaluation order,
  the Manning factor DEPTH**(1.D0/3.D0) correctly rounded on both sides):
  bit-for-bit equal to the oracle on every deck except those with hybrid
  friction, whose general pow() may differ in the last bit between the device
  and the host C library; those are held to the FP64 bar below with
  identical wet/dry flags.
* fast (opt-in, FMA contraction): modal coefficients after N steps within
  1e-10 relative (max |gpu - oracle| / max |oracle| per variable) wherever the
  slope limiter and WETDRY do not meet their branch ties (see
  test_fast_limiter_ties); integer wet/dry flags exactly.
"""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def rel_err(a, b, floor=1e-300):
    scale = max(np.abs(b).max(), floor)
    return np.abs(a - b).max() / scale


def scale_floors(deck):
    """Field scales below which a coefficient is rounding noise: 1e-6 of the
    deepest still-water depth for ZE and of sqrt(g H) H for QX/QY (a basin
    at rest has QX = QY = 0 exactly in the oracle and ~1e-20 with FMA)."""
    hmax = float(np.abs(deck.real_array("dp", deck.s.np)).max())
    q = (deck.s.g * hmax) ** 0.5 * hmax
    return (1e-6 * hmax, 1e-6 * q, 1e-6 * q)


def run_both(path, nsteps, it0=1, met=None, strict=False):
    """strict=False: the fast (FMA) build; True: the strict build."""
    deck = Deck(path)
    orc = Oracle(path, threads=4)
    hs = HydroStep(deck, strict=bool(strict))
    if met is not None:
        hs.set_met(*met)
        orc.set_met(*met)
    for it in range(it0, it0 + nsteps):
        hs.timestep(it)
        orc.step(it)
    hs.synchronize()
    g = hs.state()
    o = orc.state()
    hs.close()
    return deck, orc, g, o


def check_state(g, o, rtol=RTOL, floors=(1e-300,) * 3):
    for a, b, name, fl in zip(g[:3], o[:3], ("ZE", "QX", "QY"), floors):
        err = rel_err(a, b, fl)
        assert err <= rtol, f"{name} relative error {err:.3e} > {rtol:.0e}"
    np.testing.assert_array_equal(g[3], o[3], err_msg="WDFLG differs")


def check_bitwise(g, o):
    for a, b, name in zip(g, o, ("ZE", "QX", "QY", "WDFLG")):
        np.testing.assert_array_equal(a, b, err_msg=f"{name} not bit-identical")


STRICT_DECKS = {
    # decks without pow(): quadratic/linear friction, limiter, SSP(5,2)
    "qa_linear_ramp": dict(nr=8, nth=16, nsteps=60, nolibf=0, slopeflag=0),
    "qa_quad_limiter_ramp": dict(nr=8, nth=16, nsteps=60, nolibf=1, cf=0.0025, slopeflag=5),
    "qa_ssp52_limiter": dict(nr=12, nth=24, nsteps=60, nolibf=1, cf=0.0025, slopeflag=5, rk_stage=5),
    "qa_euler": dict(nr=8, nth=16, nsteps=60, nolibf=0, slopeflag=5, rk_stage=1, rk_order=1, dt=2.0),
    "qa_ssp33": dict(nr=8, nth=16, nsteps=60, nolibf=0, slopeflag=5, rk_stage=3, rk_order=3),
}


@pytest.mark.parametrize("name", sorted(STRICT_DECKS))
def test_strict_bitwise_synthetic(built, scratch, name):
    kw = dict(STRICT_DECKS[name])
    n = kw.pop("nsteps")
    path = decks.quarter_annulus(scratch / f"strict_{name}", nsteps=n, **kw)
    _, _, g, o = run_both(path, n, strict=True)
    check_bitwise(g, o)


@pytest.mark.parametrize("case,nsteps", [("quarter_annular", 500), ("mass_conservation", 500)])
def test_strict_bitwise_golden_decks(built, case, nsteps):
    """Reference golden decks without pow(): ocean+land edges, SSP(5,2),
    limiter (quarter_annular); ICS=2 spherical factors and rain in a closed
    basin (mass_conservation)."""
    from conftest import golden_dir
    _, _, g, o = run_both(golden_dir(case), nsteps, strict=True)
    check_bitwise(g, o)


def test_strict_wetdry_barriers_pow(built):
    """wetdry golden deck (hybrid friction -> pow, barriers, wet/dry) in
    strict mode: FP64 bar and identical wet/dry flags."""
    from conftest import golden_dir
    _, _, g, o = run_both(golden_dir("wetdry"), 300, strict=True)
    check_state(g, o)


@pytest.mark.parametrize("nramp,rk", [(1, 2), (0, 5)])
def test_fast_limiter_ties(built, scratch, nramp, rk):
    """Fast (FMA) variant with the slope limiter: the limiter's
    redistribution branches (slopelimiter.F:3592-3620) are discontinuous at
    ties (a vertex value equal to the element mean), so FMA rounding can move
    a vertex across a tie where the strict variant reproduces the oracle bit
    for bit (test_strict_bitwise_synthetic).  The difference stays well below
    the field scale and the wet/dry flags agree."""
    path = decks.quarter_annulus(scratch / f"fast_ties_{nramp}_{rk}", nr=12, nth=24, nsteps=200, nolibf=1,
                                 cf=0.0025, slopeflag=5, nramp=nramp, rk_stage=rk)
    deck, _, g, o = run_both(path, 200)
    errs = [rel_err(a, b) for a, b in zip(g[:3], o[:3])]
    print("fast limiter ties: relative differences", errs)
    assert max(errs) <= 1e-3, errs
    np.testing.assert_array_equal(g[3], o[3])


@pytest.mark.parametrize("strict", [True, False])
def test_flow_and_radiation_boundaries(built, scratch, strict):
    """Periodic flux boundary (flow_edge_hydro.F: prescribed normal flux from
    QNAM/QNPH) on one side and a radiation boundary (radiation_edge_hydro.F)
    on another, with ocean forcing and land: strict bit for bit, fast at the
    FP64 bar."""
    path = decks.quarter_annulus(scratch / f"qa_flowrad_{strict}", nr=8, nth=16, nsteps=120, flow_amp=0.05,
                                 radiation=True, nolibf=1, cf=0.0025)
    deck = Deck(path)
    assert deck.s.nfeds > 0 and deck.s.nreds > 0
    deck.close()
    _, _, g, o = run_both(path, 120, strict=strict)
    if strict:
        check_bitwise(g, o)
    else:
        check_state(g, o)


def test_quarter_annulus_config1_linear_friction(built, scratch):
    """Config 1 geometry (1024 elements, SSP(2,2), linear friction), 300
    steps, fast variant."""
    path = decks.quarter_annulus(scratch / "qa1024", nsteps=300)
    _, _, g, o = run_both(path, 300)
    check_state(g, o)


def test_quarter_annulus_ssp52_no_limiter(built, scratch):
    """Quadratic friction, SSP(5,2) (stored stage RHS), fast variant."""
    path = decks.quarter_annulus(scratch / "qa_ssp52", nr=12, nth=24, nsteps=200, nolibf=1, cf=0.0025,
                                 rk_stage=5, rk_order=2, slopeflag=0, nramp=0)
    _, _, g, o = run_both(path, 200)
    check_state(g, o)


# Fast variant on wet/dry decks: the wet/dry thresholds (H0 on vertex
# depths, wetdry.F) make the step discontinuous, so FMA rounding near a front
# is amplified over hundreds of steps beyond the 1e-10 bar that the strict
# variant holds; the wet/dry flags must still agree exactly.
RTOL_FAST_WETDRY = 1e-8


@pytest.mark.parametrize("strict", [True, False])
def test_sloping_beach_wetdry_manning(built, scratch, strict):
    """Config 2 physics on a small mesh: wet/dry, limiter, nodal Manning n.
    Strict: bit for bit (the Manning factor is correctly rounded on both
    sides)."""
    path = decks.sloping_beach(scratch / "sb_par", nx=60, ny=12, lx=3000.0, ly=600.0, nsteps=400, dt=0.5)
    _, _, g, o = run_both(path, 400, strict=strict)
    print("sloping beach: relative differences", [rel_err(a, b) for a, b in zip(g[:3], o[:3])])
    if strict:
        check_bitwise(g, o)
    else:
        check_state(g, o, rtol=RTOL_FAST_WETDRY)
    assert 0 < g[3].sum() < len(g[3])  # both wet and dry elements present


def test_strict_sloping_beach_200k_bitwise(built, scratch):
    """The bench configuration's physics (wet/dry, limiter 5, nodal Manning
    n, M2 tide) on a 200k-element beach of the same 100 x 20 km basin,
    50 steps: the strict build bit for bit (the Morton tile plan's halos and
    task lists at a size where tiles carry the full task and halo caps)."""
    path = decks.sloping_beach(scratch / "sb_200k", nx=707, ny=141, nsteps=50, dt=0.5)
    _, _, g, o = run_both(path, 50, strict=True)
    assert 0 < g[3].sum() < len(g[3])
    check_bitwise(g, o)


def test_quarter_annulus_config1_full_length_bitwise(built, scratch):
    """Config 1 in full: the 1024-element tidal quarter annulus, SSP(2,2),
    linear friction, dt = 10 s, all 4460 steps; the strict build bit for bit
    against the oracle."""
    path = decks.quarter_annulus(scratch / "qa1024_full", nsteps=4460)
    _, _, g, o = run_both(path, 4460, strict=True)
    check_bitwise(g, o)


def test_wind_nws1(built, scratch):
    """NWS=1 uniform wind stress (config 3 forcing) and pressure field."""
    path = decks.quarter_annulus(scratch / "qa_wind", nr=8, nth=16, nsteps=100, nws=1)
    d = Deck(path)
    npn = d.s.np
    x = d.real_array("x", npn)
    d.close()
    tau = 0.1 / 1000.0
    met = (np.full(npn, tau * np.cos(np.pi / 6)), np.full(npn, tau * np.sin(np.pi / 6)), 1e-4 * x / x.max())
    _, _, g, o = run_both(path, 100, met=met)
    check_state(g, o)


@pytest.mark.parametrize("case,nsteps", [("quarter_annular", 400), ("wetdry", 200), ("mass_conservation", 400)])
def test_golden_decks_state(built, case, nsteps):
    """The reference's own golden decks (ocean/land/barrier edges, hybrid
    friction, ICS=2, rain) stepped on both sides, fast variant."""
    from conftest import golden_dir
    deck, _, g, o = run_both(golden_dir(case), nsteps)
    check_state(g, o, floors=scale_floors(deck))


def test_modal2nodal_and_nodecode(built):
    from conftest import golden_dir
    path = golden_dir("wetdry")
    deck = Deck(path)
    orc = Oracle(path, threads=4)
    with HydroStep(deck) as hs:
        for it in range(1, 101):
            hs.timestep(it)
            orc.step(it)
        eta, uu, vv, nc = hs.modal2nodal()
    e2, u2, v2 = orc.modal2nodal()
    np.testing.assert_array_equal(nc, orc.nodecode())
    assert rel_err(eta, e2) <= RTOL
    assert rel_err(uu, u2) <= 1e-9 and rel_err(vv, v2) <= 1e-9


def test_run_matches_timestep_and_is_deterministic(built, scratch):
    path = decks.sloping_beach(scratch / "sb_det", nx=30, ny=6, lx=1500.0, ly=300.0, nsteps=50)
    outs = []
    for mode in ("timestep", "run", "run"):
        with HydroStep(Deck(path)) as hs:
            if mode == "timestep":
                for it in range(1, 51):
                    hs.timestep(it)
            else:
                hs.run(1, 50)
            outs.append(hs.state())
    for other in outs[1:]:
        for a, b in zip(outs[0], other):
            np.testing.assert_array_equal(a, b)  # bitwise: no atomics, fixed order


def test_numeric_error_reported_not_fatal(built, scratch):
    """A NaN planted in the host initial state comes back as a status code."""
    from dgswem_b200._abi import DgswemError
    path = decks.quarter_annulus(scratch / "qa_nan", nr=4, nth=8, nsteps=2)
    with HydroStep(Deck(path)) as hs:
        ze, qx, qy, wd = hs.state()
        ze[3, 0] = np.nan
        hs.set_state(ze, qx, qy, wd)
        hs.timestep(1)
        with pytest.raises(DgswemError, match="NaN"):
            hs.synchronize()
        hs.state()  # the context stays usable


def test_upload_download_roundtrip(built, scratch):
    path = decks.quarter_annulus(scratch / "qa_rt", nr=4, nth=8, nsteps=2)
    rng = np.random.default_rng(7)
    with HydroStep(Deck(path)) as hs:
        ze = rng.normal(size=(hs.ne, 3))
        qx = rng.normal(size=(hs.ne, 3))
        qy = rng.normal(size=(hs.ne, 3))
        wd = rng.integers(0, 2, hs.ne).astype(np.int32)
        hs.set_state(ze, qx, qy, wd)
        z2, x2, y2, w2 = hs.state()
    np.testing.assert_array_equal(z2, ze)
    np.testing.assert_array_equal(x2, qx)
    np.testing.assert_array_equal(y2, qy)
    np.testing.assert_array_equal(w2, wd)


@pytest.mark.parametrize("rk", [(1, 1), (3, 3), (5, 2)])
def test_strict_wetdry_other_rk_schemes(built, scratch, rk):
    """Wet/dry, limiter 5 and nodal Manning n with the other SSP-RK schemes
    of RK_TIME (forward Euler at a quarter of the step, SSP(3,3), the
    tabulated SSP(5,2)): every stage's limiter and WETDRY pass and the
    combinations over the stage history, bit for bit against the oracle."""
    stages, order = rk
    dt = 0.125 if stages == 1 else 0.5
    path = decks.sloping_beach(scratch / f"sb_rk{stages}{order}", nx=40, ny=8, lx=2000.0, ly=400.0, nsteps=120,
                               dt=dt, rk_stage=stages, rk_order=order)
    _, _, g, o = run_both(path, 120, strict=True)
    assert 0 < g[3].sum() < len(g[3])
    check_bitwise(g, o)
