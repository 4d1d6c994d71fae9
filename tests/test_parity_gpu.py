"""CUDA hydro step vs the FP64 oracle (GPU).

Tolerance: modal coefficients after N steps agree to 1e-10 relative
(max |gpu - oracle| / max |oracle| per variable), the FP64 bar of the drop-in;
the CUDA kernels may contract a*b+c into FMA, the oracle never does, so the
two differ by rounding only.  Integer wet/dry flags must match exactly.
"""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

RTOL = 1e-10


def rel_err(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return np.abs(a - b).max() / scale


def run_both(path, nsteps, it0=1, met=None):
    deck = Deck(path)
    orc = Oracle(path, threads=4)
    hs = HydroStep(deck)
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


def check_state(g, o, rtol=RTOL):
    for a, b, name in zip(g[:3], o[:3], ("ZE", "QX", "QY")):
        err = rel_err(a, b)
        assert err <= rtol, f"{name} relative error {err:.3e} > {rtol:.0e}"
    np.testing.assert_array_equal(g[3], o[3], err_msg="WDFLG differs")


def test_quarter_annulus_config1_linear_friction(built, scratch):
    """Config 1 geometry (1024 elements, SSP(2,2), linear friction), 300 steps."""
    path = decks.quarter_annulus(scratch / "qa1024", nsteps=300)
    _, _, g, o = run_both(path, 300)
    check_state(g, o)


def test_quarter_annulus_limiter_ssp52(built, scratch):
    """Quadratic friction, SSP(5,2) (stored stage RHS), slope limiter 5."""
    path = decks.quarter_annulus(scratch / "qa_lim", nr=12, nth=24, nsteps=200, nolibf=1, cf=0.0025,
                                 rk_stage=5, rk_order=2, slopeflag=5)
    _, _, g, o = run_both(path, 200)
    check_state(g, o)


def test_sloping_beach_wetdry_manning(built, scratch):
    """Config 2 physics on a small mesh: wet/dry, limiter, nodal Manning n."""
    path = decks.sloping_beach(scratch / "sb_par", nx=60, ny=12, lx=3000.0, ly=600.0, nsteps=400, dt=0.5)
    _, _, g, o = run_both(path, 400)
    check_state(g, o)
    assert 0 < g[3].sum() < len(g[3])  # both wet and dry elements present


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
    friction, ICS=2, rain) stepped on both sides."""
    from conftest import golden_dir
    _, _, g, o = run_both(golden_dir(case), nsteps)
    check_state(g, o)


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
