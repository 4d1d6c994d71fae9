"""Mixed-precision form (DGSWEM_CUDA_MIXED) against the FP64 oracle (GPU).

The stage kernel's edge traces, numerical fluxes, boundary ghost states,
volume terms and right-hand-side sums and the slope limiter's sweeps run in
FP32 (a variable whose vertex values lie within their node bounds keeps its
FP64 modes); the state, the SSP-RK combination (so the element-mean
elevation accumulates in FP64 across stages), the ocean depth-positivity fix
and WETDRY stay FP64.  Bars, the precision targets of the mixed form:
* elevation within 1e-5 m of the FP64 result, as nodal ETA2 on wet nodes and
  as element means (ZE mode 1);
* identical wet/dry flags and nodal wet/dry codes;
* total water volume within 1e-8 relative of the FP64 run's.
Exception: on a deck whose wet/dry fronts move (the wetdry golden deck), the
WETDRY thresholds (vertex depths against H0 + 1e-6 and H0 + 1e-10,
wetdry.F:121-398) turn the FP32 rounding of the right-hand side (~1e-7 m of
elevation) into discrete differences at front elements -- a vertex wetted
or an element re-flagged one step apart -- whose pulses propagate and decay.
The FP64 FMA form shows the same amplification at its own rounding level
(held to 1e-8 relative there instead of 1e-10).  That deck is held to
ELEV_TOL_FRONTS_M with the same flag and volume bars.
"""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

ELEV_TOL_M = 1e-5
ELEV_TOL_FRONTS_M = 5e-4
MASS_RTOL = 1e-8


def volume(deck, ze):
    s = deck.s
    ne = s.ne
    a, b, c = deck.int_array("nm", 3 * ne).reshape(3, ne) - 1
    x, y = deck.real_array("x", s.np), deck.real_array("y", s.np)
    areas = (x[a] - x[c]) * (y[b] - y[c]) + (x[c] - x[b]) * (y[a] - y[c])
    hb = deck.real_array("hb", 3 * ne).reshape(ne, 3)
    return float(np.sum((ze[:, 0] + hb[:, 0]) * areas * 0.5))


def run_mixed_vs_oracle(path, nsteps, met=None):
    deck = Deck(path)
    orc = Oracle(path, threads=4)
    with HydroStep(deck, mixed=True) as hs:
        if met is not None:
            hs.set_met(*met)
            orc.set_met(*met)
        for it in range(1, nsteps + 1):
            hs.timestep(it)
            orc.step(it)
        hs.synchronize()
        g, gn = hs.state(), hs.modal2nodal()
    o = orc.state()
    on = orc.modal2nodal() + (orc.nodecode(),)
    return deck, g, gn, o, on


def check_mixed(deck, g, gn, o, on, elev_tol=ELEV_TOL_M):
    np.testing.assert_array_equal(g[3], o[3], err_msg="WDFLG differs")
    np.testing.assert_array_equal(gn[3], on[3], err_msg="NODECODE differs")
    wet = on[3] == 1
    eta = np.abs(gn[0] - on[0])[wet].max()
    mean = np.abs(g[0][:, 0] - o[0][:, 0]).max()
    vg, vo = volume(deck, g[0]), volume(deck, o[0])
    print(f"mixed vs FP64: nodal eta {eta:.2e} m, element mean {mean:.2e} m, volume {(vg - vo) / vo:.2e}")
    assert eta <= elev_tol, f"nodal elevation error {eta:.3e} m"
    assert mean <= elev_tol, f"element-mean elevation error {mean:.3e} m"
    assert abs(vg - vo) <= MASS_RTOL * abs(vo)


def test_mixed_quarter_annulus_wind(built, scratch):
    """Config 1 geometry with the precision config's forcing: uniform wind
    stress 0.1 Pa at 30 degrees (NWS=1 kinematic stress), linear friction,
    dt 10 s, 1000 steps."""
    path = decks.quarter_annulus(scratch / "mx_wind", nsteps=1000, nws=1)
    d = Deck(path)
    npn = d.s.np
    d.close()
    tau = 0.1 / 1000.0
    met = (np.full(npn, tau * np.cos(np.pi / 6)), np.full(npn, tau * np.sin(np.pi / 6)), np.zeros(npn))
    check_mixed(*run_mixed_vs_oracle(path, 1000, met=met))


def test_mixed_limiter_quadratic_friction(built, scratch):
    path = decks.quarter_annulus(scratch / "mx_lim", nsteps=600, nolibf=1, cf=0.0025, slopeflag=5)
    check_mixed(*run_mixed_vs_oracle(path, 600))


def test_mixed_sloping_beach_wetdry(built, scratch):
    """Config 2 physics on a small mesh: wet/dry, limiter, nodal Manning n."""
    path = decks.sloping_beach(scratch / "mx_sb", nx=60, ny=12, lx=3000.0, ly=600.0, nsteps=400, dt=0.5)
    deck, g, gn, o, on = run_mixed_vs_oracle(path, 400)
    assert 0 < o[3].sum() < len(o[3])
    check_mixed(deck, g, gn, o, on)


@pytest.mark.parametrize("case,nsteps", [("quarter_annular", 500), ("mass_conservation", 400)])
def test_mixed_golden_decks(built, case, nsteps):
    """The reference's golden decks without moving fronts (SSP(5,2) +
    limiter; ICS=2 and rain in a closed basin)."""
    from conftest import golden_dir
    check_mixed(*run_mixed_vs_oracle(golden_dir(case), nsteps))


def test_mixed_golden_wetdry_fronts(built):
    """wetdry golden deck (moving wet/dry fronts with H0 = 7.5 m, barriers,
    hybrid friction, SSP(5,2)): identical flags and volume, elevation within
    the front bar (see the module docstring)."""
    from conftest import golden_dir
    check_mixed(*run_mixed_vs_oracle(golden_dir("wetdry"), 400), elev_tol=ELEV_TOL_FRONTS_M)


def test_mixed_and_strict_exclude_each_other(built, scratch):
    import ctypes as C
    from dgswem_b200 import _abi
    path = decks.quarter_annulus(scratch / "mx_flags", nr=4, nth=8, nsteps=2)
    with pytest.raises(ValueError):
        HydroStep(Deck(path), strict=True, mixed=True)
    deck = Deck(path)
    lib = _abi.load()
    h = C.c_void_p()
    rc = lib.dgswem_cuda_create(deck.setup, 0, HydroStep.STRICT | HydroStep.MIXED, C.byref(h))
    assert rc != 0 and not h.value
    deck.close()
