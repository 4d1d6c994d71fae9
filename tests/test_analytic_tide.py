"""The quarter-annulus tide against its analytic solution (Lynch and Gray,
1978: analytic solutions for testing tidal models), an independent check of
the oracle's physics and of the device path, beside their parity with the
reference's golden outputs.

Config 1's basin with the linearised equations (NOLIFA = NOLICA = NOLICAT =
0: NLEQ = 0, LEQ = 1) and linear friction tau: depth h = h0 (r/r0)^2 between
the land arc r = r0 and the ocean arc r = r1, land on the radial sides, the
M2 tide of amplitude A on the ocean arc.  The elevation is radial,
zeta = Re(Z(r) e^{i w t}); with q = h u the equations

    d zeta/dt + div q = 0,   dq/dt + tau q = -g h grad zeta

give (1/r) d/dr (r h dZ/dr) = beta Z, beta = (-w^2 + i w tau) / g.  With
h = h0 x^2, x = r/r0, this is the Euler equation x^2 Z'' + 3 x Z' = (beta
r0^2 / h0) Z, solved by x^s with s^2 + 2 s = beta r0^2 / h0, so
Z = C1 x^s1 + C2 x^s2 with Z'(1) = 0 (no normal flow at the land arc) and
Z(r1/r0) = A.  The model runs past its ramp until the transient has decayed
(five periods at tau = 1e-4 1/s), then the nodal elevation is sampled over a
sixth period and fitted with cos, sin and a constant: its complex amplitude
against Z at every node.  DG of degree 1 converges at second order; at
config 1's 16 x 32 cells the largest nodal error is 0.34 % of A (the
solution's own amplitude varies over 0.30 - 0.56 m and its phase over 36
degrees across the basin).
"""
import math
from pathlib import Path

import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks
from oracle_lib import Oracle

G, H0, AMP, TAU, OMEGA = 9.81, 3.048, 0.3048, 1e-4, decks.M2_OMEGA
R0, R1 = 60960.0, 152400.0
DT, PERIODS, NSAMP = 10.0, 5, 24
PERIOD_STEPS = 2.0 * math.pi / OMEGA / DT


def analytic(r):
    """Complex elevation amplitude Z(r) of the linear tide."""
    d = np.sqrt(1.0 + (-OMEGA ** 2 + 1j * OMEGA * TAU) * R0 ** 2 / (G * H0) + 0j)
    s1, s2 = -1.0 + d, -1.0 - d
    x1 = R1 / R0
    c1 = AMP / (x1 ** s1 - s1 / s2 * x1 ** s2)
    c2 = -c1 * s1 / s2
    x = np.asarray(r) / R0
    return c1 * x ** s1 + c2 * x ** s2


def linear_tide(path: Path, nr: int, nth: int):
    path = decks.quarter_annulus(path, nr=nr, nth=nth, amp=AMP, nolifa=0, nolica=0, nolicat=0, nolibf=0,
                                 tau=TAU, dt=DT, nsteps=10 ** 6, dramp=0.5)
    with Deck(path) as d:
        assert d.s.nleq == 0.0 and d.s.leq == 1.0
        r = np.hypot(d.real_array("x", d.s.np), d.real_array("y", d.s.np))
    return path, r


def fitted_amplitude(times, etas):
    """Least-squares fit eta = a cos(w t) + b sin(w t) + c per node: a - i b."""
    t = np.asarray(times)
    basis = np.stack([np.cos(OMEGA * t), np.sin(OMEGA * t), np.ones_like(t)], 1)
    coef, *_ = np.linalg.lstsq(basis, np.asarray(etas), rcond=None)
    return coef[0] - 1j * coef[1]


def sample(advance, nodal_eta):
    """Run past the ramp and the transient, then sample one period:
    advance(it0, n) steps n steps from it0, nodal_eta() reads ETA2."""
    n0 = int(round(PERIODS * PERIOD_STEPS))
    advance(1, n0)
    it, step = n0 + 1, int(round(PERIOD_STEPS / NSAMP))
    times, etas = [], []
    for _ in range(NSAMP):
        advance(it, step)
        it += step
        times.append((it - 1) * DT)  # model time at the end of step it - 1
        etas.append(nodal_eta().copy())
    return fitted_amplitude(times, etas)


def oracle_error(path, r):
    orc = Oracle(path, threads=4)
    try:
        z = sample(lambda it0, n: orc.run(it0, it0 + n - 1), lambda: orc.modal2nodal()[0])
    finally:
        orc.close()
    err = np.abs(z - analytic(r)) / AMP
    return float(err.max()), float(np.sqrt(np.mean(err ** 2)))


def test_analytic_solution_sanity():
    """Z meets its boundary conditions and the ODE, checked by central
    differences (truncation ~1e-6 relative at this step; a wrong root or
    constant gives O(1) residuals)."""
    assert abs(analytic(R1) - AMP) < 1e-14
    h = 1e-3 * R0
    dz = (analytic(R0 + h) - analytic(R0 - h)) / (2 * h)
    assert abs(dz) * R0 < 1e-4 * AMP
    r = np.linspace(1.2 * R0, 0.9 * R1, 7)
    beta = (-OMEGA ** 2 + 1j * OMEGA * TAU) / G
    flux = lambda rr: rr * H0 * (rr / R0) ** 2 * (analytic(rr + h) - analytic(rr - h)) / (2 * h)  # noqa: E731
    lhs = (flux(r + h) - flux(r - h)) / (2 * h) / r
    assert np.abs(lhs - beta * analytic(r)).max() < 1e-4 * np.abs(beta * analytic(r)).max()


def test_oracle_matches_analytic_tide(built, tmp_path):
    """The oracle at config 1's 16 x 32 cells and at half that resolution:
    the largest nodal error below 0.5 % of the amplitude at 16 x 32, the RMS
    error falling at second order (measured 0.48 % -> 0.12 %)."""
    errs = []
    for nr, nth in ((8, 16), (16, 32)):
        path, r = linear_tide(tmp_path / f"tide_{nr}", nr, nth)
        errs.append(oracle_error(path, r))
    print(f"analytic tide: max/rms error of A {errs}")
    assert errs[1][0] < 5e-3
    assert math.log2(errs[0][1] / errs[1][1]) > 1.7


@pytest.mark.gpu
def test_device_matches_analytic_tide(built, tmp_path):
    """The strict device build on config 1's mesh: the same bound, and the
    oracle's fitted amplitudes within 1e-10 of A (the strict state is
    bit-identical to the oracle's; nodal output is held to 1e-10 relative)."""
    path, r = linear_tide(tmp_path / "tide_gpu", 16, 32)
    with HydroStep(Deck(path), strict=True) as hs:
        z = sample(hs.run, lambda: hs.modal2nodal()[0])
    err = np.abs(z - analytic(r)) / AMP
    print(f"analytic tide on the device: max {err.max():.2e}, rms {np.sqrt(np.mean(err ** 2)):.2e} of A")
    assert err.max() < 5e-3
    orc = Oracle(path, threads=4)
    try:
        zo = sample(lambda it0, n: orc.run(it0, it0 + n - 1), lambda: orc.modal2nodal()[0])
    finally:
        orc.close()
    assert np.abs(z - zo).max() <= 1e-10 * AMP
