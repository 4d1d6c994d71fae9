"""Convergence order of the oracle's p=1 and p=2 paths (CPU).

The reference's p=2 path is broken (its interior edges integrate modes 1-3
only), so the oracle's p=2 restatement -- the p-generic edge sums, the
6-point area rule, the 4-point Lobatto edge rule and the orthogonal basis of
degree 2 -- has no golden output to be pinned to.  It is checked here by its
order of accuracy instead: a linear standing wave in a closed, flat basin
(NLEQ=0, LEQ=1, no friction), eta = A cos(k x) cos(w t), w = k sqrt(g H),
started from the L2 projection of the exact state on nested meshes and
compared with the exact elevation after 800 s.  DG of degree p converges at
order p+1 in L2 for this smooth problem.
"""
import math

import numpy as np
import pytest

from dgswem_b200 import Deck, decks
from oracle_lib import Oracle

L, W, H, A, G = 10e3, 2.5e3, 10.0, 0.1, 9.81
K = math.pi / L
OMEGA = K * math.sqrt(G * H)
DT, NSTEPS = 2.0, 400


def basin(path, nx: int, p: int):
    ny = nx // 4
    xs, ys = np.linspace(0.0, L, nx + 1), np.linspace(0.0, W, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    elems = decks._grid_triangles(nx, ny)
    nid = lambda i, j: i * (ny + 1) + j + 1  # noqa: E731
    # closed basin: the whole perimeter is land, in two segments
    outer = [nid(i, 0) for i in range(nx + 1)] + [nid(nx, j) for j in range(1, ny + 1)] + \
            [nid(i, ny) for i in range(nx - 1, -1, -1)]
    left = [nid(0, j) for j in range(ny, -1, -1)]
    ctl = decks.Controls(title="standing wave", nolibf=0, tau=0.0, nolifa=0, nolica=0, nolicat=0, dt=DT,
                         nsteps=NSTEPS, rk_stage=3, rk_order=3, slopeflag=0, nramp=0,
                         extra={"pl": p, "ph": p})
    decks.write_deck(path, X.ravel(), Y.ravel(), np.full(X.size, H), elems, [], [(outer, 0), (left, 0)], ctl)
    return X.ravel(), Y.ravel(), elems - 1


def area_points(orc, x, y, elems):
    """Physical coordinates of every element's area points, the weights of
    the physical rule, and the basis there."""
    phi = orc.real_table("PHI_AREA")
    xa, ya, wa = orc.real_table("XAGP"), orc.real_table("YAGP"), orc.real_table("WAGP")
    dofh, nagp = orc.dofh, len(xa)
    phi = phi.reshape(dofh, nagp)
    n1, n2, n3 = elems[:, 0], elems[:, 1], elems[:, 2]
    # reference vertices (-1,-1), (1,-1), (-1,1) -> nodes 1, 2, 3
    l1, l2, l3 = -(xa + ya) / 2, (1 + xa) / 2, (1 + ya) / 2
    px = np.outer(x[n1], l1) + np.outer(x[n2], l2) + np.outer(x[n3], l3)
    py = np.outer(y[n1], l1) + np.outer(y[n2], l2) + np.outer(y[n3], l3)
    area = 0.5 * np.abs((x[n2] - x[n1]) * (y[n3] - y[n1]) - (x[n3] - x[n1]) * (y[n2] - y[n1]))
    wphys = np.outer(area / 2.0, wa)  # the reference triangle's area is 2
    return px, py, wphys, phi, wa


def l2_error(path, nx, p):
    x, y, elems = basin(path, nx, p)
    orc = Oracle(path)
    assert orc.dofh == (p + 1) * (p + 2) // 2
    px, py, wphys, phi, wa = area_points(orc, x, y, elems)
    minv = orc.real_table("M_INV")
    # L2 projection of eta0 = A cos(k x): c_k = M_INV(k) sum_i WAGP_i phi_k(i) eta0(x_i)
    ze = (A * np.cos(K * px) * wa[None, :]) @ phi.T * minv[None, :]
    zero = np.zeros_like(ze)
    orc.set_state(ze, zero, zero, np.ones(len(elems), np.int32))
    orc.run(1, NSTEPS)
    ze, _, _, _ = orc.state()
    orc.close()
    eta_h = ze @ phi  # at the area points
    eta = A * np.cos(K * px) * math.cos(OMEGA * DT * NSTEPS)
    return math.sqrt(float(np.sum(wphys * (eta_h - eta) ** 2)))


@pytest.mark.parametrize("p", [1, 2])
def test_standing_wave_convergence_order(built, tmp_path, p):
    errs = [l2_error(tmp_path / f"sw_p{p}_{nx}", nx, p) for nx in (8, 16, 32)]
    rates = [math.log2(errs[i] / errs[i + 1]) for i in range(2)]
    print(f"p={p} errors {errs} rates {rates}")
    assert all(r > p + 1 - 0.4 for r in rates), (errs, rates)


def bump_state(path, p):
    """The closed basin with the full nonlinear equations (NOLIFA=1) and the
    L2 projection of a Gaussian bump of elevation: (ZE modes, HB modes,
    element areas), from the oracle's tables."""
    x, y, elems = basin(path, 16, p)
    f15 = (path / "fort.15").read_text()
    for key in ("NOLIFA", "NOLICA", "NOLICAT"):  # the full nonlinear equations
        f15 = f15.replace(f"0 ! {key}\n", f"1 ! {key}\n")
    (path / "fort.15").write_text(f15)
    deck = Deck(path)
    assert deck.s.nleq == 1.0 and deck.s.leq == 0.0
    deck.close()
    orc = Oracle(path)
    px, py, wphys, phi, wa = area_points(orc, x, y, elems)
    minv = orc.real_table("M_INV")
    bump = 0.5 * np.exp(-(((px - 0.4 * L) / 1500.0) ** 2 + ((py - 0.5 * W) / 800.0) ** 2))
    ze = (bump * wa[None, :]) @ phi.T * minv[None, :]
    hb = orc.real_table("HB").reshape(len(elems), orc.dofh)
    orc.close()
    return ze, hb, np.sum(wphys, axis=1)


def water_volume(ze, hb, area) -> float:
    """sum_e (ZE_1 + HB_1) * area (mode 1 is the element mean)."""
    return float(np.sum((ze[:, 0] + hb[:, 0]) * area))


@pytest.mark.parametrize("p", [1, 2])
def test_closed_basin_mass_conserved(built, tmp_path, p):
    """Nonlinear equations (NOLIFA=1) in the closed basin from a Gaussian
    bump: the water volume stays constant to round-off over 400 steps."""
    path = tmp_path / f"mass_p{p}"
    ze, hb, area = bump_state(path, p)
    orc = Oracle(path)
    zero = np.zeros_like(ze)
    orc.set_state(ze, zero, zero, np.ones(len(ze), np.int32))
    vol0 = water_volume(ze, hb, area)
    orc.run(1, NSTEPS)
    z, qx, _, _ = orc.state()
    orc.close()
    vol1 = water_volume(z, hb, area)
    assert np.abs(qx).max() > 1e-4  # the bump spread
    assert abs(vol1 - vol0) <= 1e-12 * vol0, (vol0, vol1)
