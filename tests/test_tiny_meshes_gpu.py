"""Meshes smaller than a warp and a tile (GPU): two to six elements, where
every tile is partial, halos and edge-task lists are a handful of entries
and every node star is cut by the boundary.  The strict build against the
oracle, bit for bit, after 20 steps: state, wet/dry flags and nodal codes.

* a 2-element quarter annulus (one cell: ocean arc, land elsewhere);
* a 4-element quarter annulus at p=2, SSP(3,3);
* 2- and 6-element sloping beaches with WETDRY, slope limiter 5 and nodal
  Manning n (the 2-element one ends dry, the 6-element one part wet, part
  dry).
"""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

NSTEPS = 20

TINY = {
    "annulus_2": lambda p: decks.quarter_annulus(p, nr=1, nth=1, nsteps=NSTEPS),
    "annulus_4_p2": lambda p: decks.quarter_annulus(p, nr=1, nth=2, nsteps=NSTEPS, rk_stage=3, rk_order=3,
                                                    extra={"pl": 2, "ph": 2}),
    "beach_2": lambda p: decks.sloping_beach(p, nx=1, ny=1, lx=1000.0, ly=500.0, nsteps=NSTEPS),
    "beach_6": lambda p: decks.sloping_beach(p, nx=3, ny=1, lx=3000.0, ly=500.0, nsteps=NSTEPS),
}


@pytest.mark.parametrize("name", sorted(TINY))
def test_tiny_mesh_strict_bitwise(built, tmp_path, name):
    path = TINY[name](tmp_path / name)
    deck = Deck(path)
    assert deck.s.ne <= 6
    orc = Oracle(path, threads=1)
    try:
        with HydroStep(deck, strict=True) as hs:
            hs.run(1, NSTEPS)
            hs.synchronize()
            g = hs.state()
            gnc = hs.modal2nodal()[3]
        orc.run(1, NSTEPS)
        o = orc.state()
        for a, b, what in zip(g, o, ("ZE", "QX", "QY", "WDFLG")):
            np.testing.assert_array_equal(a, b, err_msg=f"{name}: {what} not bit-identical")
        if deck.s.dofh == 3:
            np.testing.assert_array_equal(gnc, orc.nodecode())
    finally:
        orc.close()
        deck.close()
