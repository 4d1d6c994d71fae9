"""DG hot start (Hot_start.263 / .264 / .214): the writer's layout read back
by the deck reader with MODAL_IC = 2 (CPU), and a run restarted from a hot
start equal to the run it was taken from, bit for bit (GPU)."""
import shutil

import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks, run_case, write_hotstart
from dgswem_b200._abi import DgswemError


def _beach(path, **kw):
    return decks.sloping_beach(path, nx=24, ny=6, lx=1200.0, ly=300.0, nsteps=40, dt=0.5, dramp=0.002, **kw)


def test_hotstart_written_and_read_back(built, scratch):
    path = decks.quarter_annulus(scratch / "hs_qa", nr=4, nth=8, nsteps=10)
    d0 = Deck(path)
    ne, dofh, dtdp = d0.s.ne, d0.s.dofh, d0.s.dtdp
    hb = d0.real_array("hb", ne * dofh).reshape(ne, dofh)
    d0.close()
    rng = np.random.default_rng(3)
    ze, qx, qy = (rng.standard_normal((ne, dofh)) * 10.0 ** rng.integers(-12, 3, (ne, dofh)) for _ in range(3))
    wd = rng.integers(0, 2, ne).astype(np.int32)
    hot = decks.quarter_annulus(scratch / "hs_qa_hot", nr=4, nth=8, nsteps=10, extra={"modal_ic": 2})
    write_hotstart(hot, 1, 7, dtdp, ze, qx, qy, hb, wd)
    d = Deck(hot)
    assert d.control("modal_ic") == 2 and d.control("hotstart_it") == 7
    for name, want in (("ze", ze), ("qx", qx), ("qy", qy), ("hb", hb)):
        np.testing.assert_array_equal(d.real_array(name, ne * dofh).reshape(ne, dofh), want, err_msg=name)
    np.testing.assert_array_equal(d.int_array("wdflg", ne), wd)
    d.close()


def test_hotstart_fortran_records_and_p_check(built, scratch):
    """List-directed records as gfortran writes them: D exponents, commas,
    trailing items the reader skips; a hot start of another degree refused."""
    hot = decks.quarter_annulus(scratch / "hs_f", nr=2, nth=4, nsteps=2, extra={"modal_ic": 2})
    d0 = Deck(decks.quarter_annulus(scratch / "hs_f0", nr=2, nth=4, nsteps=2))
    ne, dofh = d0.s.ne, d0.s.dofh
    n = ne * dofh
    (hot / "Hot_start.263").write_text(" 1\n" + "".join(f"   {0.25 * i:.16E}\n".replace("E", "D") for i in range(n)))
    (hot / "Hot_start.264").write_text("  1,  1\n" + "".join(f" {i}.5D-01, -{i}.0D0\n" for i in range(n)))
    (hot / "Hot_start.214").write_text(" 40  2.0000000000000000D+00  extra\n" +
                                       "".join(f"  3.048D0  {1 if (i // dofh) % 2 else 0}\n" for i in range(n)))
    d = Deck(hot)
    assert d.control("hotstart_it") == 40
    np.testing.assert_array_equal(d.real_array("ze", n), 0.25 * np.arange(n))
    np.testing.assert_array_equal(d.real_array("qx", n), np.array([float(f"{i}.5e-01") for i in range(n)]))
    np.testing.assert_array_equal(d.real_array("qy", n), -np.arange(n, dtype=float))
    np.testing.assert_array_equal(d.int_array("wdflg", ne), np.arange(ne) % 2)
    d.close()
    (hot / "Hot_start.263").write_text(" 2\n" + "0.0\n" * n)
    with pytest.raises(DgswemError, match="INCONSISTENCY IN P"):
        Deck(hot)


@pytest.mark.gpu
def test_restart_from_hotstart_matches_straight_run(built, scratch):
    """Wet/dry beach with limiter and Manning n: 20 steps, hot start, 20
    more from the hot start == 40 steps straight, bit for bit."""
    path = _beach(scratch / "hs_beach")
    with HydroStep(Deck(path)) as hs:
        hs.run(1, 40)
        want = hs.state()
    hot = _beach(scratch / "hs_beach_hot", extra={"modal_ic": 2})
    with HydroStep(Deck(path)) as hs:
        hs.run(1, 20)
        hs.write_hotstart(hot, 20)
    d = Deck(hot)
    assert d.control("hotstart_it") == 20
    with HydroStep(d) as hs:
        hs.run(21, 20)
        got = hs.state()
    for a, b, v in zip(got, want, ("ZE", "QX", "QY", "WDFLG")):
        np.testing.assert_array_equal(a, b, err_msg=v)
    assert 0 < want[3].sum() < len(want[3])  # wet and dry elements


@pytest.mark.gpu
def test_run_case_writes_and_resumes_hotstart(built, scratch):
    """run_case with DGHOT = 1 writes the hot start at step 20; a deck with
    MODAL_IC = 2 and those files resumes at step 21 and reproduces the
    straight run's later fort.63 snapshots."""
    full = run_case(_beach(scratch / "rc_full", nspoolge=5), nsteps=40)
    first = _beach(scratch / "rc_first", nspoolge=5, extra={"dghot": 1, "dghotspool": 20})
    run_case(first, nsteps=20)
    resume = _beach(scratch / "rc_resume", nspoolge=5, extra={"modal_ic": 2})
    for f in ("Hot_start.263", "Hot_start.264", "Hot_start.214"):
        shutil.copy(first / f, resume / f)
    later = run_case(resume, nsteps=40)
    want = [s for s in full if s[0] > 20]
    assert len(later) == len(want) == 4
    for (ia, a), (ib, b) in zip(later, want):
        assert ia == ib
        np.testing.assert_array_equal(a, b)
