"""NWS = 1 meteorological forcing read from fort.22 (met_forcing.F:49-66):
NP records "NHG, WSX2, WSY2, PR2" per MET_FORCING call, one call per RK
stage (DG_hydro_timestep.F:104).

CPU: the library's host reader (dgswem_met_reader, the one the handle uses)
against the values written, across list-directed record layouts (blanks,
tabs, commas, D exponents, a record split over lines, extra values after
the fourth); end of file and bad values are errors; the oracle reading the
deck's fort.22 equals the oracle given the same constant fields.
GPU: a deck with fields that change every stage stepped by the library
(dgswem_cuda_met_file) and by the oracle, bit for bit (strict build), and
run_case reading the deck's fort.22."""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks
from dgswem_b200._abi import DgswemError
from dgswem_b200.hydro import MetReader, run_case
from oracle_lib import Oracle


def fields(np_, nblocks, seed=5):
    rng = np.random.default_rng(seed)
    for b in range(nblocks):
        yield (1e-4 * (1 + 0.1 * b) * rng.uniform(0.5, 1.5, np_), -5e-5 * rng.uniform(0.5, 1.5, np_),
               1e-2 * rng.standard_normal(np_))


def test_reader_values_and_record_layouts(built, tmp_path):
    np_ = 5
    blocks = list(fields(np_, 3))
    decks.write_fort22(tmp_path / "fort.22", blocks)
    with MetReader(tmp_path / "fort.22", np_) as r:
        for b in blocks:
            got = r.next()
            for a, w in zip(got, b):
                np.testing.assert_array_equal(a, w)
        assert r.calls == 3
        with pytest.raises(DgswemError, match="end of file"):
            r.next()
    # list-directed layouts: commas, tabs, D exponents, a record over two
    # lines, values after the fourth skipped, blank lines inside a record
    text = ("1, 1.5D-4, -2.0d-5, 3.0\n"
            "2\t2.5E-4\t-3.0E-5\t4.0 99 98\n"
            "3 3.5e-4\n"
            "\n"
            "-4.0e-5 5.0\n")
    (tmp_path / "f22b").write_text(text)
    with MetReader(tmp_path / "f22b", 3) as r:
        wsx, wsy, pr = r.next()
    np.testing.assert_array_equal(wsx, [1.5e-4, 2.5e-4, 3.5e-4])
    np.testing.assert_array_equal(wsy, [-2.0e-5, -3.0e-5, -4.0e-5])
    np.testing.assert_array_equal(pr, [3.0, 4.0, 5.0])
    (tmp_path / "f22c").write_text("1 0.1 0.2 x\n")
    with MetReader(tmp_path / "f22c", 1) as r:
        with pytest.raises(DgswemError, match="not a number"):
            r.next()
    with pytest.raises(DgswemError, match="cannot open"):
        MetReader(tmp_path / "missing", 1)


def test_oracle_fort22_equals_constant_fields(built, scratch):
    """A fort.22 that repeats one field at every stage gives the oracle the
    same run as orc_set_met with that field (the ramp applied per stage the
    same way)."""
    path = decks.quarter_annulus(scratch / "f22_const", nr=6, nth=12, nsteps=10, nws=1)
    d = Deck(path)
    npn, nrk = d.s.np, d.s.nrk
    d.close()
    w = next(fields(npn, 1))
    decks.write_fort22(path / "fort.22", [w] * (10 * nrk))
    a = Oracle(path)
    a.run(1, 10)
    sa = a.state()
    b = Oracle(path)
    b.set_met(*w)  # replaces the deck's fort.22
    b.run(1, 10)
    sb = b.state()
    for x, y in zip(sa, sb):
        np.testing.assert_array_equal(x, y)
    assert np.abs(sa[1]).max() > 0


@pytest.mark.gpu
def test_library_fort22_matches_oracle_bitwise(built, scratch):
    """Fields that change at every RK stage: the library reads fort.22 per
    stage like the oracle (and the reference); strict build bit for bit, in
    steps of several launches (dgswem_cuda_run) and one at a time."""
    n = 30
    path = decks.quarter_annulus(scratch / "f22_var", nr=8, nth=16, nsteps=n, nws=1, nolibf=1, cf=0.0025,
                                 slopeflag=5)
    d = Deck(path)
    decks.write_fort22(path / "fort.22", fields(d.s.np, n * d.s.nrk))
    orc = Oracle(path, threads=4)
    orc.run(1, n)
    o = orc.state()
    with HydroStep(d, strict=True) as hs:
        hs.met_file(path / "fort.22")
        hs.run(1, n // 2)
        for it in range(n // 2 + 1, n + 1):
            hs.timestep(it)
        hs.synchronize()
        g = hs.state()
        with pytest.raises(DgswemError, match="end of file"):
            hs.timestep(n + 1)
    for a, b in zip(g, o):
        np.testing.assert_array_equal(a, b)
    d.close()


@pytest.mark.gpu
def test_run_case_reads_fort22(built, scratch):
    n = 12
    path = decks.quarter_annulus(scratch / "f22_case", nr=6, nth=12, nsteps=n, nws=1)
    d = Deck(path)
    decks.write_fort22(path / "fort.22", fields(d.s.np, n * d.s.nrk, seed=9))
    d.close()
    snaps = run_case(path, nsteps=n, strict=True)
    assert snaps
    it, eta = snaps[-1]
    orc = Oracle(path)
    orc.run(1, it)
    e2, _, _ = orc.modal2nodal()
    np.testing.assert_allclose(eta, np.where(np.abs(e2) <= 1e-30, 0.0, e2), rtol=1e-13, atol=0)
