"""The library's standalone input path (READ_INPUT + PREP_DG restated in
dgswem_b200/csrc/deck.cpp) against the oracle: integer edge tables are
compared bit for bit, real setup arrays exactly."""
import numpy as np
import pytest

from conftest import GOLDEN_CASES, golden_dir
from dgswem_b200 import Deck, decks
from oracle_lib import Oracle


def _decks(scratch):
    out = [golden_dir(c) for c in GOLDEN_CASES]
    out.append(decks.quarter_annulus(scratch / "qa_small", nr=8, nth=16, nsteps=20))
    out.append(decks.sloping_beach(scratch / "sb_small", nx=40, ny=8, nsteps=20))
    # periodic flux (ibtype 2) and radiation (ibtype 30) boundaries
    out.append(decks.quarter_annulus(scratch / "qa_flowrad", nr=8, nth=16, nsteps=20, flow_amp=0.05,
                                     radiation=True))
    return out


def test_edge_tables_bit_exact(built, scratch):
    for path in _decks(scratch):
        d = Deck(path)
        o = Oracle(path)
        s = d.s
        ned, ne = s.nedges, s.ne
        assert ned == o.info("nedges"), path
        for name, n in [("nedno", 2 * ned), ("nedel", 2 * ned), ("nedsd", 2 * ned)]:
            np.testing.assert_array_equal(d.int_array(name, n), o.int_table(name.upper()), err_msg=f"{path} {name}")
        # NELED(3,NE) is stored [l + 3*e] in both
        np.testing.assert_array_equal(d.int_array("neled", 3 * ne), o.int_table("NELED"))
        for name, cnt in [("niedn", s.nieds), ("nledn", s.nleds), ("needn", s.needs), ("nfedn", s.nfeds),
                          ("nredn", s.nreds), ("nebsegn", s.nebseg), ("nibsegn", 2 * s.nibseg)]:
            np.testing.assert_array_equal(d.int_array(name, cnt), o.int_table(name.upper()),
                                          err_msg=f"{path} {name}")
        ze0, _, _, wd0 = o.state()
        np.testing.assert_array_equal(d.int_array("wdflg", ne), wd0)
        np.testing.assert_array_equal(d.real_array("ze", 3 * ne), ze0.ravel())
        np.testing.assert_array_equal(d.real_array("dp", s.np), o.real_table("DP"))
        np.testing.assert_array_equal(d.real_array("x", s.np), o.real_table("X"))
        np.testing.assert_array_equal(d.real_array("y", s.np), o.real_table("Y"))
        np.testing.assert_array_equal(d.real_array("hb", 3 * ne), o.real_table("HB"))
        assert s.nrk == o.info("nrk")
        d.close()
        o.close()


def test_wetdry_golden_deck_contents(built):
    d = Deck(golden_dir("wetdry"))
    s = d.s
    # wetdry golden: external barriers (type 3) and internal barriers (type 24)
    assert s.nebseg > 0 and s.nibseg > 0 and s.needs > 0
    assert s.nolifa == 2 and s.nrk == 5 and s.ifhybf == 1
    assert d.control("nspoolge") == 100 and d.control("nt") == 1728


def test_deck_errors_are_status_codes(built, scratch):
    from dgswem_b200._abi import DgswemError
    with pytest.raises(DgswemError, match="cannot open"):
        Deck(scratch / "does_not_exist")
    bad = decks.quarter_annulus(scratch / "qa_cw", nr=2, nth=2, nsteps=1)
    text = (bad / "fort.14").read_text().split("\n")
    # flip the first element to clockwise order (read_input.F:1408-1419 stops)
    parts = text[2 + 9].split()
    text[2 + 9] = " ".join([parts[0], parts[1], parts[2], parts[4], parts[3]])
    (bad / "fort.14").write_text("\n".join(text))
    with pytest.raises(DgswemError, match="clockwise"):
        Deck(bad)


def test_p2_deck(built, scratch):
    """fort.dg with pl = ph = 2: DOFH = 6, the bathymetry's six modes (the
    linear nodal depth's modes 1-3, zeros above) equal to the oracle's, and
    the edge tables of the same mesh; the limiter and wet/dry refused at p=2
    as the reference has them at p=1 only."""
    from dgswem_b200._abi import DgswemError
    p2 = {"extra": {"pl": 2, "ph": 2}}
    path = decks.quarter_annulus(scratch / "deck_p2", nr=4, nth=8, nsteps=2, **p2)
    d = Deck(path)
    ne = d.s.ne
    assert d.s.dofh == 6
    hb = d.real_array("hb", 6 * ne).reshape(ne, 6)
    orc = Oracle(path)
    assert orc.dofh == 6
    np.testing.assert_array_equal(hb, orc.real_table("HB").reshape(ne, 6))
    assert not hb[:, 3:].any()
    np.testing.assert_array_equal(d.int_array("nedno", 2 * d.s.nedges), orc.int_table("NEDNO"))
    orc.close()
    d.close()
    for kw in ({"slopeflag": 5}, {"nolifa": 2}):
        bad = decks.quarter_annulus(scratch / f"deck_p2_{next(iter(kw))}", nr=4, nth=8, nsteps=2, **kw, **p2)
        with pytest.raises(DgswemError, match="p = 1 only"):
            Deck(bad)


def test_line_endings_do_not_change_the_deck(built, scratch):
    """The reader splits its files into records at line feeds, in parallel
    chunks: CRLF line endings, blank lines after the tables and a last line
    without a line feed give the same deck as the plain files."""
    import shutil
    plain = decks.sloping_beach(scratch / "le_plain", nx=40, ny=8, nsteps=20)
    crlf = scratch / "le_crlf"
    shutil.rmtree(crlf, ignore_errors=True)
    shutil.copytree(plain, crlf)
    for name in ("fort.14", "fort.15", "fort.13"):
        text = (plain / name).read_text()
        (crlf / name).write_text(text.rstrip("\n").replace("\n", "\r\n") + ("\r\n\r\n" if name == "fort.14" else ""),
                                 newline="")
    a, b = Deck(plain), Deck(crlf)
    s, t = a.s, b.s
    assert (s.ne, s.np, s.nedges) == (t.ne, t.np, t.nedges)
    for name, n in [("nm", 3 * s.ne), ("nedno", 2 * s.nedges), ("nedel", 2 * s.nedges), ("neled", 3 * s.ne)]:
        np.testing.assert_array_equal(a.int_array(name, n), b.int_array(name, n), err_msg=name)
    for name, n in [("x", s.np), ("y", s.np), ("dp", s.np)]:
        np.testing.assert_array_equal(a.real_array(name, n), b.real_array(name, n), err_msg=name)
    a.close()
    b.close()
