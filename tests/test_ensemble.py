"""dgswem_deck_merge (host only): the merged setup holds every member's mesh
side by side with ids offset, and members that differ in what the kernels
read as one value are rejected."""
import numpy as np
import pytest

from dgswem_b200 import Deck, decks
from dgswem_b200._abi import DgswemError
from dgswem_b200.ensemble import make_members


def _offsets(ds, attr):
    return np.concatenate([[0], np.cumsum([getattr(d.s, attr) for d in ds])])


def test_merge_concatenates_with_offsets(built, scratch):
    specs = decks.ensemble_specs(5, seed=11, ne_min=300, ne_max=2000)
    ds, _ = make_members(scratch / "ens_merge", specs, nsteps=10)
    m = Deck.merge(ds)
    s = m.s
    eo, no, edo = _offsets(ds, "ne"), _offsets(ds, "np"), _offsets(ds, "nedges")
    assert (s.ne, s.np, s.nedges) == (eo[-1], no[-1], edo[-1])
    for k in ("nieds", "nleds", "needs"):
        assert getattr(s, k) == sum(getattr(d.s, k) for d in ds)
    nm = m.int_array("nm", 3 * s.ne).reshape(3, s.ne)
    neled = m.int_array("neled", 3 * s.ne)
    nedno = m.int_array("nedno", 2 * s.nedges)
    nedel = m.int_array("nedel", 2 * s.nedges)
    nedsd = m.int_array("nedsd", 2 * s.nedges)
    hb = m.real_array("hb", 3 * s.ne)
    x = m.real_array("x", s.np)
    man = m.real_array("manning", s.np)
    lists = {k: (m.int_array(k, getattr(s, c)), c) for k, c in (("niedn", "nieds"), ("nledn", "nleds"),
                                                                ("needn", "needs"))}
    lo = {k: 0 for k in lists}
    emo = m.real_array("emo_dg", 2 * s.needs)
    eoff = 0
    for i, d in enumerate(ds):
        t = d.s
        np.testing.assert_array_equal(nm[:, eo[i]:eo[i + 1]], d.int_array("nm", 3 * t.ne).reshape(3, t.ne) + no[i])
        le = d.int_array("neled", 3 * t.ne)
        np.testing.assert_array_equal(neled[3 * eo[i]:3 * eo[i + 1]], np.where(le == 0, 0, le + edo[i]))
        np.testing.assert_array_equal(nedno[2 * edo[i]:2 * edo[i + 1]], d.int_array("nedno", 2 * t.nedges) + no[i])
        de = d.int_array("nedel", 2 * t.nedges)
        np.testing.assert_array_equal(nedel[2 * edo[i]:2 * edo[i + 1]], np.where(de == 0, 0, de + eo[i]))
        np.testing.assert_array_equal(nedsd[2 * edo[i]:2 * edo[i + 1]], d.int_array("nedsd", 2 * t.nedges))
        np.testing.assert_array_equal(hb[3 * eo[i]:3 * eo[i + 1]], d.real_array("hb", 3 * t.ne))
        np.testing.assert_array_equal(x[no[i]:no[i + 1]], d.real_array("x", t.np))
        np.testing.assert_array_equal(man[no[i]:no[i + 1]], d.real_array("manning", t.np))
        for k, (arr, c) in lists.items():
            n = getattr(t, c)
            np.testing.assert_array_equal(arr[lo[k]:lo[k] + n], d.int_array(k, n) + edo[i])
            lo[k] += n
        # EMO_DG(1, NEEDS, 2): both endpoint rows of each member's ocean edges
        e1 = d.real_array("emo_dg", 2 * t.needs)
        np.testing.assert_array_equal(emo[eoff:eoff + t.needs], e1[:t.needs])
        np.testing.assert_array_equal(emo[s.needs + eoff:s.needs + eoff + t.needs], e1[t.needs:])
        eoff += t.needs
    m.close()


def test_merge_rejects_incompatible_members(built, scratch):
    a = decks.ensemble_member(scratch / "inc_a", "rectangle", 400, 1.0, 0.02, 1)
    b = decks.ensemble_member(scratch / "inc_b", "annulus", 400, 1.0, 0.02, 2, dt=0.25)
    with pytest.raises(DgswemError, match="time step"):
        Deck.merge([Deck(a), Deck(b)])
    c = decks.quarter_annulus(scratch / "inc_c", nr=4, nth=8, nsteps=2)  # linear friction, no wet/dry
    with pytest.raises(DgswemError, match="physics switch"):
        Deck.merge([Deck(a), Deck(c)])
    with pytest.raises(DgswemError, match="empty"):
        Deck.merge([])


def test_merge_p2_members(built, scratch):
    """p=2 members: six bathymetry modes per element carried over."""
    p2 = {"extra": {"pl": 2, "ph": 2}}
    a = decks.quarter_annulus(scratch / "p2m_a", nr=4, nth=8, nsteps=2, **p2)
    b = decks.quarter_annulus(scratch / "p2m_b", nr=6, nth=6, nsteps=2, **p2)
    da, db = Deck(a), Deck(b)
    m = Deck.merge([da, db])
    assert m.s.dofh == 6 and m.s.ne == da.s.ne + db.s.ne
    hb = m.real_array("hb", 6 * m.s.ne)
    np.testing.assert_array_equal(hb[:6 * da.s.ne], da.real_array("hb", 6 * da.s.ne))
    np.testing.assert_array_equal(hb[6 * da.s.ne:], db.real_array("hb", 6 * db.s.ne))
    m.close()
