"""Partition plan of the partitioned handles (host only, no GPU).

Partition p owns a contiguous range of the elements' Morton order; its halo
lists must agree with its peers' (what p sends q is what q expects from p, in
the same order), cover every element an owned element's stage reads from
another partition, and be the same when each partition computes them in its
own process (world size 2, gloo)."""
import ctypes as C
import json
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from dgswem_b200 import Deck, _abi

ROOT = Path(__file__).resolve().parents[1]


def halo_ids(deck, part, nparts, peer, kind):
    lib = _abi.load()
    ns, nr = C.c_int(), C.c_int()
    _abi.check(lib.dgswem_part_halo_ids(deck.setup, part, nparts, peer, kind, None, C.byref(ns), None, C.byref(nr)))
    snd = np.zeros(max(ns.value, 1), np.int32)
    rcv = np.zeros(max(nr.value, 1), np.int32)
    _abi.check(lib.dgswem_part_halo_ids(deck.setup, part, nparts, peer, kind,
                                        snd.ctypes.data_as(C.POINTER(C.c_int)), C.byref(ns),
                                        rcv.ctypes.data_as(C.POINTER(C.c_int)), C.byref(nr)))
    return snd[:ns.value], rcv[:nr.value]


def owners(deck, nparts):
    """Owner of every element, from the receive lists of the other parts plus
    the elements nobody receives (checked below to be a partition)."""
    ne = deck.s.ne
    own = np.full(ne, -1)
    for p in range(nparts):
        for q in range(nparts):
            if q == p:
                continue
            for kind in (0, 1):
                snd, _ = halo_ids(deck, p, nparts, q, kind)
                own[snd] = p
    return own


@pytest.mark.parametrize("nparts", [2, 3, 5])
@pytest.mark.parametrize("case", ["wetdry", "quarter_annular"])
def test_halo_lists_agree_and_cover(built, case, nparts):
    from conftest import golden_dir
    deck = Deck(golden_dir(case))
    s = deck.s
    ne, ned = s.ne, s.nedges
    nedel = deck.int_array("nedel", 2 * ned).reshape(ned, 2) - 1
    nm = deck.int_array("nm", 3 * ne).reshape(3, ne).T - 1
    own = owners(deck, nparts)
    for p in range(nparts):
        for q in range(nparts):
            if p == q:
                continue
            for kind in (0, 1):
                snd, _ = halo_ids(deck, p, nparts, q, kind)
                _, rcv = halo_ids(deck, q, nparts, p, kind)
                np.testing.assert_array_equal(snd, rcv)
                assert np.all(np.diff(snd) > 0)
    # every edge neighbour across partitions is in the full-state halo
    for a, b in nedel:
        if a < 0 or b < 0 or own[a] < 0 or own[b] < 0 or own[a] == own[b]:
            continue
        snd, _ = halo_ids(deck, own[a], nparts, own[b], 1)
        assert a in set(snd.tolist())
    # every node neighbour across partitions is in the means halo
    by_node = {}
    for e in range(ne):
        for n in nm[e]:
            by_node.setdefault(int(n), []).append(e)
    for els in by_node.values():
        for a in els:
            for b in els:
                if own[a] >= 0 and own[b] >= 0 and own[a] != own[b]:
                    snd, _ = halo_ids(deck, own[a], nparts, own[b], 0)
                    assert a in set(snd.tolist())


def test_partition_index_errors(built):
    from conftest import golden_dir
    deck = Deck(golden_dir("quarter_annular"))
    lib = _abi.load()
    ns, nr = C.c_int(), C.c_int()
    assert lib.dgswem_part_halo_ids(deck.setup, 2, 2, 0, 1, None, C.byref(ns), None, C.byref(nr)) == 1
    assert lib.dgswem_part_halo_ids(deck.setup, 0, 2, 5, 1, None, C.byref(ns), None, C.byref(nr)) == 1
    assert lib.dgswem_part_halo_ids(deck.setup, 0, 2, 1, 7, None, C.byref(ns), None, C.byref(nr)) == 1


def test_halo_lists_two_gloo_ranks(built, tmp_path):
    """Each rank computes its own partition's lists in its own process; the
    ranks swap them over gloo and check they match."""
    from conftest import golden_dir
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    worker = ROOT / "tests" / "partition_ranks_worker.py"
    procs = [subprocess.Popen([sys.executable, str(worker), str(r), "2", str(port), str(golden_dir("wetdry")),
                               str(tmp_path / f"rank{r}.json")]) for r in range(2)]
    for p in procs:
        assert p.wait(timeout=300) == 0
    for r in range(2):
        res = json.loads((tmp_path / f"rank{r}.json").read_text())
        assert res["agree"] and res["nsend"] > 0
