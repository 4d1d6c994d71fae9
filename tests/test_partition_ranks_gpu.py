"""The one-partition-per-process driver (DistributedPartition) run for real:
two processes, each a rank of a gloo group stepping its own partition on
cuda:0, the halos staged through pinned host buffers (transport "host").
No kernel waits on the other rank: every exchange is a host-side send and
receive between launches.  The assembled owned rows must equal the
single-handle run bit for bit, as the in-process PartitionedRun does
(tests/test_partition_gpu.py)."""
import socket
import subprocess
import sys
from pathlib import Path

import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, decks

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]


def free_port() -> int:
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        return sk.getsockname()[1]


def run_two_ranks(path, nsteps, strict, tmp_path, overlap=True):
    port = free_port()
    worker = ROOT / "tests" / "partition_gpu_worker.py"
    outs = [tmp_path / f"rank{r}.npz" for r in range(2)]
    procs = [subprocess.Popen([sys.executable, str(worker), str(r), "2", str(port), str(path), str(nsteps),
                               str(int(strict)), str(outs[r]), str(int(overlap))]) for r in range(2)]
    try:
        for p in procs:
            assert p.wait(timeout=600) == 0
    finally:
        for p in procs:
            if p.poll() is None:
                p.kill()
    parts = [np.load(o) for o in outs]
    ze, qx, qy = (np.full_like(parts[0][k], np.nan) for k in ("ze", "qx", "qy"))
    wd = np.full_like(parts[0]["wd"], -1)
    for d in parts:
        own = d["wd"] >= 0
        assert not np.any(wd[own] >= 0), "an element owned by both ranks"
        ze[own], qx[own], qy[own], wd[own] = d["ze"][own], d["qx"][own], d["qy"][own], d["wd"][own]
    assert np.all(wd >= 0), "an element owned by no rank"
    assert sum(int(d["owned"]) for d in parts) == len(wd)
    return ze, qx, qy, wd


def single(path, nsteps, strict):
    with HydroStep(Deck(path), strict=strict) as hs:
        hs.run(1, nsteps)
        return hs.state()


@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("case", ["wetdry_golden", "beach"])
def test_two_ranks_host_transport_bitwise(built, scratch, tmp_path, case, overlap):
    """Reference wetdry golden deck (barriers, hybrid friction, wet/dry) and
    a limiter + Manning sloping beach, strict build; with and without the
    overlapped stage order."""
    if case == "wetdry_golden":
        from conftest import golden_dir
        path, n = golden_dir("wetdry"), 100
    else:
        path, n = decks.sloping_beach(scratch / "sb_ranks", nx=60, ny=12, lx=3000.0, ly=600.0, nsteps=150,
                                      dt=0.5), 150
    ref = single(path, n, True)
    got = run_two_ranks(path, n, True, tmp_path, overlap)
    for a, b, name in zip(got, ref, ("ZE", "QX", "QY", "WDFLG")):
        np.testing.assert_array_equal(a, b, err_msg=f"{name} differs from the single-handle run")
    assert 0 < ref[3].sum() < len(ref[3])
