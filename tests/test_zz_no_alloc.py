"""dgswem_cuda_modal2nodal_noalloc (GPU): the nodal output path whose scratch
is a static device array instead of an allocated buffer.

Collected last (file name) so that it also runs after every other GPU test
has created and destroyed handles on the device; it must pass alone in a
fresh process too.  Compared with dgswem_cuda_modal2nodal, the existing
entry point, which launches the same kernel on the same state: the results
must be equal bit for bit.
"""
import ctypes as C

import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, PartitionedRun, decks
from dgswem_b200._abi import DgswemError, check

pytestmark = pytest.mark.gpu

MAX_NODES = 1 << 20  # DGSWEM_CUDA_NOALLOC_MAX_NODES
ERR_ARG = 1  # DGSWEM_ERR_ARG


def check_same(got, want):
    for a, b, name in zip(got, want, ("ETA2", "UU2", "VV2", "NODECODE")):
        np.testing.assert_array_equal(a, b, err_msg=f"{name} differs")


def test_noalloc_matches_modal2nodal_two_calls_in_a_row(built):
    """Two noalloc calls in a row after stepping, then two more after further
    steps (the scratch carries nothing over between calls), each against the
    existing entry point on the same state.  wetdry golden deck: wet and dry
    elements, so NODECODE has both values."""
    from conftest import golden_dir
    with HydroStep(Deck(golden_dir("wetdry"))) as hs:
        assert hs.np <= MAX_NODES
        it = 1
        for _ in range(2):
            for _ in range(60):
                hs.timestep(it)
                it += 1
            first = hs.modal2nodal_noalloc()
            second = hs.modal2nodal_noalloc()
            want = hs.modal2nodal()
            check_same(first, want)
            check_same(second, want)
            assert 0 < want[3].sum() < hs.np


def test_noalloc_two_handles_same_device(built, scratch):
    """Handles of different meshes on one device share the scratch; calls in
    sequence see only their own mesh's nodes."""
    a = decks.quarter_annulus(scratch / "na_a", nr=8, nth=16, nsteps=20, nolibf=1, cf=0.0025, slopeflag=5)
    b = decks.sloping_beach(scratch / "na_b", nx=40, ny=8, lx=2000.0, ly=400.0, nsteps=20, dt=0.5)
    with HydroStep(Deck(a)) as ha, HydroStep(Deck(b)) as hb:
        ha.run(1, 20)
        hb.run(1, 20)
        for _ in range(2):
            check_same(ha.modal2nodal_noalloc(), ha.modal2nodal())
            check_same(hb.modal2nodal_noalloc(), hb.modal2nodal())


def test_noalloc_rejects_more_nodes_than_the_scratch(built, scratch):
    """NP above DGSWEM_CUDA_NOALLOC_MAX_NODES: DGSWEM_ERR_ARG with a message
    naming the limit; the handle stays usable through the existing path."""
    path = decks.sloping_beach(scratch / "na_big", nx=1025, ny=1023, lx=100e3, ly=100e3, nsteps=2)
    with HydroStep(Deck(path)) as hs:
        assert hs.np > MAX_NODES
        with pytest.raises(DgswemError, match="DGSWEM_CUDA_NOALLOC_MAX_NODES"):
            hs.modal2nodal_noalloc()
        eta, _, _, nc = hs.modal2nodal()
        assert eta.shape == (hs.np,) and nc.shape == (hs.np,)


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double)) if a is not None else None


def test_noalloc_null_outputs(built, scratch):
    """Any output may be NULL: ETA2 and NODECODE skipped, UU2 and VV2
    copied, equal to the existing entry point's."""
    path = decks.sloping_beach(scratch / "na_null", nx=40, ny=8, lx=2000.0, ly=400.0, nsteps=20, dt=0.5)
    with HydroStep(Deck(path)) as hs:
        hs.run(1, 20)
        want = hs.modal2nodal()
        uu, vv = np.full(hs.np, np.nan), np.full(hs.np, np.nan)
        for _ in range(2):
            check(hs._lib.dgswem_cuda_modal2nodal_noalloc(hs._h, None, _dp(uu), _dp(vv), None))
            np.testing.assert_array_equal(uu, want[1])
            np.testing.assert_array_equal(vv, want[2])


def test_noalloc_rejects_null_p2_and_partition_handles(built, scratch):
    """The entry point serves p=1 whole-mesh handles: a NULL handle, a p=2
    handle and a partition handle get DGSWEM_ERR_ARG."""
    from dgswem_b200 import _abi
    lib = _abi.load()
    assert lib.dgswem_cuda_modal2nodal_noalloc(None, None, None, None, None) == ERR_ARG
    p2 = decks.quarter_annulus(scratch / "na_p2", nr=4, nth=8, nsteps=2, extra={"pl": 2, "ph": 2})
    with HydroStep(Deck(p2)) as hs:
        assert hs.dofh == 6
        with pytest.raises(DgswemError, match="p=1 only") as e:
            hs.modal2nodal_noalloc()
        assert e.value.status == ERR_ARG
    qa = decks.quarter_annulus(scratch / "na_part", nr=8, nth=16, nsteps=2)
    with PartitionedRun(Deck(qa), 2) as pr:
        with pytest.raises(DgswemError, match="whole mesh"):
            pr.parts[0].modal2nodal_noalloc()
