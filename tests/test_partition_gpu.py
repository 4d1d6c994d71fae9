"""Partitioned mesh on one GPU: 2-4 partition handles stepped in lock-step
with their halos moved through device buffers reproduce the single-handle
run bit for bit (the per-element arithmetic and the summation orders do not
depend on the partition), in both kernel variants, on decks with ocean
forcing, the slope limiter, wet/dry, Manning friction and internal barriers."""
import numpy as np
import pytest

from dgswem_b200 import Deck, HydroStep, PartitionedRun, decks

pytestmark = pytest.mark.gpu


def single_and_parts(path, nsteps, nparts, strict, overlap=False):
    deck = Deck(path)
    with HydroStep(deck, strict=strict) as hs:
        hs.run(1, nsteps)
        ref = hs.state()
    with PartitionedRun(deck, nparts, strict=strict, overlap=overlap) as pr:
        info = [hs.part_info() for hs in pr.parts]
        assert sum(i["owned"] for i in info) == deck.s.ne
        assert all(i["local"] > i["owned"] for i in info)
        pr.run(1, nsteps)
        got = pr.state()
    return ref, got


def check_equal(ref, got):
    for a, b, name in zip(got, ref, ("ZE", "QX", "QY", "WDFLG")):
        np.testing.assert_array_equal(a, b, err_msg=f"{name} differs from the single-handle run")


@pytest.mark.parametrize("strict", [True, False])
@pytest.mark.parametrize("nparts", [2, 3])
def test_wetdry_barriers(built, strict, nparts):
    from conftest import golden_dir
    ref, got = single_and_parts(golden_dir("wetdry"), 150, nparts, strict)
    check_equal(ref, got)


@pytest.mark.parametrize("nparts", [2, 4])
def test_sloping_beach_limiter_manning(built, scratch, nparts):
    path = decks.sloping_beach(scratch / "sb_part", nx=40, ny=10, lx=2000.0, ly=500.0, nsteps=200, dt=0.5)
    ref, got = single_and_parts(path, 200, nparts, strict=False)
    check_equal(ref, got)
    assert 0 < ref[3].sum() < len(ref[3])


def test_quarter_annulus_ocean_forcing(built, scratch):
    path = decks.quarter_annulus(scratch / "qa_part", nr=8, nth=16, nsteps=120, nolibf=1, cf=0.0025, slopeflag=5)
    ref, got = single_and_parts(path, 120, 3, strict=True)
    check_equal(ref, got)


def test_partition_handle_rejects_whole_mesh_calls(built, scratch):
    from dgswem_b200._abi import DgswemError
    path = decks.quarter_annulus(scratch / "qa_part_err", nr=4, nth=8, nsteps=2)
    with HydroStep(Deck(path), part=1, nparts=2) as hs:
        with pytest.raises(DgswemError, match="partitioned"):
            hs.timestep(1)
        with pytest.raises(DgswemError, match="whole mesh"):
            hs.modal2nodal()


def test_partitions_with_other_tile_shapes(built):
    """Each partition's tile plan rebuilt for another tile and limiter shape
    (dgswem_cuda_set_shapes on a partition handle: tiles cover its owned
    elements) still reproduces the single-handle run bit for bit."""
    from conftest import golden_dir
    deck = Deck(golden_dir("wetdry"))
    with HydroStep(deck) as hs:
        hs.run(1, 80)
        ref = hs.state()
    nshape = len(HydroStep.shapes()["tile"])
    with PartitionedRun(deck, 3) as pr:
        for i, p in enumerate(pr.parts):
            p.set_shapes((i + 1) % nshape, i % len(HydroStep.shapes()["limiter"]))
        pr.run(1, 80)
        got = pr.state()
    check_equal(ref, got)


@pytest.mark.parametrize("strict", [True, False])
def test_overlapped_stage_order(built, scratch, strict):
    """Each stage after the first split around the exchange before it: the
    tiles that read no ghost launched before the halo moves, the others
    after the unpack (the order DistributedPartition uses to overlap the
    transfer).  Bit-identical to the single handle; internal-barrier tiles
    count as boundary tiles."""
    from conftest import golden_dir
    beach = decks.sloping_beach(scratch / "sb_overlap", nx=60, ny=12, lx=3000.0, ly=600.0, nsteps=100, dt=0.5)
    for path, n in ((golden_dir("wetdry"), 100), (beach, 100)):
        deck = Deck(path)
        with PartitionedRun(deck, 3, strict=strict, overlap=True) as pr:
            splits = [hs.tile_split() for hs in pr.parts]
        assert sum(a for a, _ in splits) > 0 and all(b > 0 for _, b in splits), splits
        ref, got = single_and_parts(path, n, 3, strict, overlap=True)
        check_equal(ref, got)
