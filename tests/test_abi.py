"""The C-ABI library without a GPU: it loads, exports every entry point
include/dgswem_cuda.h declares, and a create call on a machine without a GPU
fails with a status code instead of aborting."""
import ctypes as C
import re
from pathlib import Path

import pytest

from dgswem_b200 import _abi, Deck, decks

HEADER = Path(__file__).resolve().parents[1] / "include" / "dgswem_cuda.h"


def declared_functions():
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(dgswem_(?:cuda|deck)_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(built):
    lib = _abi.load()
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in _abi.SIGNATURES, f"{name} missing from the ctypes mirror"


def test_setup_struct_mirror_matches_header(built):
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    body = text[text.index("typedef struct dgswem_cuda_setup {"):text.index("} dgswem_cuda_setup;")]
    fields = []
    for decl in body.split(";")[:-1]:
        decl = decl.split("{")[-1].strip()
        names = [n.strip().lstrip("*") for n in re.sub(r"^(const\s+)?(int|double)\s*\*?", "", decl).split(",")]
        fields += [n for n in names if n]
    assert fields == [f[0] for f in _abi.Setup._fields_]


def test_create_without_gpu_returns_status(built, scratch):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    path = decks.quarter_annulus(scratch / "qa_nogpu", nr=2, nth=4, nsteps=1)
    d = Deck(path)
    h = C.c_void_p()
    rc = _abi.load().dgswem_cuda_create(d.setup, 0, 0, C.byref(h))
    assert rc == 2 and not h.value  # DGSWEM_ERR_CUDA, no handle, process alive
    buf = C.create_string_buffer(256)
    _abi.load().dgswem_cuda_last_error(buf, 256)
    assert buf.value


def test_bad_arguments(built):
    lib = _abi.load()
    h = C.c_void_p()
    assert lib.dgswem_cuda_create(None, 0, 0, C.byref(h)) == 1
    assert lib.dgswem_cuda_hydro_timestep(None, 1) == 1


@pytest.mark.parametrize("table,index,value,message", [
    ("nm", 5, 10**6, "NM refers to a node"),
    ("nm", 0, 0, "NM refers to a node"),
    ("neled", 7, -3, "NELED refers to an edge"),
    ("nedel", 4, 10**7, "NEDEL refers to an element"),
    ("nedsd", 0, 4, "NEDSD is not a local edge number"),
    ("needn", 0, 0, "NEEDN refers to an edge"),
    ("nledn", 3, 10**6, "NLEDN refers to an edge"),
])
def test_inconsistent_mesh_is_an_argument_error(built, scratch, table, index, value, message):
    """The drop-in create checks the host's integer mesh tables before any
    of them indexes an array (on the host, before the device is touched):
    an out-of-range id is DGSWEM_ERR_ARG with a message, not a fault."""
    path = decks.quarter_annulus(scratch / "qa_badmesh", nr=2, nth=4, nsteps=1)
    with Deck(path) as d:
        arr = getattr(d.setup.contents, table)
        old = arr[index]
        arr[index] = value
        try:
            h = C.c_void_p()
            rc = _abi.load().dgswem_cuda_create(d.setup, 0, 0, C.byref(h))
            buf = C.create_string_buffer(256)
            _abi.load().dgswem_cuda_last_error(buf, 256)
        finally:
            arr[index] = old
        assert rc == 1 and not h.value, (rc, buf.value)
        assert message in buf.value.decode()


def test_valid_meshes_pass_the_mesh_check(built, scratch):
    """create's range check accepts every kind of mesh the library reads:
    barriers (the wetdry golden deck), flow and radiation edges, p=2, a
    merged ensemble.  Without a GPU create then fails at the device query
    (DGSWEM_ERR_CUDA), with one it succeeds; never DGSWEM_ERR_ARG."""
    from conftest import golden_dir
    specs = decks.ensemble_specs(3, seed=5, ne_min=200, ne_max=600)
    members = [Deck(decks.ensemble_member(scratch / f"vm_m{i}", s["kind"], s["ne"], s["amp"], s["n_manning"],
                                          s["seed"])) for i, s in enumerate(specs)]
    paths = [golden_dir("wetdry"),
             decks.quarter_annulus(scratch / "vm_flowrad", nr=4, nth=8, nsteps=1, flow_amp=0.05, radiation=True),
             decks.quarter_annulus(scratch / "vm_p2", nr=4, nth=8, nsteps=1, rk_stage=3, rk_order=3,
                                   extra={"pl": 2, "ph": 2})]
    checked = [Deck(p) for p in paths] + [Deck.merge(members)]
    lib = _abi.load()
    for d in checked:
        h = C.c_void_p()
        rc = lib.dgswem_cuda_create(d.setup, 0, 0, C.byref(h))
        buf = C.create_string_buffer(256)
        lib.dgswem_cuda_last_error(buf, 256)
        assert rc in (0, 2), (rc, buf.value)
        if rc == 0:
            lib.dgswem_cuda_destroy(h)
        d.close()
    for m in members:
        m.close()
