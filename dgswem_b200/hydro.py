"""Python host mirror of the drop-in DG hydro step.

``HydroStep`` wraps one ``dgswem_cuda`` handle: the device-resident
replacement for the reference's ``DG_HYDRO_TIMESTEP(IT)``
(src/DG_hydro_timestep.F:24) with the surrounding calls of ``DG_TIMESTEP``
(src/DG_timestep.F:11-50): ``modal2nodal`` and the state download the output
writer needs.  ``Deck`` is the standalone input path (fort.14/15/dg/13 ->
READ_INPUT + PREP_DG) that a Fortran host does not need.

State arrays use the reference's Fortran layout of one RK stage slice,
ZE(DOFH, NE): numpy shape ``(ne, dofh)`` in C order.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _abi


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


class Deck:
    """An input deck directory read by libdgswem_cuda (no GPU needed)."""

    def __init__(self, path):
        self.path = Path(path)
        self._lib = _abi.load()
        h = C.c_void_p()
        _abi.check(self._lib.dgswem_deck_open(str(self.path).encode(), C.byref(h)))
        self._h = h
        self.setup = self._lib.dgswem_deck_setup(h)

    @classmethod
    def merge(cls, decks) -> "Deck":
        """dgswem_deck_merge: one deck holding the given decks' meshes side by
        side (ensemble members in order; ids offset by the preceding
        members' counts).  The members may be closed afterwards."""
        decks = list(decks)
        lib = _abi.load()
        arr = (C.POINTER(_abi.Setup) * len(decks))(*[d.setup for d in decks])
        h = C.c_void_p()
        _abi.check(lib.dgswem_deck_merge(arr, len(decks), C.byref(h)))
        self = cls.__new__(cls)
        self.path = None
        self._lib = lib
        self._h = h
        self.setup = lib.dgswem_deck_setup(h)
        return self

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dgswem_deck_close(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def control(self, key: str) -> int:
        v = C.c_int()
        _abi.check(self._lib.dgswem_deck_int(self._h, key.encode(), C.byref(v)))
        return v.value

    @property
    def s(self) -> _abi.Setup:
        return self.setup.contents

    def int_array(self, name: str, n: int) -> np.ndarray:
        p = getattr(self.s, name)
        return np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0, np.int32)

    def real_array(self, name: str, n: int) -> np.ndarray:
        p = getattr(self.s, name)
        return np.ctypeslib.as_array(p, shape=(n,)).copy() if n else np.zeros(0)


class MetReader:
    """Host reader of an NWS = 1 fort.22 (dgswem_met_reader): each ``next()``
    is one MET_FORCING call's NP records (wsx2, wsy2, pr2) in input node
    order (met_forcing.F:49-66)."""

    def __init__(self, path, np_: int):
        self._lib = _abi.load()
        self.np = int(np_)
        h = C.c_void_p()
        _abi.check(self._lib.dgswem_met_reader_open(str(path).encode(), self.np, C.byref(h)))
        self._h = h

    def next(self):
        w = [np.empty(self.np) for _ in range(3)]
        _abi.check(self._lib.dgswem_met_reader_next(self._h, *[_dptr(a) for a in w]))
        return tuple(w)

    @property
    def calls(self) -> int:
        return int(self._lib.dgswem_met_reader_calls(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dgswem_met_reader_close(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


class HydroStep:
    """Device-resident DG hydro time step on one GPU (the drop-in for
    DG_HYDRO_TIMESTEP).  ``setup`` is a ``Deck`` or a pointer to a filled
    ``dgswem_cuda_setup``."""

    STRICT = 1  # DGSWEM_CUDA_STRICT (the default form)
    MIXED = 2   # DGSWEM_CUDA_MIXED
    FAST = 4    # DGSWEM_CUDA_FAST

    def __init__(self, setup, device: int = 0, strict: bool | None = None, part: int = 0, nparts: int = 1,
                 mixed: bool = False, fast: bool = False):
        """The kernels: strict (the default; compiled without FMA contraction,
        bit-identical to the FP64 oracle), fast (``fast=True``, or
        ``strict=False``: FMA contraction) or mixed (``mixed=True``: FP32
        edge, volume and limiter arithmetic, FP64 state, SSP combination and
        wet/dry).  nparts > 1 makes a partition handle
        (dgswem_cuda_create_part), stepped by ``PartitionedRun``."""
        self._lib = _abi.load()
        fast = bool(fast) or (strict is False and not mixed)
        if sum((bool(strict), fast, bool(mixed))) > 1:
            raise ValueError("strict, fast and mixed exclude each other")
        self.mixed = bool(mixed)
        self.fast = fast
        self.strict = not (self.mixed or self.fast)
        self._deck = setup if isinstance(setup, Deck) else None
        sp = setup.setup if isinstance(setup, Deck) else setup
        s = sp.contents
        self.ne, self.np, self.dofh, self.nrk = s.ne, s.np, s.dofh, s.nrk
        self.slopeflag = s.slopeflag
        self.part, self.nparts = int(part), int(nparts)
        h = C.c_void_p()
        flags = self.MIXED if self.mixed else (self.FAST if self.fast else 0)
        if self.nparts == 1:
            _abi.check(self._lib.dgswem_cuda_create(sp, int(device), flags, C.byref(h)))
        else:
            _abi.check(self._lib.dgswem_cuda_create_part(sp, self.part, self.nparts, int(device), flags, C.byref(h)))
        self._h = h
        self.device = int(device)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.dgswem_cuda_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- stepping -------------------------------------------------------------
    def timestep(self, it: int) -> None:
        """DG_HYDRO_TIMESTEP(IT): queue one full time step."""
        _abi.check(self._lib.dgswem_cuda_hydro_timestep(self._h, int(it)))

    def run(self, it0: int, nsteps: int) -> None:
        _abi.check(self._lib.dgswem_cuda_run(self._h, int(it0), int(nsteps)))

    def synchronize(self) -> None:
        _abi.check(self._lib.dgswem_cuda_synchronize(self._h))

    @property
    def kernel_launches(self) -> int:
        return int(self._lib.dgswem_cuda_kernel_launches(self._h))

    def set_stream(self, stream_handle: int | None) -> None:
        """Launch on a caller's cudaStream_t, used as given (0 is the CUDA
        default stream), e.g. ``torch.cuda.Stream().cuda_stream``."""
        _abi.check(self._lib.dgswem_cuda_set_stream(self._h, C.c_void_p(stream_handle or 0)))

    def set_graph(self, steps: int) -> None:
        """dgswem_cuda_set_graph: replay whole steps of ``run`` as CUDA graphs
        of ``steps`` (even) steps; 0 turns graphs off."""
        _abi.check(self._lib.dgswem_cuda_set_graph(self._h, int(steps)))

    def write_hotstart(self, path, it: int, hb=None) -> None:
        """The DG hot start of the current state at step ``it`` (write_hotstart):
        HB from this handle's deck unless given."""
        if hb is None:
            if self._deck is None:
                raise ValueError("hb is needed when the handle was not created from a Deck")
            hb = self._deck.real_array("hb", self.dofh * self.ne).reshape(self.ne, self.dofh)
        ze, qx, qy, wd = self.state()
        s = self._deck.s if self._deck is not None else None
        dtdp = s.dtdp if s is not None else 0.0
        write_hotstart(path, {3: 1, 6: 2}[self.dofh], it, dtdp, ze, qx, qy, hb, wd)

    # ---- tile / block shapes and the autotuner ----
    @staticmethod
    def shapes() -> dict:
        """dgswem_cuda_shapes: the stage tile shapes ``(elements, threads)``
        and the limiter shapes ``(threads, resident blocks per SM)`` the
        kernels are compiled for."""
        lib = _abi.load()
        nt, nl = C.c_int(), C.c_int()
        te = np.zeros(_abi.MAX_SHAPES, np.int32)
        tt = np.zeros(_abi.MAX_SHAPES, np.int32)
        lt = np.zeros(_abi.MAX_SHAPES, np.int32)
        lb = np.zeros(_abi.MAX_SHAPES, np.int32)
        _abi.check(lib.dgswem_cuda_shapes(C.byref(nt), _iptr(te), _iptr(tt), C.byref(nl), _iptr(lt), _iptr(lb)))
        return {"tile": [(int(te[i]), int(tt[i])) for i in range(nt.value)],
                "limiter": [(int(lt[i]), int(lb[i])) for i in range(nl.value)]}

    def set_shapes(self, tile: int = -1, limiter: int = -1) -> None:
        """dgswem_cuda_set_shapes: stage tile shape / limiter block by index
        into ``shapes()`` (-1 keeps the current one)."""
        _abi.check(self._lib.dgswem_cuda_set_shapes(self._h, int(tile), int(limiter)))

    def get_shapes(self) -> tuple[int, int]:
        t, l = C.c_int(), C.c_int()
        _abi.check(self._lib.dgswem_cuda_get_shapes(self._h, C.byref(t), C.byref(l)))
        return t.value, l.value

    def autotune(self, it: int = 1, steps: int = 10, reps: int = 3, cached: bool = True) -> dict:
        """dgswem_cuda_autotune: time ``steps`` steps from step ``it`` with
        every tile shape, then every limiter block, keep the fastest; the
        state is left as it was.  Returns the picked indices and the
        milliseconds per step of each shape (None: not timed)."""
        sh = self.shapes()
        mt = np.zeros(_abi.MAX_SHAPES, np.float64)
        ml = np.zeros(_abi.MAX_SHAPES, np.float64)
        flags = _abi.TUNE_CACHED if cached else 0
        _abi.check(self._lib.dgswem_cuda_autotune(self._h, int(it), int(steps), int(reps), flags, _dptr(mt),
                                                  _dptr(ml)))
        t, l = self.get_shapes()
        fix = lambda v: None if v < 0 else float(v)  # noqa: E731
        return {"tile": t, "limiter": l, "tile_shape": sh["tile"][t], "limiter_shape": sh["limiter"][l],
                "ms_tile": [fix(mt[i]) for i in range(len(sh["tile"]))],
                "ms_limiter": [fix(ml[i]) for i in range(len(sh["limiter"]))]}

    @property
    def stream_handle(self) -> int:
        return int(self._lib.dgswem_cuda_stream(self._h) or 0)

    KERNEL_KINDS = ("stage_p1", "node_minmax", "limit_wetdry", "other")

    def profile(self, enable: bool = True) -> None:
        """Start (and reset) per-kernel CUDA-event timing on the launching stream."""
        _abi.check(self._lib.dgswem_cuda_profile(self._h, int(bool(enable))))

    def profile_read(self) -> dict:
        ms = (C.c_double * 4)()
        n = (C.c_longlong * 4)()
        _abi.check(self._lib.dgswem_cuda_profile_read(self._h, ms, n))
        return {k: (float(ms[i]), int(n[i])) for i, k in enumerate(self.KERNEL_KINDS)}

    # -- state ----------------------------------------------------------------
    def state(self):
        """(ze, qx, qy, wdflg) of stage 1; ze has shape (ne, dofh).  A
        partition fills its owned elements' rows (the others are NaN / -1)."""
        ze = np.full((self.ne, self.dofh), np.nan)
        qx = np.full_like(ze, np.nan)
        qy = np.full_like(ze, np.nan)
        wd = np.full(self.ne, -1, np.int32)
        _abi.check(self._lib.dgswem_cuda_download_state(self._h, _dptr(ze), _dptr(qx), _dptr(qy), _iptr(wd)))
        return ze, qx, qy, wd

    def download_into(self, ze, qx, qy, wdflg=None) -> None:
        """Download into caller-owned (e.g. pinned) float64 / int32 buffers."""
        _abi.check(self._lib.dgswem_cuda_download_state(
            self._h, _dptr(ze), _dptr(qx), _dptr(qy), _iptr(wdflg) if wdflg is not None else None))

    def set_state(self, ze, qx, qy, wdflg=None) -> None:
        ze = np.ascontiguousarray(ze, dtype=np.float64)
        qx = np.ascontiguousarray(qx, dtype=np.float64)
        qy = np.ascontiguousarray(qy, dtype=np.float64)
        wd = None if wdflg is None else np.ascontiguousarray(wdflg, dtype=np.int32)
        _abi.check(self._lib.dgswem_cuda_upload_state(self._h, _dptr(ze), _dptr(qx), _dptr(qy),
                                                      _iptr(wd) if wd is not None else None))

    # -- partition handles (dgswem_cuda_create_part) ----------------------------
    def part_info(self) -> dict:
        v = [C.c_int() for _ in range(4)]
        _abi.check(self._lib.dgswem_cuda_part_info(self._h, *[C.byref(x) for x in v]))
        return dict(zip(("part", "nparts", "owned", "local"), (x.value for x in v)))

    TILES = {"all": 0, "interior": 1, "boundary": 2}

    def stage_rhs(self, it: int, irk: int, tiles: str = "all") -> None:
        """One stage's right-hand side and SSP update of the owned elements;
        tiles="interior" / "boundary" splits it in the two launches of
        dgswem_cuda_stage_rhs_tiles (interior first, then boundary)."""
        _abi.check(self._lib.dgswem_cuda_stage_rhs_tiles(self._h, int(it), int(irk), self.TILES[tiles]))

    def tile_split(self) -> tuple[int, int]:
        """(interior, boundary) tile counts of the stage launches."""
        a, b = C.c_int(), C.c_int()
        _abi.check(self._lib.dgswem_cuda_tile_split(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def stage_limit(self, irk: int) -> None:
        _abi.check(self._lib.dgswem_cuda_stage_limit(self._h, int(irk)))

    def step_end(self) -> None:
        _abi.check(self._lib.dgswem_cuda_step_end(self._h))

    def halo_count(self, kind: int, peer: int):
        ns, nr = C.c_int(), C.c_int()
        _abi.check(self._lib.dgswem_cuda_halo_count(self._h, int(kind), int(peer), C.byref(ns), C.byref(nr)))
        return ns.value, nr.value

    def halo_pack(self, kind: int, peer: int, irk: int, dev_ptr: int) -> None:
        _abi.check(self._lib.dgswem_cuda_halo_pack(self._h, int(kind), int(peer), int(irk), C.c_void_p(dev_ptr)))

    def halo_unpack(self, kind: int, peer: int, irk: int, dev_ptr: int) -> None:
        _abi.check(self._lib.dgswem_cuda_halo_unpack(self._h, int(kind), int(peer), int(irk), C.c_void_p(dev_ptr)))

    def met_file(self, path) -> None:
        """dgswem_cuda_met_file: read NWS = 1 fields from fort.22 before every
        RK stage, as MET_FORCING does (None detaches the file)."""
        _abi.check(self._lib.dgswem_cuda_met_file(self._h, None if path is None else str(path).encode()))

    def set_met(self, wsx2, wsy2, pr2) -> None:
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (wsx2, wsy2, pr2)]
        _abi.check(self._lib.dgswem_cuda_set_met(self._h, *[_dptr(v) for v in a]))

    def modal2nodal(self, eta_out=None):
        """(eta2, uu2, vv2, nodecode) at the nodes (write_results.F:14-170)."""
        eta = eta_out if eta_out is not None else np.empty(self.np)
        uu = np.empty(self.np)
        vv = np.empty(self.np)
        nc = np.empty(self.np, np.int32)
        _abi.check(self._lib.dgswem_cuda_modal2nodal(self._h, _dptr(eta), _dptr(uu), _dptr(vv), _iptr(nc)))
        return eta, uu, vv, nc

    def modal2nodal_noalloc(self):
        """modal2nodal through dgswem_cuda_modal2nodal_noalloc: the nodal
        scratch is the library's static device array, no device allocation."""
        eta = np.empty(self.np)
        uu = np.empty(self.np)
        vv = np.empty(self.np)
        nc = np.empty(self.np, np.int32)
        _abi.check(self._lib.dgswem_cuda_modal2nodal_noalloc(self._h, _dptr(eta), _dptr(uu), _dptr(vv),
                                                             _iptr(nc)))
        return eta, uu, vv, nc


class PartitionedRun:
    """A mesh split into ``nparts`` partition handles stepped in lock-step by
    one process, the halos moved between the handles through device buffers
    (the stage sequence of DG_hydro_timestep.F with the ghost updates of
    :493-514 and :555-579).  ``devices`` places the partitions (default: all
    on GPU 0); partitions on one device share one stream, so every pack,
    unpack and kernel of a stage is ordered without host synchronisation.
    Across devices the halo moves by peer copies with a device
    synchronisation per exchange.  A multi-process run replaces the buffer
    moves by NCCL send/receive of the same packed buffers."""

    HALO_WIDTH = (3, 10)  # doubles per element of halo kinds 0 and 1

    def __init__(self, setup, nparts: int, devices=None, strict: bool | None = None, mixed: bool = False,
                 overlap: bool = False):
        """overlap=True runs each stage after the first as two launches around
        the exchange that precedes it -- the tiles that read no ghost before
        the halo moves, the others after -- the order DistributedPartition
        uses to hide the transfer (bit-identical to the plain order)."""
        import torch
        self._torch = torch
        self.overlap = bool(overlap)
        self.nparts = int(nparts)
        self.devices = list(devices) if devices is not None else [0] * self.nparts
        if len(self.devices) != self.nparts:
            raise ValueError("one device per partition")
        self.parts = [HydroStep(setup, device=d, strict=strict, part=p, nparts=self.nparts, mixed=mixed)
                      for p, d in enumerate(self.devices)]
        self.ne, self.nrk, self.dofh = self.parts[0].ne, self.parts[0].nrk, self.parts[0].dofh
        self.slopeflag = self.parts[0].slopeflag
        self.streams = {d: torch.cuda.Stream(device=d) for d in sorted(set(self.devices))}
        for hs, d in zip(self.parts, self.devices):
            hs.set_stream(self.streams[d].cuda_stream)
        self.single_device = len(self.streams) == 1
        # per (kind, sender p, receiver q): a buffer on p's device, and on q's
        # device when they differ
        self.buf = {}
        for kind in (0, 1):
            w = self.HALO_WIDTH[kind]
            for p in range(self.nparts):
                for q in range(self.nparts):
                    if p == q:
                        continue
                    ns, _ = self.parts[p].halo_count(kind, q)
                    _, nr = self.parts[q].halo_count(kind, p)
                    if ns != nr:
                        raise RuntimeError(f"halo lists disagree: {p}->{q} sends {ns}, {q} expects {nr}")
                    if ns == 0:
                        continue
                    src = torch.empty(ns * w, dtype=torch.float64, device=f"cuda:{self.devices[p]}")
                    dst = src if self.devices[p] == self.devices[q] else \
                        torch.empty(ns * w, dtype=torch.float64, device=f"cuda:{self.devices[q]}")
                    self.buf[(kind, p, q)] = (src, dst)

    def close(self):
        for hs in self.parts:
            hs.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _exchange(self, kind: int, irk: int) -> None:
        for (k, p, q), (src, _) in self.buf.items():
            if k == kind:
                self.parts[p].halo_pack(kind, q, irk, src.data_ptr())
        if not self.single_device:
            for d in self.streams:
                self._torch.cuda.synchronize(d)
            for (k, p, q), (src, dst) in self.buf.items():
                if k == kind and dst is not src:
                    dst.copy_(src)
            for d in self.streams:
                self._torch.cuda.synchronize(d)
        for (k, p, q), (_, dst) in self.buf.items():
            if k == kind:
                self.parts[q].halo_unpack(kind, p, irk, dst.data_ptr())

    def timestep(self, it: int) -> None:
        for irk in range(1, self.nrk + 1):
            for hs in self.parts:
                hs.stage_rhs(it, irk, "boundary" if self.overlap and irk > 1 else "all")
            if self.slopeflag != 0:
                self._exchange(0, irk)
            for hs in self.parts:
                hs.stage_limit(irk)
            if self.overlap and irk < self.nrk:
                # the next stage's interior tiles before the halo moves
                for hs in self.parts:
                    hs.stage_rhs(it, irk + 1, "interior")
            self._exchange(1, irk)
        for hs in self.parts:
            hs.step_end()

    def run(self, it0: int, nsteps: int) -> None:
        for it in range(it0, it0 + nsteps):
            self.timestep(it)

    def synchronize(self) -> None:
        for hs in self.parts:
            hs.synchronize()

    def state(self):
        """(ze, qx, qy, wdflg) of the whole mesh, each partition's owned rows."""
        ze = np.full((self.ne, self.dofh), np.nan)
        qx, qy = np.full_like(ze, np.nan), np.full_like(ze, np.nan)
        wd = np.full(self.ne, -1, np.int32)
        for hs in self.parts:
            hs.download_into(ze, qx, qy, wd)
        return ze, qx, qy, wd


class DistributedPartition:
    """One partition per process (torch.distributed): rank r steps partition
    r of the group and moves its halos -- the reference's MPI ghost updates
    (messenger_elem.F:832-980, after the SSP update and after the limiter /
    WETDRY, DG_hydro_timestep.F:493-514, 555-579) -- as the packed buffers
    that ``PartitionedRun`` moves by device copies.

    transport="nccl": the device buffers go by NCCL send/receive (one GPU
    per rank, over NVLink); the handle launches on torch's current stream,
    so every pack, transfer and unpack is stream-ordered after the kernels
    that produce its data.  transport="host": the packed buffers are copied
    to pinned host buffers and moved with the group's backend (gloo) --
    for ranks that share a GPU or have no NCCL; each exchange synchronises
    the stream before sending.  Every rank issues the same sequence of
    exchanges (one per halo kind and stage); no kernel waits on another
    rank."""

    TRANSPORTS = ("nccl", "host")

    def __init__(self, setup, strict: bool | None = None, group=None, mixed: bool = False,
                 transport: str = "nccl", overlap: bool = True):
        """overlap: each stage after the first runs its tiles that read no
        ghost while the exchange before it is in flight (NCCL: on the stream,
        concurrent with the transfer; host: on the GPU while the host sends
        and receives), the others after the unpack; bit-identical to the
        plain order."""
        import torch
        import torch.distributed as dist
        if transport not in self.TRANSPORTS:
            raise ValueError(f"transport must be one of {self.TRANSPORTS}")
        self._torch, self._dist, self._group = torch, dist, group
        self.transport = transport
        self.overlap = bool(overlap)
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        dev = torch.cuda.current_device()
        self.hs = HydroStep(setup, device=dev, strict=strict, part=self.rank, nparts=self.world, mixed=mixed)
        self.hs.set_stream(torch.cuda.current_stream().cuda_stream)
        self.nrk, self.slopeflag = self.hs.nrk, self.hs.slopeflag
        self.ne = self.hs.ne
        # (kind, peer) -> (device send, device receive, nsend, nrecv, host send, host receive)
        self.buf = {}
        host = transport == "host"
        for kind in (0, 1):
            w = PartitionedRun.HALO_WIDTH[kind]
            for q in range(self.world):
                if q == self.rank:
                    continue
                ns, nr = self.hs.halo_count(kind, q)
                if ns or nr:
                    mk = lambda n, pin=False: torch.empty(max(n, 1) * w, dtype=torch.float64,  # noqa: E731
                                                          **({"pin_memory": True} if pin else {"device": dev}))
                    self.buf[(kind, q)] = (mk(ns), mk(nr), ns, nr, mk(ns, True) if host else None,
                                           mk(nr, True) if host else None)

    def close(self):
        self.hs.close()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _exchange(self, kind: int, irk: int, between=None) -> None:
        """Pack, move and unpack halo kind ``kind`` of stage buffer ``irk``;
        ``between()`` launches work that reads no ghost while the halo is in
        flight."""
        dist = self._dist
        bufs = [(q, b) for (k, q), b in sorted(self.buf.items()) if k == kind]
        for q, (snd, _, ns, _, _, _) in bufs:
            if ns:
                self.hs.halo_pack(kind, q, irk, snd.data_ptr())
        if self.transport == "nccl":
            ops = []
            for q, (snd, rcv, ns, nr, _, _) in bufs:
                if ns:
                    ops.append(dist.P2POp(dist.isend, snd, q, self._group))
                if nr:
                    ops.append(dist.P2POp(dist.irecv, rcv, q, self._group))
            reqs = dist.batch_isend_irecv(ops) if ops else []
            if between is not None:
                between()
            for req in reqs:
                req.wait()
        else:
            stream = self._torch.cuda.current_stream()
            for q, (snd, _, ns, _, hsnd, _) in bufs:
                if ns:
                    hsnd.copy_(snd, non_blocking=True)
            stream.synchronize()
            reqs = []
            for q, (_, _, ns, nr, hsnd, hrcv) in bufs:
                if ns:
                    reqs.append(dist.isend(hsnd, q, self._group))
                if nr:
                    reqs.append(dist.irecv(hrcv, q, self._group))
            if between is not None:
                between()
            for req in reqs:
                req.wait()
            for q, (_, rcv, _, nr, _, hrcv) in bufs:
                if nr:
                    rcv.copy_(hrcv, non_blocking=True)
        for q, (_, rcv, _, nr, _, _) in bufs:
            if nr:
                self.hs.halo_unpack(kind, q, irk, rcv.data_ptr())

    def timestep(self, it: int) -> None:
        for irk in range(1, self.nrk + 1):
            self.hs.stage_rhs(it, irk, "boundary" if self.overlap and irk > 1 else "all")
            if self.slopeflag != 0:
                self._exchange(0, irk)
            self.hs.stage_limit(irk)
            between = None
            if self.overlap and irk < self.nrk:
                between = (lambda nxt: lambda: self.hs.stage_rhs(it, nxt, "interior"))(irk + 1)
            self._exchange(1, irk, between)
        self.hs.step_end()

    def run(self, it0: int, nsteps: int) -> None:
        for it in range(it0, it0 + nsteps):
            self.timestep(it)

    def owned_state(self):
        """(ze, qx, qy, wdflg) in input numbering: this rank's owned
        elements' rows, the others NaN / -1."""
        return self.hs.state()


def run_case(path, out=None, device: int = 0, nsteps: int | None = None, strict: bool | None = None,
             mixed: bool = False, hot_dir=None):
    """Run a deck like the reference program (dgswem.F:341-373 time loop with
    DG_TIMESTEP and the fort.63 block of write_results.F:445-500).  NWS = 1
    reads its wind stress and pressure from the deck's fort.22 at every RK
    stage (met_forcing.F:49-66).  Returns the
    list of (it, eta2) snapshots; writes them to ``out`` when given.  A deck
    with MODAL_IC = 2 starts from its DG hot start at step ITHS + 1; with
    DGHOT = 1 the DG hot start is written (to ``hot_dir``, the deck's
    directory by default, as the reference does) every DGHOTSPOOL steps and
    at the last step (write_results.F:1197-1240)."""
    deck = Deck(path)
    nt = deck.control("nt") if nsteps is None else nsteps
    it0 = deck.control("hotstart_it") + 1 if deck.control("modal_ic") == 2 else 1
    dghot, dghotspool = deck.control("dghot"), deck.control("dghotspool")
    hot_dir = Path(path) if hot_dir is None else Path(hot_dir)
    nspool, ts, tf = deck.control("nspoolge"), deck.control("ntcysge"), deck.control("ntcyfge")
    noutge = deck.control("noutge")
    nolifa = deck.s.nolifa
    snaps = []
    with HydroStep(deck, device, strict=strict, mixed=mixed) as hs:
        if deck.s.nws == 1:
            fort22 = Path(path) / "fort.22"
            if not fort22.exists():
                raise FileNotFoundError(f"{fort22}: NWS = 1 reads the met fields from fort.22 every stage")
            hs.met_file(fort22)
        count = 0
        for it in range(it0, nt + 1):
            hs.timestep(it)
            if dghot == 1 and (it % dghotspool == 0 or it == nt):
                hs.write_hotstart(hot_dir, it)
            if noutge != 0 and ts < it <= tf:
                count += 1
                if count == nspool:
                    eta, _, _, nc = hs.modal2nodal()
                    eta = np.where(np.abs(eta) <= 1e-30, 0.0, eta)
                    if nolifa == 2:
                        eta = np.where(nc == 0, -99999.0, eta)
                    snaps.append((it, eta.copy()))
                    count = 0
        hs.synchronize()
    if out is not None:
        write_fort63(out, snaps, deck.s.np, deck.s.dtdp * nspool, nspool, deck.s.statim, deck.s.dtdp)
    deck.close()
    return snaps


def write_hotstart(path, ph: int, it: int, dtdp: float, ze, qx, qy, hb, wdflg) -> None:
    """DG hot start files in the reference's layout (write_results.F:1197-1240,
    read back by prep_DG.F:1403-1445 with MODAL_IC = 2): Hot_start.263 holds
    PH, then ZE(K,J) one per record; Hot_start.264 PH PH, then QX(K,J)
    QY(K,J); Hot_start.214 IT DTDP, then HB(K,J) WDFLG(J); records in the
    order J = 1..NE, K = 1..DOFH.  ze, qx, qy, hb: (ne, dofh) arrays; values
    with 18 significant digits (exact round trip)."""
    path = Path(path)
    path.mkdir(parents=True, exist_ok=True)
    ze, qx, qy, hb = (np.asarray(a, dtype=np.float64) for a in (ze, qx, qy, hb))
    ne, dofh = ze.shape
    with open(path / "Hot_start.263", "w") as f:
        f.write(f" {ph}\n")
        np.savetxt(f, ze.reshape(-1, 1), fmt=" %.17E")
    with open(path / "Hot_start.264", "w") as f:
        f.write(f" {ph} {ph}\n")
        np.savetxt(f, np.column_stack([qx.ravel(), qy.ravel()]), fmt=" %.17E")
    with open(path / "Hot_start.214", "w") as f:
        f.write(f" {it} {dtdp:.17E}\n")
        wd = np.repeat(np.asarray(wdflg, dtype=np.int64), dofh)
        for h, w in zip(hb.ravel(), wd):
            f.write(f" {h:.17E} {w}\n")


def write_fort63(path, snaps, np_, dt_out, nspool, statim, dtdp):
    """fort.63 in the reference's layout (write_results.F:458-500)."""
    with open(path, "w") as f:
        f.write(f"{'dgswem-b200':<32s}  {'fort.63':<24s}  {'':<24s}\n")
        f.write(f" {len(snaps):10d} {np_:10d} {dt_out:15.7E} {nspool:5d} {1:5d}\n")
        for it, eta in snaps:
            f.write(f"  {it * dtdp + statim * 86400.0:20.10E}     {it:10d}\n")
            for i, v in enumerate(eta, 1):
                f.write(f"  {i:8d}  {v:16.8E}\n")
