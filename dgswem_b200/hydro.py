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


class HydroStep:
    """Device-resident DG hydro time step on one GPU (the drop-in for
    DG_HYDRO_TIMESTEP).  ``setup`` is a ``Deck`` or a pointer to a filled
    ``dgswem_cuda_setup``."""

    STRICT = 1  # DGSWEM_CUDA_STRICT

    def __init__(self, setup, device: int = 0, strict: bool = False):
        """strict=True selects the kernels compiled without FMA contraction
        (bitwise reproducible against the non-contracting FP64 oracle);
        the default is the FMA-contracted fast form."""
        self._lib = _abi.load()
        self.strict = bool(strict)
        self._deck = setup if isinstance(setup, Deck) else None
        sp = setup.setup if isinstance(setup, Deck) else setup
        s = sp.contents
        self.ne, self.np, self.dofh, self.nrk = s.ne, s.np, s.dofh, s.nrk
        h = C.c_void_p()
        flags = self.STRICT if strict else 0
        _abi.check(self._lib.dgswem_cuda_create(sp, int(device), flags, C.byref(h)))
        self._h = h

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
        """(ze, qx, qy, wdflg) of stage 1; ze has shape (ne, dofh)."""
        ze = np.empty((self.ne, self.dofh))
        qx = np.empty_like(ze)
        qy = np.empty_like(ze)
        wd = np.empty(self.ne, np.int32)
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


def run_case(path, out=None, device: int = 0, nsteps: int | None = None, strict: bool = False):
    """Run a deck like the reference program (dgswem.F:341-373 time loop with
    DG_TIMESTEP and the fort.63 block of write_results.F:445-500).  Returns the
    list of (it, eta2) snapshots; writes them to ``out`` when given."""
    deck = Deck(path)
    nt = deck.control("nt") if nsteps is None else nsteps
    nspool, ts, tf = deck.control("nspoolge"), deck.control("ntcysge"), deck.control("ntcyfge")
    noutge = deck.control("noutge")
    nolifa = deck.s.nolifa
    snaps = []
    with HydroStep(deck, device, strict=strict) as hs:
        count = 0
        for it in range(1, nt + 1):
            hs.timestep(it)
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


def write_fort63(path, snaps, np_, dt_out, nspool, statim, dtdp):
    """fort.63 in the reference's layout (write_results.F:458-500)."""
    with open(path, "w") as f:
        f.write(f"{'dgswem-b200':<32s}  {'fort.63':<24s}  {'':<24s}\n")
        f.write(f" {len(snaps):10d} {np_:10d} {dt_out:15.7E} {nspool:5d} {1:5d}\n")
        for it, eta in snaps:
            f.write(f"  {it * dtdp + statim * 86400.0:20.10E}     {it:10d}\n")
            for i, v in enumerate(eta, 1):
                f.write(f"  {i:8d}  {v:16.8E}\n")
