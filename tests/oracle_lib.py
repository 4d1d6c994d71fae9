"""ctypes access to the CPU FP64 oracle (oracle/_build/liboracle.so).

Test infrastructure only: the oracle is the checker the CUDA path is compared
against; nothing in the dgswem_b200 package imports it.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
ORACLE_SO = ROOT / "oracle" / "_build" / "liboracle.so"
_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)
_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not ORACLE_SO.exists():
            import subprocess
            subprocess.run(["make", "-s", "-C", str(ROOT / "oracle")], check=True)
        L = C.CDLL(str(ORACLE_SO))
        L.orc_open.restype = C.c_void_p
        L.orc_open.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.orc_close.argtypes = [C.c_void_p]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_info_int.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_info_real.restype = C.c_double
        L.orc_info_real.argtypes = [C.c_void_p, C.c_char_p]
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_run.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_get_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _ip]
        L.orc_set_state.argtypes = [C.c_void_p, _dp, _dp, _dp, _ip]
        L.orc_get_hb.argtypes = [C.c_void_p, _dp]
        L.orc_get_nodecode.argtypes = [C.c_void_p, _ip]
        L.orc_modal2nodal.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_set_met.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_get_int_table.argtypes = [C.c_void_p, C.c_char_p, _ip, C.c_int]
        L.orc_get_real_table.argtypes = [C.c_void_p, C.c_char_p, _dp, C.c_int]
        L.orc_run_case.argtypes = [C.c_char_p, C.c_char_p, C.c_char_p, C.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class Oracle:
    def __init__(self, path, threads: int = 1):
        L = lib()
        L.orc_set_threads(int(threads))
        err = C.create_string_buffer(1024)
        h = L.orc_open(str(path).encode(), err, len(err))
        if not h:
            raise RuntimeError(f"oracle failed to open {path}: {err.value.decode()}")
        self.h = C.c_void_p(h)
        self.ne = self.info("ne")
        self.np = self.info("np")
        self.dofh = self.info("dofh")

    def close(self):
        if self.h:
            lib().orc_close(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def info(self, key):
        return lib().orc_info_int(self.h, key.encode())

    def info_real(self, key):
        return lib().orc_info_real(self.h, key.encode())

    def step(self, it):
        if lib().orc_step(self.h, int(it)):
            raise RuntimeError("oracle step failed")

    def run(self, it0, it1):
        if lib().orc_run(self.h, int(it0), int(it1)):
            raise RuntimeError("oracle run failed")

    def state(self):
        ze = np.empty((self.ne, self.dofh))
        qx, qy = np.empty_like(ze), np.empty_like(ze)
        wd = np.empty(self.ne, np.int32)
        lib().orc_get_state(self.h, _d(ze), _d(qx), _d(qy), _i(wd))
        return ze, qx, qy, wd

    def set_state(self, ze, qx, qy, wd):
        ze, qx, qy = (np.ascontiguousarray(a, dtype=np.float64) for a in (ze, qx, qy))
        wd = np.ascontiguousarray(wd, dtype=np.int32)
        lib().orc_set_state(self.h, _d(ze), _d(qx), _d(qy), _i(wd))

    def modal2nodal(self):
        e, u, v = (np.empty(self.np) for _ in range(3))
        lib().orc_modal2nodal(self.h, _d(e), _d(u), _d(v))
        return e, u, v

    def nodecode(self):
        nc = np.empty(self.np, np.int32)
        lib().orc_get_nodecode(self.h, _i(nc))
        return nc

    def set_met(self, wsx, wsy, pr):
        a = [np.ascontiguousarray(v, dtype=np.float64) for v in (wsx, wsy, pr)]
        lib().orc_set_met(self.h, *[_d(v) for v in a])

    def int_table(self, name):
        n = lib().orc_get_int_table(self.h, name.encode(), None, 0)
        out = np.empty(max(n, 0), np.int32)
        lib().orc_get_int_table(self.h, name.encode(), _i(out), n)
        return out

    def real_table(self, name):
        n = lib().orc_get_real_table(self.h, name.encode(), None, 0)
        out = np.empty(max(n, 0))
        lib().orc_get_real_table(self.h, name.encode(), _d(out), n)
        return out


def run_case(path, out_path):
    err = C.create_string_buffer(1024)
    rc = lib().orc_run_case(str(path).encode(), str(out_path).encode(), err, len(err))
    if rc:
        raise RuntimeError(f"oracle run failed: {err.value.decode()}")


def read_fort63(path):
    lines = [ln for ln in Path(path).read_text().split("\n") if ln.strip()]
    npn = int(lines[1].split()[1])
    its, etas = [], []
    i = 2
    while i < len(lines):
        its.append(int(lines[i].split()[1]))
        etas.append([float(ln.split()[1]) for ln in lines[i + 1:i + 1 + npn]])
        i += 1 + npn
    return np.array(its), np.array(etas)
