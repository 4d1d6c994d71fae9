"""Gradients of a gauge misfit through the discrete adjoint of the DG hydro step.

J = sum over steps k = 1..N and gauges g of (ZE at gauge g after step k -
obs[k-1, g])**2, a function of the element-mean Manning n (``nbar``, one per
element) and the bathymetry modes (``hb``, HB(3, NE) as an (NE, 3) array).

``GaugeMisfitProblem.forward`` runs the N steps from the initial state and
keeps revolve-style checkpoints: the state every C = ceil(sqrt(N)) steps
(``dgswem_cuda_misfit_forward``).  ``gradient`` sweeps back segment by
segment (``dgswem_cuda_adjoint_sweep``): it reloads a checkpoint, re-runs the
segment keeping its (at most C) step states and RK stage states, then walks
the steps backwards, seeding the misfit's derivative at each step's state and
carrying the cotangent back through the step's stages.  Device memory: about
sqrt(N) checkpoints plus NRK*sqrt(N) states of one segment.  ``GaugeMisfit``
wraps both as a ``torch.autograd.Function``.

No counterpart in the reference.  The adjoint covers NLEQ=1, ICS=1, land and
ocean edges, linear / quadratic / Manning friction, slope limiter 5 and WETDRY
with their branches frozen at the forward's (``dgswem_cuda_adjoint_begin``
rejects the rest).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _abi
from .hydro import Deck, HydroStep

# p=1 corner map: ZE at vertex v = m1 + PC[v][1] m2 + PC[v][2] m3
# (inverse of m1=(v1+v2+v3)/3, m2=-(v1+v2)/6+v3/3, m3=(-v1+v2)/2)
PC = np.array([[1.0, -1.0, -1.0], [1.0, -1.0, 1.0], [1.0, 2.0, 0.0]])


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def locate_gauges(deck: Deck, xy) -> tuple[np.ndarray, np.ndarray]:
    """Element (1-based) and ZE basis values (ng, 3) of each gauge point:
    the element containing it, and 1 plus the corner-map combinations of its
    barycentric weights (ZE is linear on an element at p=1)."""
    s = deck.s
    ne = s.ne
    nm = deck.int_array("nm", 3 * ne).reshape(3, ne) - 1
    x, y = deck.real_array("x", s.np), deck.real_array("y", s.np)
    xa, xb, xc = x[nm[0]], x[nm[1]], x[nm[2]]
    ya, yb, yc = y[nm[0]], y[nm[1]], y[nm[2]]
    det = (yb - yc) * (xa - xc) + (xc - xb) * (ya - yc)
    elem, phi = [], []
    for px, py in np.asarray(xy, dtype=np.float64):
        l1 = ((yb - yc) * (px - xc) + (xc - xb) * (py - yc)) / det
        l2 = ((yc - ya) * (px - xc) + (xa - xc) * (py - yc)) / det
        l3 = 1.0 - l1 - l2
        inside = np.nonzero((l1 >= -1e-12) & (l2 >= -1e-12) & (l3 >= -1e-12))[0]
        if len(inside) == 0:
            raise ValueError(f"gauge ({px}, {py}) lies in no element")
        e = int(inside[0])
        lam = np.array([l1[e], l2[e], l3[e]])
        elem.append(e + 1)
        phi.append(lam @ PC)
    return np.array(elem, dtype=np.int32), np.array(phi)


def element_manning(deck: Deck) -> np.ndarray:
    """Element mean of the nodal Manning n, the value the friction uses."""
    s = deck.s
    nm = deck.int_array("nm", 3 * s.ne).reshape(3, s.ne) - 1
    n = deck.real_array("manning", s.np)
    return (n[nm[0]] + n[nm[1]] + n[nm[2]]) / 3.0


class GaugeMisfitProblem:
    def __init__(self, deck: Deck, gauge_elem, gauge_phi, nsteps: int, obs=None, it0: int = 1, device: int = 0,
                 met=None, checkpoint_every: int | None = None):
        self.deck = deck
        self.hs = HydroStep(deck, device=device)
        self._lib = self.hs._lib
        self.nsteps, self.it0 = int(nsteps), int(it0)
        self.elem = np.ascontiguousarray(gauge_elem, dtype=np.int32)
        self.phi = np.ascontiguousarray(gauge_phi, dtype=np.float64).reshape(-1, 3)
        self.ng = len(self.elem)
        _abi.check(self._lib.dgswem_cuda_gauges(self.hs._h, self.ng, _ip(self.elem), _dp(self.phi.ravel())))
        if met is not None:
            self.hs.set_met(*met)
        self.obs = None if obs is None else np.asarray(obs, dtype=np.float64).reshape(self.nsteps, self.ng)
        self.C = checkpoint_every or max(1, math.ceil(math.sqrt(self.nsteps)))
        self.n_outer = (self.nsteps + self.C - 1) // self.C
        # slot 0: the initial state (and the first checkpoint); the forward's
        # checkpoints and the sweep's segment states follow
        _abi.check(self._lib.dgswem_cuda_state_save(self.hs._h, 0))
        self.eta = None

    def close(self):
        self.hs.close()

    def set_params(self, nbar=None, hb=None) -> None:
        nb = None if nbar is None else np.ascontiguousarray(nbar, dtype=np.float64)
        h = None if hb is None else np.ascontiguousarray(hb, dtype=np.float64).reshape(-1)
        _abi.check(self._lib.dgswem_cuda_set_params(self.hs._h, None if nb is None else _dp(nb),
                                                    None if h is None else _dp(h)))

    def _gauge_eta(self) -> np.ndarray:
        out = np.empty(self.ng)
        _abi.check(self._lib.dgswem_cuda_gauge_eta(self.hs._h, _dp(out)))
        return out

    def run(self) -> np.ndarray:
        """The N steps from the initial state (dgswem_cuda_misfit_forward:
        checkpoints every C steps in slots 0, 1, ..); ZE at the gauges after
        each step, (N, ng)."""
        lib, h = self._lib, self.hs._h
        _abi.check(lib.dgswem_cuda_state_load(h, 0))
        eta = np.empty(self.nsteps * self.ng)
        _abi.check(lib.dgswem_cuda_misfit_forward(h, self.it0, self.nsteps, self.C, _dp(eta)))
        self.eta = eta.reshape(self.nsteps, self.ng)
        return self.eta

    def forward(self) -> float:
        eta = self.run()
        if self.obs is None:
            raise ValueError("no observations")
        return float(np.sum((eta - self.obs) ** 2))

    def _residual(self) -> np.ndarray:
        if self.eta is None or self.obs is None:
            raise ValueError("run forward first")
        return np.ascontiguousarray(2.0 * (self.eta - self.obs))

    def _read(self):
        ne = self.hs.ne
        gn, ghb = np.empty(ne), np.empty(3 * ne)
        _abi.check(self._lib.dgswem_cuda_adjoint_read(self.hs._h, _dp(gn), _dp(ghb), None, None, None))
        return gn, ghb.reshape(ne, 3)

    def gradient(self):
        """(dJ/dnbar (NE,), dJ/dHB (NE, 3)) at the parameters of the last
        forward (dgswem_cuda_adjoint_sweep)."""
        w = self._residual().ravel()
        _abi.check(self._lib.dgswem_cuda_adjoint_sweep(self.hs._h, self.it0, self.nsteps, self.C, _dp(w)))
        return self._read()

    def gradient_stepwise(self):
        """The same gradient through the step-wise entry points (state slots,
        dgswem_cuda_adjoint_seed / _step), as a host that keeps its own
        checkpoints would drive them: per segment, the states from the
        checkpoint are re-run and saved, then each step is recomputed and
        reversed."""
        lib, h = self._lib, self.hs._h
        resid = self._residual()
        _abi.check(lib.dgswem_cuda_adjoint_begin(h))
        base = 2 * self.n_outer + self.C  # slots above those of the sweep
        for seg in range(self.n_outer - 1, -1, -1):
            k0, k1 = seg * self.C, min((seg + 1) * self.C, self.nsteps)
            _abi.check(lib.dgswem_cuda_state_load(h, seg))
            for k in range(k0, k1):
                _abi.check(lib.dgswem_cuda_state_save(h, base + (k - k0)))
                if k + 1 < k1:
                    self.hs.timestep(self.it0 + k)
            for k in range(k1, k0, -1):  # step k maps state k-1 to state k
                w = np.ascontiguousarray(resid[k - 1])
                _abi.check(lib.dgswem_cuda_adjoint_seed(h, _dp(w)))
                _abi.check(lib.dgswem_cuda_state_load(h, base + (k - 1 - k0)))
                _abi.check(lib.dgswem_cuda_adjoint_step(h, self.it0 + k - 1))
        return self._read()


def _torch_function():
    import torch

    class GaugeMisfit(torch.autograd.Function):
        """J(nbar, hb) of a ``GaugeMisfitProblem``; backward runs the discrete
        adjoint.  nbar: (NE,) float64; hb: (NE, 3) float64."""

        @staticmethod
        def forward(ctx, nbar, hb, problem):
            problem.set_params(nbar.detach().cpu().numpy(), hb.detach().cpu().numpy())
            j = problem.forward()
            ctx.problem = problem
            ctx.dev = nbar.device
            return torch.tensor(j, dtype=torch.float64, device=nbar.device)

        @staticmethod
        def backward(ctx, gj):
            gn, ghb = ctx.problem.gradient()
            gn = torch.from_numpy(gn).to(ctx.dev) * gj
            ghb = torch.from_numpy(ghb).to(ctx.dev) * gj
            return gn, ghb, None

    return GaugeMisfit


_GAUGE_MISFIT = None


def __getattr__(name):
    # GaugeMisfit is built on first use so that importing this module does not
    # import torch
    global _GAUGE_MISFIT
    if name == "GaugeMisfit":
        if _GAUGE_MISFIT is None:
            _GAUGE_MISFIT = _torch_function()
        return _GAUGE_MISFIT
    raise AttributeError(name)
