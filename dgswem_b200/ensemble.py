"""Batched ensembles: many independent meshes advanced by one handle.

``Ensemble`` merges the members' decks (``dgswem_deck_merge``: the meshes side
by side, ids offset) and creates one device handle on the merged setup, so
every kernel launch of a step covers all members -- 3 launches per RK stage
whatever the number of members.  Results are split back per member in the
members' own numbering.  Per-member forcing: tidal amplitudes per open-boundary
edge and Manning n per node (from each member's deck) and wind / pressure per
node (``set_met``).  The time step, RK scheme, physics switches and tidal
constituents are shared (the merge checks them).  No counterpart in the
reference, which runs one mesh per program.
"""
from __future__ import annotations

import numpy as np

from .hydro import Deck, HydroStep


class Ensemble:
    def __init__(self, decks, device: int = 0, mixed: bool = True, strict: bool | None = None):
        self.members = list(decks)
        if not self.members:
            raise ValueError("empty ensemble")
        self.ne = np.array([d.s.ne for d in self.members])
        self.np_ = np.array([d.s.np for d in self.members])
        self.elem_off = np.concatenate([[0], np.cumsum(self.ne)])
        self.node_off = np.concatenate([[0], np.cumsum(self.np_)])
        self.deck = Deck.merge(self.members)
        self.hs = HydroStep(self.deck, device=device, strict=strict, mixed=mixed)
        self.nrk = self.hs.nrk

    def __len__(self):
        return len(self.members)

    def close(self):
        if getattr(self, "hs", None) is not None:
            self.hs.close()
            self.hs = None
        if getattr(self, "deck", None) is not None:
            self.deck.close()
            self.deck = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def total_elements(self) -> int:
        return int(self.elem_off[-1])

    # -- forcing and stepping ---------------------------------------------------
    def set_met(self, wsx, wsy, pr) -> None:
        """Per-member nodal met fields (lists with one array per member, NWS=1
        kinematic stress and pressure head), concatenated in member order."""
        cat = [np.concatenate([np.asarray(a, dtype=np.float64) for a in f]) for f in (wsx, wsy, pr)]
        for a in cat:
            if a.shape != (self.node_off[-1],):
                raise ValueError("one nodal array per member, member node counts")
        self.hs.set_met(*cat)

    def timestep(self, it: int) -> None:
        self.hs.timestep(it)

    def run(self, it0: int, nsteps: int) -> None:
        self.hs.run(it0, nsteps)

    def synchronize(self) -> None:
        self.hs.synchronize()

    def autotune(self, it: int = 1, steps: int = 10, reps: int = 3, cached: bool = True) -> dict:
        """Tile and limiter block shapes for the merged mesh, timed over all
        members' whole steps (HydroStep.autotune); the states stay as they were."""
        return self.hs.autotune(it, steps, reps, cached)

    # -- results per member -------------------------------------------------------
    def _split_elems(self, arrays):
        return [tuple(a[self.elem_off[i]:self.elem_off[i + 1]] for a in arrays) for i in range(len(self))]

    def states(self):
        """[(ZE, QX, QY, WDFLG)] per member, each in the member's element numbering."""
        return self._split_elems(self.hs.state())

    def modal2nodal(self):
        """[(ETA2, UU2, VV2, NODECODE)] per member, in the member's node numbering."""
        out = self.hs.modal2nodal()
        return [tuple(a[self.node_off[i]:self.node_off[i + 1]] for a in out) for i in range(len(self))]


def _write_member(args):
    from . import decks as gen
    path, sp, nsteps = args
    gen.ensemble_member(path, sp["kind"], sp["ne"], sp["amp"], sp["n_manning"], sp["seed"], nsteps=nsteps)
    return str(path)


def make_members(root, specs, nsteps: int = 2000, workers: int = 1):
    """Write the member decks of ``decks.ensemble_specs`` under ``root`` (the
    missing ones; with ``workers`` > 1 in a spawn-started process pool) and
    open them; returns (decks, met) with met = (wsx, wsy, pr) lists of
    per-member nodal fields (uniform kinematic wind stress of each member's
    speed and direction, zero pressure)."""
    from pathlib import Path
    root = Path(root)
    paths = [root / f"member_{i:04d}" for i in range(len(specs))]
    todo = [(p, sp, nsteps) for p, sp in zip(paths, specs) if not (p / "fort.13").exists()]  # written last
    if todo and workers > 1:
        import multiprocessing as mp
        from concurrent.futures import ProcessPoolExecutor
        with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as pool:
            list(pool.map(_write_member, todo))
    else:
        for t in todo:
            _write_member(t)
    out, wsx, wsy, pr = [], [], [], []
    for path, sp in zip(paths, specs):
        d = Deck(path)
        out.append(d)
        npn = d.s.np
        t = sp["wind_pa"] / 1000.0  # kinematic stress (rho0 = 1000 kg/m^3)
        a = np.radians(sp["wind_deg"])
        wsx.append(np.full(npn, t * np.cos(a)))
        wsy.append(np.full(npn, t * np.sin(a)))
        pr.append(np.zeros(npn))
    return out, (wsx, wsy, pr)
