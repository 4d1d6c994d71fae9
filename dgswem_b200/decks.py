"""Synthetic DG-SWEM input decks (fort.14 / fort.15 / fort.dg / fort.13).

The meshes follow the fort.14 conventions of the reference's mesh generator
(tests/slopingbeach/slopingbeach.py) and its test decks: counter-clockwise
elements, an open (elevation) boundary segment, land segments of type 0.

* ``quarter_annulus``: r in [60.96, 152.4] km, theta in [0, pi/2], nr x nth
  cells split into triangles, h = 3.048 (r / 60.96 km)^2 m, M2 forcing on the
  outer arc, land walls elsewhere, linear friction.
* ``sloping_beach``: Lx x Ly rectangle, right-triangle split, depth linear
  from 20 m offshore to -2 m (dry land) plus seeded Gaussian noise, M2 forcing
  on the offshore edge, nodal Manning n = 0.025 +-20 % (fort.13), wetting and
  drying, slope limiter 5.

Nodes and elements are numbered column by column along the short side, so
edge neighbours sit a few hundred entries apart in every array.
"""
from __future__ import annotations

import io
import math
import os
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

M2_OMEGA = 1.405257e-4  # 1/s, period 44712 s


@dataclass
class Controls:
    """fort.15 / fort.dg fields the hydro path reads."""

    title: str = "dgswem-b200 synthetic"
    ics: int = 1
    nolibf: int = 0
    nolifa: int = 1
    nolica: int = 1
    nolicat: int = 1
    nws: int = 0
    nramp: int = 1
    g: float = 9.81
    dt: float = 10.0
    nsteps: int = 100
    dramp: float = 1.0
    h0: float = 0.01
    slam0: float = 0.0
    sfea0: float = 0.0
    tau: float = 1e-4
    cf: float = 0.0025
    hbreak: float = 1.0
    ftheta: float = 10.0
    fgamma: float = 1.0 / 3.0
    cori: float = 0.0
    amig: float = M2_OMEGA
    nspoolge: int = 0
    rk_stage: int = 2
    rk_order: int = 2
    slopeflag: int = 0
    rainfall: int = 0
    manning: bool = False
    extra: dict = field(default_factory=dict)


def _fmt(v: float) -> str:
    return repr(float(v))


def _savetxt_chunk(args) -> str:
    arr, fmt = args
    buf = io.StringIO()
    np.savetxt(buf, arr, fmt=fmt)
    return buf.getvalue()


def _savetxt(f, arr, fmt, rows_per_chunk: int = 250_000) -> None:
    """np.savetxt of ``arr`` into ``f``; tables of more than a million rows
    are formatted in chunks on spawned worker processes (the same text)."""
    n = len(arr)
    workers = min(16, os.cpu_count() or 1)
    if n <= 1_000_000 or workers < 2:
        np.savetxt(f, arr, fmt=fmt)
        return
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    chunks = [(arr[i:i + rows_per_chunk], fmt) for i in range(0, n, rows_per_chunk)]
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as pool:
        for text in pool.map(_savetxt_chunk, chunks):
            f.write(text)


def write_deck(path, x, y, dp, elems, open_segs, land_segs, ctl: Controls, emo=None, efa=None,
               manning=None, flow=None):
    """Write fort.14, fort.15, fort.dg (and fort.13 when ``manning`` is given).

    elems: (ne, 3) 1-based counter-clockwise connectivity.  open_segs: list of
    1-based node arrays.  land_segs: list of (node array, ibtype).  flow: for
    periodic flux boundaries (ibtype 2/12/22), (frequency, nodal factor,
    equilibrium argument in degrees, amplitudes, phases in degrees) with one
    amplitude and phase per flux-boundary node, in boundary order."""
    path = Path(path)
    path.mkdir(parents=True, exist_ok=True)
    npn, ne = len(x), len(elems)
    ids = np.arange(1, npn + 1)
    with open(path / "fort.14", "w") as f:
        f.write(f"{ctl.title}\n{ne} {npn}\n")
        _savetxt(f, np.column_stack([ids, x, y, dp]), fmt=["%d", "%.10f", "%.10f", "%.10f"])
        _savetxt(f, np.column_stack([np.arange(1, ne + 1), np.full(ne, 3), elems]), fmt="%d")
        neta = sum(len(s) for s in open_segs)
        f.write(f"{len(open_segs)} ! NOPE\n{neta} ! NETA\n")
        for s in open_segs:
            f.write(f"{len(s)}\n")
            np.savetxt(f, np.asarray(s)[:, None], fmt="%d")
        nvel = sum(len(s) for s, _ in land_segs)
        f.write(f"{len(land_segs)} ! NBOU\n{nvel} ! NVEL\n")
        for s, ib in land_segs:
            f.write(f"{len(s)} {ib}\n")
            np.savetxt(f, np.asarray(s)[:, None], fmt="%d")
    neta = sum(len(s) for s in open_segs)
    if emo is None:
        emo = np.zeros(neta)
    if efa is None:
        efa = np.zeros(neta)
    nwp = 1 if manning is not None else 0
    nt = ctl.nsteps
    rnday = nt * ctl.dt / 86400.0
    nspool = ctl.nspoolge if ctl.nspoolge > 0 else max(nt, 1)
    lines = [
        ctl.title[:32], "dgswem-b200", "1 ! NFOVER", "1 ! NABOUT", "0 ! NSCREEN", "0 ! IHOT",
        f"{ctl.ics} ! ICS", "0 ! IM", f"{ctl.nolibf} ! NOLIBF", f"{ctl.nolifa} ! NOLIFA",
        f"{ctl.nolica} ! NOLICA", f"{ctl.nolicat} ! NOLICAT", f"{nwp} ! NWP",
    ]
    if nwp:
        lines.append("mannings_n_at_sea_floor")
    lines += [
        "0 ! NCOR", "0 ! NTIP", f"{ctl.nws} ! NWS", f"{ctl.nramp} ! NRAMP", f"{_fmt(ctl.g)} ! G",
        "0.005 ! TAU0", f"{_fmt(ctl.dt)} ! DT", "0.0 ! STATIM", "0.0 ! REFTIM", f"{_fmt(rnday)} ! RNDAY",
        f"{_fmt(ctl.dramp)} ! DRAMP", "0.35 0.30 0.35 ! A00 B00 C00",
    ]
    lines.append(f"{_fmt(ctl.h0)} 0 0 0.01 ! H0" if ctl.nolifa == 2 else f"{_fmt(ctl.h0)} ! H0")
    lines.append(f"{_fmt(ctl.slam0)} {_fmt(ctl.sfea0)} ! SLAM0 SFEA0")
    if ctl.nolibf == 0:
        lines.append(f"{_fmt(ctl.tau)} ! TAU")
    elif ctl.nolibf == 1:
        lines.append(f"{_fmt(ctl.cf)} ! CF")
    else:
        lines.append(f"{_fmt(ctl.cf)} {_fmt(ctl.hbreak)} {_fmt(ctl.ftheta)} {_fmt(ctl.fgamma)} ! CF HBREAK FTHETA FGAMMA")
    lines += ["0.0 ! ESLM", f"{_fmt(ctl.cori)} ! CORI", "0 ! NTIF"]
    nbfr = 1 if neta else 0
    lines.append(f"{nbfr} ! NBFR")
    if nbfr:
        lines += ["M2", f"{_fmt(ctl.amig)} 1.0 0.0", "M2"]
        lines += [f"{_fmt(a)} {_fmt(p)}" for a, p in zip(emo, efa)]
    lines += ["110.0 ! ANGINN"]
    if flow is not None:  # periodic flux boundary forcing (read_input.F:2971-3045)
        w, ffac, face, famp, fph = flow
        lines += ["1 ! NFFR", "FLOW", f"{_fmt(w)} {_fmt(ffac)} {_fmt(face)}", "FLOW"]
        lines += [f"{_fmt(a)} {_fmt(ph)}" for a, ph in zip(famp, fph)]
    lines += ["0 0.0 1.0 1 ! NOUTE", "0 ! NSTAE", "0 0.0 1.0 1 ! NOUTV", "0 ! NSTAV"]
    if ctl.nws != 0:
        lines += ["0 0.0 1.0 1 ! NOUTM", "0 ! NSTAM"]
    lines += [f"1 0.0 {_fmt(rnday + 1.0)} {nspool} ! NOUTGE", "0 0.0 1.0 1 ! NOUTGV", "0 ! NFREQ",
              "0.0 1.0 1 0.0 ! THAS", "0 0 0 0 ! NHASE", "0 1000000 ! NHSTAR", "1 0 1.E-10 25 ! ITITER"]
    (path / "fort.15").write_text("\n".join(lines) + "\n")
    dg = {
        "dgswe": 1, "pl": 1, "ph": 1, "px": 1, "fluxtype": 2, "rk_stage": ctl.rk_stage,
        "rk_order": ctl.rk_order, "modal_ic": 0, "dghot": 0, "dghotspool": 86400,
        "slopeflag": ctl.slopeflag, "artdif": 0, "sedflag": 0, "rainfall": ctl.rainfall,
    }
    dg.update(ctl.extra)
    (path / "fort.dg").write_text("! dgswem-b200 synthetic deck\n" +
                                  "".join(f"{k} = {v}\n" for k, v in dg.items()))
    if manning is not None:
        with open(path / "fort.13", "w") as f:
            f.write(f"{ctl.title}\n{npn}\n1\nmannings_n_at_sea_floor\nunitless\n1\n0.025\n")
            f.write(f"mannings_n_at_sea_floor\n{npn}\n")
            np.savetxt(f, np.column_stack([ids, manning]), fmt=["%d", "%.10f"])
    return path


def write_fort22(path, blocks) -> Path:
    """fort.22 of NWS = 1 (met_forcing.F:49-66): for each MET_FORCING call
    (one per RK stage of every step, in order) a block of NP records
    "NHG WSX2 WSY2 PR2"; ``blocks`` yields (wsx2, wsy2, pr2) arrays of NP
    values in input node order.  Values with 17 significant digits (exact
    round trip)."""
    path = Path(path)
    with open(path, "w") as f:
        for wsx, wsy, pr in blocks:
            n = len(wsx)
            _savetxt(f, np.column_stack([np.arange(1, n + 1), wsx, wsy, pr]),
                     fmt=["%d", "%.17E", "%.17E", "%.17E"])
    return path


def _grid_triangles(ni: int, nj: int) -> np.ndarray:
    """Node (i, j) -> i*(nj+1) + j + 1; two CCW triangles per cell, ordered
    column by column (j fastest)."""
    i, j = np.meshgrid(np.arange(ni), np.arange(nj), indexing="ij")
    a = (i * (nj + 1) + j + 1).ravel()
    b = ((i + 1) * (nj + 1) + j + 1).ravel()
    c = ((i + 1) * (nj + 1) + j + 2).ravel()
    d = (i * (nj + 1) + j + 2).ravel()
    t1 = np.stack([a, b, c], 1)
    t2 = np.stack([a, c, d], 1)
    return np.stack([t1, t2], 1).reshape(-1, 3)


def quarter_annulus(path, nr: int = 16, nth: int = 32, amp: float = 0.3048, flow_amp: float | None = None,
                    radiation: bool = False, **kw) -> Path:
    """Tidal quarter annulus (the reference's quarter_annular geometry).

    flow_amp: make the radial side at 90 degrees a periodic flux boundary
    (ibtype 2) with normal flux amplitude flow_amp (m^2/s) at the tide's
    frequency; radiation: make the inner arc a radiation boundary (ibtype 30).
    Otherwise both are land (ibtype 0)."""
    ctl = Controls(title="quarter annulus", nolibf=0, nolifa=1, tau=1e-4, dt=10.0, nsteps=4460,
                   rk_stage=2, rk_order=2, slopeflag=0, h0=1.0, nramp=1, dramp=2.0)
    for k, v in kw.items():
        setattr(ctl, k, v)
    r0, r1 = 60960.0, 152400.0
    r = np.linspace(r0, r1, nr + 1)
    th = np.linspace(0.0, 0.5 * math.pi, nth + 1)
    R, T = np.meshgrid(r, th, indexing="ij")
    x = (R * np.cos(T)).ravel()
    y = (R * np.sin(T)).ravel()
    dp = (3.048 * (R / r0) ** 2).ravel()
    x[np.abs(x) < 1e-6] = 0.0
    elems = _grid_triangles(nr, nth)
    nid = lambda i, j: i * (nth + 1) + j + 1  # noqa: E731
    ocean = [nid(nr, j) for j in range(nth + 1)]
    if flow_amp is None and not radiation:
        land = [nid(i, nth) for i in range(nr, -1, -1)] + [nid(0, j) for j in range(nth - 1, -1, -1)] + \
               [nid(i, 0) for i in range(1, nr + 1)]
        return write_deck(path, x, y, dp, elems, [ocean], [(land, 0)], ctl,
                          emo=np.full(len(ocean), amp), efa=np.zeros(len(ocean)))
    top = [nid(i, nth) for i in range(nr, -1, -1)]
    inner = [nid(0, j) for j in range(nth, -1, -1)]
    bottom = [nid(i, 0) for i in range(0, nr + 1)]
    segs = [(top, 2 if flow_amp is not None else 0), (inner, 30 if radiation else 0), (bottom, 0)]
    flow = None
    if flow_amp is not None:
        flow = (ctl.amig, 1.0, 0.0, np.full(len(top), flow_amp), np.zeros(len(top)))
    return write_deck(path, x, y, dp, elems, [ocean], segs, ctl,
                      emo=np.full(len(ocean), amp), efa=np.zeros(len(ocean)), flow=flow)


def sloping_beach(path, nx: int = 2236, ny: int = 447, lx: float = 100e3, ly: float = 20e3,
                  seed: int = 20261203, amp: float = 1.0, **kw) -> Path:
    """Wet/dry sloping beach basin with a seeded rough bed and Manning n."""
    ctl = Controls(title="sloping beach", nolibf=1, nolifa=2, cf=0.0025, dt=0.5, nsteps=2000,
                   rk_stage=2, rk_order=2, slopeflag=5, h0=0.01, nramp=1, dramp=1.0, manning=True)
    for k, v in kw.items():
        setattr(ctl, k, v)
    rng = np.random.default_rng(seed)
    xs = np.linspace(0.0, lx, nx + 1)
    ys = np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    dp = 20.0 + (-2.0 - 20.0) * X / lx + rng.normal(0.0, 0.05, X.shape)
    elems = _grid_triangles(nx, ny)
    nid = lambda i, j: i * (ny + 1) + j + 1  # noqa: E731
    ocean = [nid(0, j) for j in range(ny, -1, -1)]
    land = [nid(i, 0) for i in range(0, nx + 1)] + [nid(nx, j) for j in range(1, ny + 1)] + \
           [nid(i, ny) for i in range(nx - 1, -1, -1)]
    manning = 0.025 * rng.uniform(0.8, 1.2, X.size)
    return write_deck(path, X.ravel(), Y.ravel(), dp.ravel(), elems, [ocean], [(land, 0)], ctl,
                      emo=np.full(len(ocean), amp), efa=np.zeros(len(ocean)), manning=manning)


# ---- batched ensembles -------------------------------------------------------
ENSEMBLE_KINDS = ("rectangle", "annulus")


def ensemble_member(path, kind: str, ne: int, amp: float, n_manning: float, seed: int, dt: float = 0.5,
                    nsteps: int = 2000) -> Path:
    """One member of a batched ensemble, about ``ne`` elements: a 20 x 4 km
    rectangular basin sloping from 20 m to -2 m (wet/dry shore, seeded
    0.05 m bed noise; kind "rectangle") or the quarter annulus of the
    reference's tidal test (kind "annulus").  Tidal amplitude ``amp`` (m) on
    the open boundary, uniform nodal Manning n.  All members share what a
    merged ensemble requires to be common: Manning friction, WETDRY, slope
    limiter 5, NWS=1 (nodal met fields set per member at run time),
    SSP(2,2), H0 = 0.01 m and the time step (0.5 s is stable for the finest
    200k-element members of either kind)."""
    ctl = Controls(title=f"ensemble {kind}", nolibf=1, nolifa=2, cf=0.0025, dt=dt, nsteps=nsteps, rk_stage=2,
                   rk_order=2, slopeflag=5, h0=0.01, nramp=1, dramp=1.0, manning=True, nws=1)
    rng = np.random.default_rng(seed)
    if kind == "rectangle":
        nx = max(5, int(round(math.sqrt(ne * 5 / 2))))
        ny = max(1, int(round(ne / (2 * nx))))
        lx, ly = 20e3, 4e3
        xs, ys = np.linspace(0.0, lx, nx + 1), np.linspace(0.0, ly, ny + 1)
        X, Y = np.meshgrid(xs, ys, indexing="ij")
        dp = 20.0 + (-2.0 - 20.0) * X / lx + rng.normal(0.0, 0.05, X.shape)
        elems = _grid_triangles(nx, ny)
        nid = lambda i, j: i * (ny + 1) + j + 1  # noqa: E731
        ocean = [nid(0, j) for j in range(ny, -1, -1)]
        land = [nid(i, 0) for i in range(0, nx + 1)] + [nid(nx, j) for j in range(1, ny + 1)] + \
               [nid(i, ny) for i in range(nx - 1, -1, -1)]
        x, y, dp = X.ravel(), Y.ravel(), dp.ravel()
    elif kind == "annulus":
        nr = max(2, int(round(math.sqrt(ne / 4))))
        nth = max(2, int(round(ne / (2 * nr))))
        r0, r1 = 60960.0, 152400.0
        R, T = np.meshgrid(np.linspace(r0, r1, nr + 1), np.linspace(0.0, 0.5 * math.pi, nth + 1), indexing="ij")
        x, y = (R * np.cos(T)).ravel(), (R * np.sin(T)).ravel()
        x[np.abs(x) < 1e-6] = 0.0
        dp = (3.048 * (R / r0) ** 2).ravel()
        elems = _grid_triangles(nr, nth)
        nid = lambda i, j: i * (nth + 1) + j + 1  # noqa: E731
        ocean = [nid(nr, j) for j in range(nth + 1)]
        land = [nid(i, nth) for i in range(nr, -1, -1)] + [nid(0, j) for j in range(nth - 1, -1, -1)] + \
               [nid(i, 0) for i in range(1, nr + 1)]
    else:
        raise ValueError(f"unknown ensemble member kind {kind!r}")
    return write_deck(path, x, y, dp, elems, [ocean], [(land, 0)], ctl, emo=np.full(len(ocean), amp),
                      efa=np.zeros(len(ocean)), manning=np.full(len(x), n_manning))


def ensemble_specs(n: int, seed: int = 20261203, ne_min: int = 5000, ne_max: int = 200000) -> list:
    """Seeded member parameters of the batched configuration: element counts
    log-uniform in [ne_min, ne_max], rectangle or quarter annulus, tidal
    amplitude U[0.2, 2] m, Manning n U[0.015, 0.04], wind stress U[0, 0.3] Pa
    (direction U[0, 360) degrees)."""
    rng = np.random.default_rng(seed)
    ne = np.exp(rng.uniform(math.log(ne_min), math.log(ne_max), n)).astype(int)
    kinds = rng.integers(0, 2, n)
    amp = rng.uniform(0.2, 2.0, n)
    nman = rng.uniform(0.015, 0.04, n)
    wind = rng.uniform(0.0, 0.3, n)
    wdir = rng.uniform(0.0, 360.0, n)
    return [dict(kind=ENSEMBLE_KINDS[int(kinds[i])], ne=int(ne[i]), amp=float(amp[i]), n_manning=float(nman[i]),
                 wind_pa=float(wind[i]), wind_deg=float(wdir[i]), seed=seed + 1 + i) for i in range(n)]


def smooth_basin(path, nx: int = 158, ny: int = 32, lx: float = 20e3, ly: float = 4e3, amp: float = 0.5,
                 n0: float = 0.025, dt: float = 1.0, nsteps: int = 100, **kw) -> Path:
    """Always-wet rectangular basin with smooth fields, for gradient checks:
    depth 20 m at the open (x = 0) edge to 5 m at the far wall plus a smooth
    Gaussian shoal, nodal Manning n = n0 (1 + 0.2 sin) varying smoothly,
    quadratic friction with the Manning floor CF = 1e-4 (below every
    element's Manning coefficient, so no element sits on it), no WETDRY, no slope limiter, SSP(2,2), tide of
    amplitude ``amp`` on the open edge, land elsewhere."""
    ctl = Controls(title="smooth basin", nolibf=1, nolifa=1, cf=1e-4, dt=dt, nsteps=nsteps, rk_stage=2, rk_order=2,
                   slopeflag=0, h0=0.01, nramp=1, dramp=0.05, manning=True)
    for k, v in kw.items():
        setattr(ctl, k, v)
    xs, ys = np.linspace(0.0, lx, nx + 1), np.linspace(0.0, ly, ny + 1)
    X, Y = np.meshgrid(xs, ys, indexing="ij")
    dp = 20.0 - 15.0 * X / lx - 3.0 * np.exp(-(((X - 0.6 * lx) / (0.1 * lx)) ** 2 + ((Y - 0.5 * ly) / (0.2 * ly)) ** 2))
    elems = _grid_triangles(nx, ny)
    nid = lambda i, j: i * (ny + 1) + j + 1  # noqa: E731
    ocean = [nid(0, j) for j in range(ny, -1, -1)]
    land = [nid(i, 0) for i in range(0, nx + 1)] + [nid(nx, j) for j in range(1, ny + 1)] + \
           [nid(i, ny) for i in range(nx - 1, -1, -1)]
    manning = n0 * (1.0 + 0.2 * np.sin(2 * math.pi * X / lx) * np.cos(math.pi * Y / ly))
    return write_deck(path, X.ravel(), Y.ravel(), dp.ravel(), elems, [ocean], [(land, 0)], ctl,
                      emo=np.full(len(ocean), amp), efa=np.zeros(len(ocean)), manning=manning.ravel())
