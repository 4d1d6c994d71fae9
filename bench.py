#!/usr/bin/env python3
"""Benchmark of the B200 DG hydro time step (DOF-stage updates/s).

Workload: the sloping-beach basin (100 x 20 km, 2236 x 447 cells split into
1,998,984 triangles), FP64 DG p=1, SSP-RK(2,2), wetting/drying, slope limiter
5, nodal Manning n = 0.025 +-20 %, dt = 0.5 s.  A "step" is one
DG_HYDRO_TIMESTEP over the whole mesh.  The deck is generated (seeded) into
--workdir and read through the library's fort.14/15/dg/13 reader.

    python bench.py [--steps K] [--warmup W] [--gpus N]
    python bench.py --impl reference          # CPU arm (the FP64 oracle)

Multi-GPU (torchrun): each rank steps its own replica of the basin; the path
has no data exchange between independent meshes (weak scaling, replicas only).
The "partitioned" object is the strong-scaling form: the one bench mesh split
into one partition per rank, with the halo exchange over NCCL.

Each handle's tile and limiter block shapes are picked after warm-up by the
library's autotuner (whole steps with each shape, the state restored
afterwards; "tiles" objects give the picks and per-shape times);
--no-autotune keeps the default shapes.

The line's "mixed" object is the mixed-precision form (FP32 edge, volume and
limiter terms; FP64 state, SSP combination and wet/dry) on the same deck: its
rate, its speed-up over the FP64 line and its error against the FP64 form.
The "config3" object is the 8M-element quarter annulus with wind (config 3):
at p=1 and at p=2 (SSP-RK(3,3)), FP64 and mixed rates and the mixed forms'
errors against FP64 after 5000 steps of a quickly ramped copy.  The line's
"other_variant" object is the opt-in FMA build on the bench deck, and
"parity" the headline build against the FP64 oracle after the CPU sample's
steps.

    python bench.py --adjoint-only [--adjoint-nx NX --adjoint-ny NY --adjoint-steps K --adjoint-no-fd]
    python bench.py --p2-only [--config3-nr NR --config3-nth NTH --config3-p2-steps K --config3-p2-err-steps K]

run the adjoint object or the config-3 p=2 objects alone (the profiling
drivers of those kernels).
The "ensemble" object is the batched configuration: 256 seeded members of
5k-200k elements (about 13.5M in all) advanced by one handle in mixed
precision, with the batched-vs-one-at-a-time rate of its first 16 members.
The "adjoint" object times the discrete adjoint (gradient of a gauge misfit
w.r.t. Manning n and bathymetry) against the forward on the 1M-element wet/dry
sloping beach, 2000 steps, and gives its central finite-difference check on a
10k-element smooth subcase.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

DOFS_PER_ELEMENT = 9  # 3 variables x 3 modes at p=1
# Algorithmic bytes per element and stage of the stage kernel (the model of
# config 2 for the path): state 2.5 x 72 (stage state in and out, and the
# step-start state on the second of two stages) + HB modes 24 + inverse
# Jacobian and area 40 + neighbour element ids 12 + WDFLG read and write 8 +
# Manning n 8.
STAGE_KERNEL_BYTES = 2.5 * 72 + 24 + 40 + 12 + 8 + 8
# the whole RK stage adds the limiter's node ids 12 and the node min/max
# written and read back 24
STEP_BYTES_PER_ELEMENT_STAGE = STAGE_KERNEL_BYTES + 12 + 24
# what stage_p1 reads beyond that model, per element-stage: the geometry rows
# it copies to shared memory (normals, Jacobian terms, XLEN/AREAS, mean
# Manning n: 112 B where the model counts 40 + 8), the tile plan (1.63 edge
# tasks of 8 bytes and 0.25 halo ids per element on the Morton-ordered mesh)
# and the packed edge kinds / task slots
STAGE_OVERHEAD_BYTES = {"geometry_rows_beyond_model": 112 - 48, "tile_plan": 14, "edge_info": 8}
# DRAM bytes per element of one stage_p1 launch (strict build),
# dram__bytes_read.sum + dram__bytes_write.sum from ncu on the same deck at
# 999,492 elements: the mean of a stage-1 (292.2) and a stage-2 (368.6)
# launch; traffic grows with the element count.
STAGE_TRAFFIC_BYTES = 0.5 * (292.2 + 368.6)


def rank_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(ms: float, world: int, dist=None, device: str = "cuda") -> float:
    """The slowest rank's time: every rank's device-timed milliseconds reduced
    with MAX (NCCL on the GPUs; gloo with device="cpu")."""
    if world <= 1 or dist is None:
        return float(ms)
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world: int, ne: int, nrk: int, steps: int, ms: float) -> float:
    """DOF-stage updates/s of the whole job: every rank steps its own basin
    of ne elements (weak scaling), timed by the slowest rank."""
    return world * DOFS_PER_ELEMENT * ne * nrk * steps / (ms / 1e3)


def ensure_deck(workdir: Path, nx: int, ny: int, rank: int, world: int, dist=None) -> Path:
    from dgswem_b200 import decks
    path = workdir / f"sloping_beach_{nx}x{ny}"
    done = path / ".complete"
    if rank == 0 and not done.exists():
        decks.sloping_beach(path, nx=nx, ny=ny, nsteps=2000, dt=0.5)
        done.write_text("ok\n")
    if world > 1 and dist is not None:
        dist.barrier()
    return path


def rank0_first(rank: int, world: int, dist, fn):
    """fn() on rank 0 first -- it writes decks into the shared work directory
    -- then, after a barrier, on the other ranks, which find the decks
    complete and only open them (no two ranks write the same files); every
    rank gets fn's result."""
    out = fn() if rank == 0 else None
    if world > 1 and dist is not None:
        dist.barrier()
    if rank != 0:
        out = fn()
    return out


def config3_deck(workdir, nr: int, nth: int, p: int = 1, dramp: float | None = None) -> Path:
    """The config-3 quarter annulus (nr x nth cells, dt = 0.5 s, NWS=1, DG of
    degree p; the tide and wind ramp over ``dramp`` days, the generator's two
    days by default) under workdir, written unless complete.  p=1 steps with
    SSP-RK(2,2); p=2 with SSP-RK(3,3): DG of degree 2 needs a third-order RK
    for linear stability (with RK2 the p=2 run grows without bound, which
    5000 steps of a quickly ramped tide show)."""
    from dgswem_b200 import decks
    path = Path(workdir) / (f"config3_{nr}x{nth}" + ("" if p == 1 else f"_p{p}") +
                            ("" if dramp is None else f"_ramp{dramp:g}"))
    done = path / ".complete"
    if not done.exists():
        kw = {} if dramp is None else {"dramp": dramp}
        if p == 2:
            kw.update(rk_stage=3, rk_order=3)
        decks.quarter_annulus(path, nr=nr, nth=nth, nsteps=5000, dt=0.5, nws=1, extra={"pl": p, "ph": p}, **kw)
        done.write_text("ok\n")
    return path


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def mass(deck, ze) -> float:
    """Total water volume: sum over elements of (ZE mode 1 + HB mode 1) * area."""
    s = deck.s
    ne = s.ne
    nm = deck.int_array("nm", 3 * ne).reshape(3, ne) - 1
    x, y = deck.real_array("x", s.np), deck.real_array("y", s.np)
    a, b, c = nm
    areas = (x[a] - x[c]) * (y[b] - y[c]) + (x[c] - x[b]) * (y[a] - y[c])
    hb = deck.real_array("hb", 3 * ne).reshape(ne, 3)
    return float(np.sum((ze[:, 0] + hb[:, 0]) * areas * 0.5))


def autotune(h, args, it: int) -> dict | None:
    """Tile and limiter block shapes picked by the library's autotuner
    (dgswem_cuda_autotune: whole steps from step ``it`` with each shape,
    state restored), with its per-shape milliseconds per step; None with
    --no-autotune (the default shapes)."""
    if args.no_autotune:
        return None
    t0 = time.perf_counter()
    r = h.autotune(it=it, steps=args.tune_steps, reps=3, cached=True)
    r["tune_s"] = time.perf_counter() - t0
    return r


def mixed_arm(deck, stream, args, world: int, dist, device: int) -> dict:
    """The mixed-precision form (DGSWEM_CUDA_MIXED) on the same deck: its rate
    (same timing rules as the FP64 line), per-kernel times, and its error
    against the headline FP64 build after ``--mixed-err-steps`` steps from the
    initial state (nodal elevation and velocity, element-mean elevation, total
    water volume, wet/dry flags)."""
    import torch
    from dgswem_b200 import HydroStep
    hm = HydroStep(deck, device=device, mixed=True)
    hm.set_stream(stream.cuda_stream)
    hm.run(1, args.warmup)
    tiles = autotune(hm, args, args.warmup + 1)
    it = graphs_on(hm, args, args.warmup + 1)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    hm.run(it, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dist, "cuda")
    hm.set_graph(0)
    hm.profile(True)
    hm.run(it + args.steps, 20)
    prof = hm.profile_read()
    hm.profile(False)
    hm.close()
    value = whole_job_rate(world, deck.s.ne, deck.s.nrk, args.steps, ms)
    # error against the FP64 form, both from the deck's initial state
    n = args.mixed_err_steps
    outs = []
    for kw in (variant_kwargs(args.variant), {"mixed": True}):
        with HydroStep(deck, device=device, **kw) as h:
            h.set_stream(stream.cuda_stream)
            h.run(1, n)
            h.synchronize()
            outs.append((h.state(), h.modal2nodal()))
    (sf, nf), (sm, nmx) = outs
    wet = (nf[3] == 1) & (nmx[3] == 1)
    mf, mm = mass(deck, sf[0]), mass(deck, sm[0])
    err = {"steps": n,
           "eta_nodal_linf_m": float(np.abs(nmx[0] - nf[0])[wet].max()),
           "ze_mean_linf_m": float(np.abs(sm[0][:, 0] - sf[0][:, 0]).max()),
           "vel_nodal_linf_ms": float(max(np.abs(nmx[1] - nf[1])[wet].max(), np.abs(nmx[2] - nf[2])[wet].max())),
           "mass_rel": (mm - mf) / mf,
           "wdflg_differ": int((sm[3] != sf[3]).sum())}
    return {"value": value, "unit": "DOF-stage/s", "ms_per_step": ms / args.steps,
            "dtype": "f32 edge/volume/limiter terms, f64 state, SSP, wet/dry",
            "per_kernel_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items() if v[1]},
            "tiles": tiles, "err_vs_fp64": err}


def graphs_on(h, args, it: int) -> int:
    """With --graph-steps > 0: whole-step CUDA graphs for the handle's run
    call (dgswem_cuda_set_graph), captured by running one chunk from step
    ``it`` outside any timing; returns the next step."""
    if not args.graph_steps:
        return it
    h.set_graph(args.graph_steps)
    h.run(it, args.graph_steps)
    return it + args.graph_steps


def config3_met(npn: int):
    """Config 3's uniform wind stress of 0.1 Pa at 30 degrees (NWS=1:
    WSX2 = tau/rho0 cos 30, WSY2 = tau/rho0 sin 30, PR2 = 0) on npn nodes."""
    tau_rho = 0.1 / 1000.0
    return (np.full(npn, tau_rho * math.cos(math.radians(30.0))), np.full(npn, tau_rho * math.sin(math.radians(30.0))),
            np.zeros(npn))


def config3_p2(args, stream, device: int, world: int, dist, met=None) -> dict:
    """Config 3 at p=2: the quarter annulus of config3_arm at p=2 (18 DOFs
    per element, SSP-RK(3,3)), the headline FP64 build and the mixed form
    timed over ``--config3-p2-steps`` steps (the "p2" and "p2_mixed"
    objects), and with ``--config3-p2-err-steps`` > 0 the mixed form's error
    against FP64 on the quickly ramped copy.  ``--p2-only`` runs this alone
    (the profiling driver of the p=2 kernels)."""
    import torch
    from dgswem_b200 import Deck, HydroStep
    nr, nth, w = args.config3_nr, args.config3_nth, args.warmup
    out = {}
    # the p=2 half: the same annulus at p=2 (18 DOFs per element), the
    # headline FP64 build and the mixed form
    path2 = rank0_first(rank_env()[0], world, dist, lambda: config3_deck(args.workdir, nr, nth, p=2))
    deck2 = Deck(path2)
    if met is None:
        met = config3_met(deck2.s.np)
    k2 = args.config3_p2_steps
    dofs = 3 * deck2.s.dofh
    for name, kw in (("p2", variant_kwargs(args.variant)), ("p2_mixed", {"mixed": True})):
        with HydroStep(deck2, device=device, **kw) as h:
            h.set_stream(stream.cuda_stream)
            h.set_met(*met)
            h.run(1, w)
            it = graphs_on(h, args, w + 1)
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h.run(it, k2)
            e1.record(stream)
            torch.cuda.synchronize()
            ms2 = max_over_ranks(e0.elapsed_time(e1), world, dist, "cuda")
            h.set_graph(0)
            h.profile(True)
            h.run(it + k2, 4)
            prof = h.profile_read()
            h.profile(False)
            h.synchronize()
            tiled = h.get_shapes()[0] >= 0
        out[name] = {"value": world * dofs * deck2.s.ne * deck2.s.nrk * k2 / (ms2 / 1e3), "unit": "DOF-stage/s",
                     "dofs_per_element": dofs, "steps": k2, "ms_per_step": ms2 / k2,
                     "stage_ms": prof["stage_p1"][0] / max(prof["stage_p1"][1], 1),
                     "dtype": "f64" if name == "p2" else "mixed (f32 traces/fluxes/volume terms, f64 sums/state/SSP)",
                     "kernels": ("p2_tile (64-element tiles, edge fluxes in shared memory)" if tiled
                                 else "p2_edges + p2_elements") + " per RK stage"}
    deck2.close()
    out["p2_mixed"]["speedup_vs_fp64"] = out["p2_mixed"]["value"] / out["p2"]["value"]
    if args.config3_p2_err_steps > 0:
        epath2 = rank0_first(rank_env()[0], world, dist,
                             lambda: config3_deck(args.workdir, nr, nth, p=2, dramp=args.config3_err_dramp))
        edeck2 = Deck(epath2)
        st2 = {}
        for name, kw in (("fp64", variant_kwargs(args.variant)), ("mixed", {"mixed": True})):
            with HydroStep(edeck2, device=device, **kw) as h:
                h.set_stream(stream.cuda_stream)
                h.set_met(*met)
                h.run(1, args.config3_p2_err_steps)
                h.synchronize()
                st2[name] = (h.state(), h.modal2nodal())
        (pf_, pnf), (pm_, pnm) = st2["fp64"], st2["mixed"]
        ne2 = edeck2.s.ne
        nm2 = edeck2.int_array("nm", 3 * ne2).reshape(3, ne2) - 1
        x2, y2 = edeck2.real_array("x", edeck2.s.np), edeck2.real_array("y", edeck2.s.np)
        hb2 = edeck2.real_array("hb", 6 * ne2).reshape(ne2, 6)
        a2, b2, c2 = nm2
        ar2 = 0.5 * ((x2[a2] - x2[c2]) * (y2[b2] - y2[c2]) + (x2[c2] - x2[b2]) * (y2[a2] - y2[c2]))
        vf, vm = np.sum((pf_[0][:, 0] + hb2[:, 0]) * ar2), np.sum((pm_[0][:, 0] + hb2[:, 0]) * ar2)
        edeck2.close()
        out["p2_mixed"]["err_vs_fp64"] = {
            "steps": args.config3_p2_err_steps, "ramp_days": args.config3_err_dramp,
            "fp64_eta_nodal_max_m": float(np.abs(pnf[0]).max()),
            "fp64_vel_nodal_max_ms": float(max(np.abs(pnf[1]).max(), np.abs(pnf[2]).max())),
            "eta_nodal_linf_m": float(np.abs(pnm[0] - pnf[0]).max()),
            "ze_mean_linf_m": float(np.abs(pm_[0][:, 0] - pf_[0][:, 0]).max()),
            "vel_nodal_linf_ms": float(max(np.abs(pnm[1] - pnf[1]).max(), np.abs(pnm[2] - pnf[2]).max())),
            "mass_rel": (vm - vf) / vf}
    return out


def config3_arm(args, stream, device: int, world: int, dist) -> dict:
    """Config 3 at p=1: the quarter annulus of config 1 refined to
    ``--config3-nr`` x ``--config3-nth`` cells (8M triangles by default),
    h = 3.048 (r / 60.96 km)^2 m, M2 tide of 0.3048 m on the outer arc,
    linear friction tau = 1e-4 1/s, dt = 0.5 s, and a uniform wind stress of
    0.1 Pa at 30 degrees (NWS=1: WSX2 = tau/rho0 cos 30, WSY2 = tau/rho0
    sin 30, PR2 = 0).  FP64 and mixed rates with the FP64 line's timing
    rules, and the mixed form's error against the FP64 form after
    ``--config3-err-steps`` steps from the same state.  With
    ``--config3-p2-steps`` > 0 the same annulus at p=2 is timed too (the
    FP64 build and the mixed form, with SSP-RK(3,3)): the "p2" and "p2_mixed"
    objects."""
    import torch
    from dgswem_b200 import Deck, HydroStep
    nr, nth = args.config3_nr, args.config3_nth
    t0 = time.perf_counter()
    path = rank0_first(rank_env()[0], world, dist, lambda: config3_deck(args.workdir, nr, nth))
    t_write = time.perf_counter() - t0
    deck = Deck(path)
    npn = deck.s.np
    met = config3_met(npn)
    k, w = args.config3_steps, args.warmup
    out = {"workload": f"quarter annulus {nr}x{nth} cells, {deck.s.ne} elements, FP64/mixed DG p=1, SSP-RK(2,2), "
                       "linear friction, wind 0.1 Pa at 30 degrees (NWS=1), dt=0.5 s",
           "elements": int(deck.s.ne), "steps": k, "warmup": w, "deck_write_s": t_write}
    states = {}
    for name, kw in (("fp64", variant_kwargs(args.variant)), ("mixed", {"mixed": True})):
        with HydroStep(deck, device=device, **kw) as h:
            h.set_stream(stream.cuda_stream)
            h.set_met(*met)
            h.run(1, w)
            tiles = autotune(h, args, w + 1)
            it = graphs_on(h, args, w + 1)
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            h.run(it, k)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = max_over_ranks(e0.elapsed_time(e1), world, dist, "cuda")
            out[name] = {"value": whole_job_rate(world, deck.s.ne, deck.s.nrk, k, ms), "unit": "DOF-stage/s",
                         "ms_per_step": ms / k,
                         "tile_shape": tiles["tile_shape"] if tiles else None}
    # the error comparison: both forms from the same initial state over
    # --config3-err-steps steps of a copy of the deck whose tide and wind
    # ramp up within the run (--config3-err-dramp days), so that the basin
    # moves
    epath = rank0_first(rank_env()[0], world, dist,
                        lambda: config3_deck(args.workdir, nr, nth, dramp=args.config3_err_dramp))
    edeck = Deck(epath)
    for name, kw in (("fp64", variant_kwargs(args.variant)), ("mixed", {"mixed": True})):
        with HydroStep(edeck, device=device, **kw) as h:
            h.set_stream(stream.cuda_stream)
            h.set_met(*met)
            h.run(1, args.config3_err_steps)
            h.synchronize()
            states[name] = (h.state(), h.modal2nodal())
    (sf, nf), (sm, nmx) = states["fp64"], states["mixed"]
    mf, mm = mass(edeck, sf[0]), mass(edeck, sm[0])
    edeck.close()
    out["mixed"]["speedup_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    if args.config3_p2_steps > 0:
        out.update(config3_p2(args, stream, device, world, dist, met))
    out["mixed"]["err_vs_fp64"] = {
        "steps": args.config3_err_steps, "ramp_days": args.config3_err_dramp,
        "fp64_eta_nodal_max_m": float(np.abs(nf[0]).max()),
        "fp64_vel_nodal_max_ms": float(max(np.abs(nf[1]).max(), np.abs(nf[2]).max())),
        "eta_nodal_linf_m": float(np.abs(nmx[0] - nf[0]).max()),
        "ze_mean_linf_m": float(np.abs(sm[0][:, 0] - sf[0][:, 0]).max()),
        "vel_nodal_linf_ms": float(max(np.abs(nmx[1] - nf[1]).max(), np.abs(nmx[2] - nf[2]).max())),
        "mass_rel": (mm - mf) / mf}
    deck.close()
    return out


def ensemble_arm(args, stream, device: int, world: int, dist) -> dict:
    """The batched configuration: ``--ensemble-members`` seeded members
    (rectangles and quarter annuli, element counts log-uniform in [5k, 200k],
    tidal amplitude, Manning n and wind drawn per member), mixed precision,
    advanced by one handle on the merged meshes.  Also times the first 16
    members as a 16-member ensemble and one member at a time (a handle per
    member, the same steps), for the batching gain on meshes of this size."""
    import torch
    from dgswem_b200 import HydroStep, decks
    from dgswem_b200.ensemble import Ensemble, make_members
    specs = decks.ensemble_specs(args.ensemble_members)
    t0 = time.perf_counter()
    ds, met = rank0_first(rank_env()[0], world, dist,
                          lambda: make_members(Path(args.workdir) / "ensemble", specs,
                                               workers=min(16, os.cpu_count() or 1)))
    t_decks = time.perf_counter() - t0
    k, w = args.ensemble_steps, args.warmup

    def timed(run, first_it):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        run(first_it, k)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    def batched(members, wsx, wsy, pr):
        with Ensemble(members, device=device, mixed=True) as ens:
            ens.hs.set_stream(stream.cuda_stream)
            ens.set_met(wsx, wsy, pr)
            ens.run(1, w)
            tiles = autotune(ens.hs, args, w + 1)
            if args.ensemble_graph_steps:
                ens.hs.set_graph(args.ensemble_graph_steps)
                ens.run(w + 1, args.ensemble_graph_steps)  # capture, outside the timing
                w1 = w + 1 + args.ensemble_graph_steps
            else:
                w1 = w + 1
            l0 = ens.hs.kernel_launches
            ms = timed(ens.run, w1)
            return ms, ens.hs.kernel_launches - l0, ens.total_elements, ens.nrk, tiles

    ms, launches, ne_tot, nrk, tiles = batched(ds, *met)
    ms = max_over_ranks(ms, world, dist, "cuda")
    sub = min(16, len(ds))
    ms_sub, _, ne_sub, _, _ = batched(ds[:sub], *(f[:sub] for f in met))
    ms_one = 0.0
    for i in range(sub):
        with HydroStep(ds[i], device=device, mixed=True) as hs:
            hs.set_stream(stream.cuda_stream)
            hs.set_met(met[0][i], met[1][i], met[2][i])
            hs.run(1, w)
            autotune(hs, args, w + 1)
            w1 = w + 1
            if args.ensemble_graph_steps:
                hs.set_graph(args.ensemble_graph_steps)
                hs.run(w1, args.ensemble_graph_steps)
                w1 += args.ensemble_graph_steps
            ms_one += timed(hs.run, w1)
    rate = lambda ne, t: DOFS_PER_ELEMENT * ne * nrk * k / (t / 1e3)  # noqa: E731
    for d in ds:
        d.close()
    return {"members": len(specs), "elements": int(ne_tot), "steps": k, "warmup": w,
            "value": whole_job_rate(world, ne_tot, nrk, k, ms), "unit": "DOF-stage/s",
            "ms_per_step": ms / k, "dtype": "mixed (f32 edge/volume/limiter, f64 state/SSP/wet-dry)",
            "gpu_launches": int(launches), "deck_write_read_s": t_decks, "tiles": tiles,
            "graph_steps": args.ensemble_graph_steps,
            "subset16": {"elements": int(ne_sub), "batched_rate": rate(ne_sub, ms_sub),
                         "one_at_a_time_rate": rate(ne_sub, ms_one), "batching_speedup": ms_one / ms_sub}}


def adjoint_arm(args, device: int) -> dict:
    """Discrete adjoint of the FP64 step (gradient of a 64-gauge elevation
    misfit w.r.t. the element-mean Manning n and the bathymetry modes, sqrt(N)
    state checkpoints, the limiter's and WETDRY's branches frozen at the
    forward's) on the adjoint configuration: the wet/dry sloping beach of
    999,040 elements (limiter 5, nodal Manning n), 2000 steps, observations
    from a forward run with Manning n 20 % larger; the tide is ramped over
    0.002 days so that the misfit sees it within the run.  Reports the forward
    and gradient times (CUDA events on the handle's stream, both including the
    host's gauge reads) and a central finite-difference check on the
    10,112-element smooth always-wet subcase."""
    import torch
    from dgswem_b200 import Deck, decks
    from dgswem_b200.adjoint import GaugeMisfitProblem, element_manning, locate_gauges
    n = args.adjoint_steps
    nx, ny = args.adjoint_nx, args.adjoint_ny
    path = decks.sloping_beach(Path(args.workdir) / f"adjoint_beach_{nx}x{ny}", nx=nx, ny=ny, lx=100e3, ly=20e3,
                               dt=0.5, nsteps=n, dramp=0.002)
    deck = Deck(path)
    rng = np.random.default_rng(20261203)
    xy = np.column_stack([rng.uniform(500.0, 8000.0, 64), rng.uniform(1e3, 19e3, 64)])
    elem, phi = locate_gauges(deck, xy)
    n0 = element_manning(deck)
    truth = GaugeMisfitProblem(deck, elem, phi, n, device=device)
    truth.set_params(nbar=1.2 * n0)
    obs = truth.run()
    truth.close()
    prob = GaugeMisfitProblem(deck, elem, phi, n, obs=obs, device=device)
    stream = torch.cuda.ExternalStream(prob.hs.stream_handle)

    def timed(fn):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1)

    prob.forward()  # warm-up
    prob.gradient()
    j, ms_f = timed(prob.forward)
    (gn, ghb), ms_b = timed(prob.gradient)
    ne = deck.s.ne
    prob.close()
    deck.close()
    out = {"workload": f"wet/dry sloping beach 100x20 km, {ne} elements, FP64, limiter 5, WETDRY, Manning n, "
                       f"64 gauges, {n} steps, checkpoints every {math.ceil(math.sqrt(n))} steps",
           "steps": n, "forward_ms": ms_f, "gradient_ms": ms_b, "gradient_over_forward": ms_b / ms_f,
           "misfit": j, "grad_norm": {"nbar": float(np.linalg.norm(gn)), "hb": float(np.linalg.norm(ghb))}}
    if args.adjoint_no_fd:
        return out
    # central finite differences on the 10k-element basin, smooth direction
    small = decks.smooth_basin(Path(args.workdir) / "adjoint_basin_10k", nsteps=300, dt=0.5, dramp=0.002)
    d = Deck(small)
    r = np.random.default_rng(3)
    e2, p2 = locate_gauges(d, np.column_stack([r.uniform(300.0, 2500.0, 16), r.uniform(300.0, 3700.0, 16)]))
    m0 = element_manning(d)
    h0 = d.real_array("hb", 3 * d.s.ne).reshape(d.s.ne, 3)
    t = GaugeMisfitProblem(d, e2, p2, 300, device=device)
    t.set_params(nbar=1.5 * m0)
    o2 = t.run()
    t.close()
    p = GaugeMisfitProblem(d, e2, p2, 300, obs=o2, device=device)
    p.set_params(m0, h0)
    p.forward()
    g1, g2 = p.gradient()
    dn = m0 * r.standard_normal(d.s.ne)
    nm = d.int_array("nm", 3 * d.s.ne).reshape(3, d.s.ne) - 1
    x = d.real_array("x", d.s.np)
    f = np.sin(2 * np.pi * x / 3000.0)
    dh = np.stack([(f[nm[0]] + f[nm[1]] + f[nm[2]]) / 3, -(f[nm[0]] + f[nm[1]]) / 6 + f[nm[2]] / 3,
                   (f[nm[1]] - f[nm[0]]) / 2], 1)
    eps = 1e-4
    jj = []
    for sgn in (1, -1):
        p.set_params(m0 + sgn * eps * dn, h0 + sgn * eps * dh)
        jj.append(p.forward())
    fd = (jj[0] - jj[1]) / (2 * eps)
    ad = float(g1 @ dn + np.sum(g2 * dh))
    p.close()
    d.close()
    out["fd_check"] = {"elements": 10112, "steps": 300, "eps": eps, "adjoint": ad, "central_fd": fd,
                       "rel_err": abs(ad - fd) / abs(fd)}
    return out


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def cpu_baseline(path: Path, nsteps: int, threads: int):
    """The FP64 oracle (test-infrastructure CPU restatement) on the host
    cores: steps 1..nsteps of the deck from its initial state, the first one
    untimed (first touch of the stage arrays).  Returns its rate over the
    timed steps, their seconds, and the oracle's state after step nsteps --
    the checker of the parity object."""
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import Oracle
    orc = Oracle(path, threads=threads)
    orc.step(1)
    t0 = time.perf_counter()
    for it in range(2, nsteps + 1):
        orc.step(it)
    dt = time.perf_counter() - t0
    ne, nrk = orc.ne, orc.info("nrk")
    state = orc.state()
    orc.close()
    return DOFS_PER_ELEMENT * ne * nrk * (nsteps - 1) / dt, dt, state


def parity(gpu_state, oracle_state, steps: int, variant: str) -> dict:
    """The headline build's state after ``steps`` steps from the deck's
    initial state against the oracle's: per variable the largest difference
    relative to the variable's largest oracle coefficient, and how many
    coefficients differ at all; wet/dry flags that differ."""
    out = {"steps": steps, "variant": variant}
    bitwise = True
    for a, b, name in zip(gpu_state[:3], oracle_state[:3], ("ZE", "QX", "QY")):
        out[f"{name}_max_rel"] = float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))
        out[f"{name}_coefficients_differ"] = int((a != b).sum())
        bitwise = bitwise and bool(np.array_equal(a, b))
    out["max_rel"] = max(out[f"{v}_max_rel"] for v in ("ZE", "QX", "QY"))
    out["wdflg_differ"] = int((gpu_state[3] != oracle_state[3]).sum())
    out["bit_identical"] = bitwise and out["wdflg_differ"] == 0
    return out


def partitioned_arm(deck, args, world: int, dist, device: int) -> dict:
    """The bench mesh split into ``world`` partitions, one per rank
    (DistributedPartition: halos by NCCL send/receive between the stage
    kernel and the limiter and after the limiter, as the reference's MPI
    ghost updates), strong scaling: the whole job advances one mesh.  At
    one rank the single partition runs through the same stage / limit entry
    points with no exchange.  Timed with CUDA events on each rank's stream,
    the slowest rank's time."""
    import torch
    from dgswem_b200 import DistributedPartition
    if world == 1 and not dist.is_initialized():
        # a one-rank group over gloo (no exchange happens) so that the
        # driver's group calls are defined
        import socket
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1)
        own_group = True
    else:
        own_group = False
    stream = torch.cuda.current_stream()
    dp = DistributedPartition(deck, **variant_kwargs(args.variant), transport="nccl")
    info = dp.hs.part_info()
    dp.run(1, args.warmup)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    k = args.partition_steps
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    dp.run(args.warmup + 1, k)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), world, dist if world > 1 else None, "cuda")
    dp.close()
    if own_group:
        dist.destroy_process_group()
    ne = deck.s.ne
    return {"workload": f"the bench mesh ({ne} elements) split into {world} partition(s), one per GPU",
            "scaling": "strong", "value": DOFS_PER_ELEMENT * ne * deck.s.nrk * k / (ms / 1e3),
            "unit": "DOF-stage/s", "steps": k, "ms_per_step": ms / k,
            "owned_elements_rank0": int(info["owned"]), "local_elements_rank0": int(info["local"]),
            "transport": "nccl send/receive of packed halos" if world > 1 else "none (one partition)"}


VARIANT_TEXT = {"strict": "strict: FP64 without FMA contraction, the oracle's evaluation order (bit-identical to it)",
                "fast": "fast: FP64 with FMA contraction"}


def variant_kwargs(variant: str) -> dict:
    return {"strict": True} if variant == "strict" else {"fast": True}


def other_variant_arm(deck, stream, args, world: int, dist, device: int) -> dict:
    """The FP64 build the headline does not use, on the same deck and timing
    rules (fewer steps): its rate, per-kernel times and shapes."""
    import torch
    from dgswem_b200 import HydroStep
    other = "fast" if args.variant == "strict" else "strict"
    with HydroStep(deck, device=device, **variant_kwargs(other)) as h:
        h.set_stream(stream.cuda_stream)
        h.run(1, args.warmup)
        tiles = autotune(h, args, args.warmup + 1)
        it = graphs_on(h, args, args.warmup + 1)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        k = args.other_variant_steps
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        h.run(it, k)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = max_over_ranks(e0.elapsed_time(e1), world, dist, "cuda")
        h.set_graph(0)
        h.profile(True)
        h.run(it + k, 10)
        prof = h.profile_read()
        h.profile(False)
    return {"variant": VARIANT_TEXT[other], "value": whole_job_rate(world, deck.s.ne, deck.s.nrk, k, ms),
            "unit": "DOF-stage/s", "steps": k, "ms_per_step": ms / k,
            "per_kernel_ms": {n: v[0] / max(v[1], 1) for n, v in prof.items() if v[1]}, "tiles": tiles}


def run_reference(args):
    rank, world, _ = rank_env()
    if rank != 0:
        return 0
    workdir = Path(args.workdir)
    workdir.mkdir(parents=True, exist_ok=True)
    path = ensure_deck(workdir, args.nx, args.ny, 0, 1)
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_lib import Oracle
    orc = Oracle(path, threads=threads)
    ne, nrk = orc.ne, orc.info("nrk")
    # each step is one full DG hydro step of the 2M-element mesh; the number of
    # timed steps is capped so the arm ends within a few minutes
    steps = max(1, min(args.steps, args.ref_max_steps))
    warm = max(1, min(args.warmup, 2))
    for it in range(1, warm + 1):
        orc.step(it)
    t0 = time.perf_counter()
    for it in range(warm + 1, warm + 1 + steps):
        orc.step(it)
    dt = time.perf_counter() - t0
    orc.close()
    value = DOFS_PER_ELEMENT * ne * nrk * steps / dt
    line = {
        "impl": "reference", "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s",
        "n_gpus": args.gpus, "steps": steps, "warmup": warm, "ms_per_step": 1e3 * dt / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, ne, nrk),
        "cpu_baseline": {"value": value, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
                         "sample": f"{steps} full hydro steps of the {ne}-element basin, OpenMP over {threads} threads; "
                                   "the Fortran reference cannot be built here (no Fortran compiler), so the "
                                   "CPU arm is the C++ FP64 restatement pinned to the reference golden outputs"},
        "e2e": {"value": value, "unit": "DOF-stage/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(args, ne, nrk):
    return {"workload": f"sloping beach 100x20 km, {ne} elements (2x{args.nx}x{args.ny}), FP64 DG p=1, "
                        f"SSP-RK({nrk},2), wet/dry + slope limiter 5 + nodal Manning n, dt=0.5 s",
            "elements": ne, "dofs": DOFS_PER_ELEMENT * ne, "rk_stages": nrk,
            "l2": "state buffers (3 x 144 MB) exceed the 126 MB L2; no flush between steps",
            "parallelism": f"replicas x{args.gpus}"}


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--nx", type=int, default=2236)
    ap.add_argument("--ny", type=int, default=447)
    ap.add_argument("--workdir", default=os.environ.get("DGSWEM_BENCH_DIR", "/tmp/dgswem_b200_bench"))
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--variant", choices=["strict", "fast"], default="strict",
                    help="FP64 kernel build of the headline: strict (no FMA contraction, bit-identical to the "
                         "oracle) or fast (FMA contraction)")
    ap.add_argument("--other-variant-steps", type=int, default=20,
                    help="timed steps of the other FP64 build on the same deck (0: skip)")
    ap.add_argument("--partition-steps", type=int, default=20,
                    help="timed steps of the partitioned arm: the bench mesh split over the ranks (0: skip)")
    ap.add_argument("--cpu-steps", type=int, default=12,
                    help="oracle steps from the initial state: the cpu_baseline sample and the parity check")
    ap.add_argument("--ref-max-steps", type=int, default=40)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision arm")
    ap.add_argument("--no-autotune", action="store_true", help="keep the default tile / limiter block shapes")
    ap.add_argument("--tune-steps", type=int, default=10, help="steps per shape timing of the autotuner")
    ap.add_argument("--config3-steps", type=int, default=100,
                    help="timed steps of the 8M-element config-3 annulus with wind (0: skip)")
    ap.add_argument("--config3-nr", type=int, default=1000)
    ap.add_argument("--config3-nth", type=int, default=4000)
    ap.add_argument("--config3-err-steps", type=int, default=5000,
                    help="steps of the config-3 mixed-vs-FP64 error comparison")
    ap.add_argument("--config3-p2-err-steps", type=int, default=5000,
                    help="steps of the p=2 mixed-vs-FP64 error comparison (0: skip)")
    ap.add_argument("--config3-err-dramp", type=float, default=0.01,
                    help="tide and wind ramp (days) of the error comparison's deck")
    ap.add_argument("--config3-p2-steps", type=int, default=50, help="timed steps of the p=2 config-3 annulus (0: skip)")
    ap.add_argument("--ensemble-members", type=int, default=256, help="members of the batched ensemble (0: skip)")
    ap.add_argument("--ensemble-steps", type=int, default=2000)
    ap.add_argument("--graph-steps", type=int, default=8,
                    help="whole steps per CUDA graph in the headline arm (even; 0: plain launches)")
    ap.add_argument("--ensemble-graph-steps", type=int, default=8,
                    help="whole steps per CUDA graph in the ensemble arm (even; 0: plain launches)")
    ap.add_argument("--adjoint-steps", type=int, default=2000, help="steps of the adjoint arm (0: skip)")
    ap.add_argument("--adjoint-nx", type=int, default=1580, help="cells along the adjoint beach (x)")
    ap.add_argument("--adjoint-ny", type=int, default=316, help="cells across the adjoint beach (y)")
    ap.add_argument("--adjoint-no-fd", action="store_true",
                    help="skip the adjoint arm's finite-difference check on the 10k-element basin")
    ap.add_argument("--p2-only", action="store_true",
                    help="only the config-3 p=2 timing (--config3-nr/-nth/-p2-steps/-p2-err-steps): the p=2 "
                         "kernels' profiling driver")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="run only the adjoint arm (a driver for profiling its kernels) and print its object")
    ap.add_argument("--mixed-err-steps", type=int, default=200,
                    help="steps of the mixed-vs-FP64 error comparison")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        return run_reference(args)

    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from dgswem_b200 import Deck, HydroStep

    rank, world, local = rank_env()
    torch.cuda.set_device(local)
    if args.adjoint_only:
        Path(args.workdir).mkdir(parents=True, exist_ok=True)
        if rank == 0:
            print(json.dumps({"adjoint": adjoint_arm(args, local)}), flush=True)
        return 0
    if args.p2_only:
        Path(args.workdir).mkdir(parents=True, exist_ok=True)
        if rank == 0:
            stream = torch.cuda.Stream(device=local)
            torch.cuda.set_stream(stream)
            print(json.dumps({"config3_p2": config3_p2(args, stream, local, 1, None)}), flush=True)
        return 0
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    workdir = Path(args.workdir)
    workdir.mkdir(parents=True, exist_ok=True)
    path = ensure_deck(workdir, args.nx, args.ny, rank, world, dist if world > 1 else None)
    # host setup: deck read + edge graph (READ_INPUT/PREP_DG), then device
    # create (orders, tile plan, geometry table, uploads); wall clock
    t_setup0 = time.perf_counter()
    deck = Deck(path)
    t_setup1 = time.perf_counter()
    vkw = variant_kwargs(args.variant)
    hs = HydroStep(deck, device=local, **vkw)
    torch.cuda.synchronize()
    t_setup2 = time.perf_counter()
    ne, nrk = hs.ne, hs.nrk
    # all work on one dedicated stream; the events below are recorded on it
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    hs.set_stream(stream.cuda_stream)

    # warm-up, then the shapes (each timing restores the state)
    hs.run(1, args.warmup)
    tiles = autotune(hs, args, args.warmup + 1)
    torch.cuda.synchronize()
    it0 = args.warmup + 1
    if args.graph_steps:
        # whole-step CUDA graphs of the library's run call, captured outside
        # the timing
        hs.set_graph(args.graph_steps)
        hs.run(it0, args.graph_steps)
        it0 += args.graph_steps
        torch.cuda.synchronize()

    sampler = ClockSampler(local)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = hs.kernel_launches
    sampler.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    hs.run(it0, args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clocks = sampler.stop()
    launches = hs.kernel_launches - launches0
    if args.graph_steps:
        hs.set_graph(0)  # the per-kernel timing, the e2e and parity legs launch step by step
    ms = e0.elapsed_time(e1)
    ms_max = max_over_ranks(ms, world, dist if world > 1 else None, "cuda")
    hs.synchronize()
    it0 += args.steps
    value = whole_job_rate(world, ne, nrk, args.steps, ms_max)

    # per-kernel event timing of the dominant kernel (same stream)
    prof_steps = 20
    hs.profile(True)
    hs.run(it0, prof_steps)
    prof = hs.profile_read()
    hs.profile(False)
    it0 += prof_steps
    stage_ms, stage_n = prof["stage_p1"]
    avg_stage_s = stage_ms / 1e3 / max(stage_n, 1)
    peak, peak_kind = measured_peak()
    achieved = STAGE_KERNEL_BYTES * ne / avg_stage_s / 1e9
    stage_total_ms = sum(v[0] for v in prof.values())
    stage_total_n = prof["stage_p1"][1]
    step_achieved = STEP_BYTES_PER_ELEMENT_STAGE * ne * nrk / (ms_max / args.steps / 1e3) / 1e9

    # end to end through the C-ABI with host buffers: every step uploads the
    # state from pinned host memory, steps, and downloads the new state
    pin = lambda shape, dt: torch.empty(shape, dtype=dt, pin_memory=True)  # noqa: E731
    hze, hqx, hqy = (pin((ne, 3), torch.float64) for _ in range(3))
    hwd = pin((ne,), torch.int32)
    hs.download_into(hze.numpy(), hqx.numpy(), hqy.numpy(), hwd.numpy())
    nz, nqx, nqy, nwd = (a.numpy() for a in (hze, hqx, hqy, hwd))
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    x0.record(stream)
    for i in range(args.e2e_steps):
        hs.set_state(nz, nqx, nqy, nwd)
        hs.timestep(it0 + i)
        hs.download_into(nz, nqx, nqy, nwd)
    x1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(x0.elapsed_time(x1), world, dist if world > 1 else None, "cuda")
    e2e_value = whole_job_rate(world, ne, nrk, args.e2e_steps, e2e_ms)
    state_bytes = 9 * 8 * ne + 4 * ne
    hs.synchronize()

    line = {
        "metric": "DOF-stage updates/s", "value": value, "unit": "DOF-stage/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded sloping-beach deck; no public dataset)",
        "config": workload_config(args, ne, nrk),
        "gpu_launches": int(launches),
        "graph_steps": args.graph_steps,
        "setup_s": {"deck_read": t_setup1 - t_setup0, "device_create": t_setup2 - t_setup1},
        "tiles": tiles,
        "clocks": clocks,
        "e2e": {"value": e2e_value, "unit": "DOF-stage/s", "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes,
                "how": "per step: upload ZE/QX/QY/WDFLG from pinned host memory, one hydro step, download"},
        "variant": VARIANT_TEXT[args.variant],
        "roofline": {"bound": "hbm", "kernel": "stage_p1", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": STAGE_TRAFFIC_BYTES * ne,
                     "traffic_source": "ncu dram bytes per element of a stage-1 and a stage-2 launch (999,492 elements), "
                                       "scaled by the element count",
                     "algorithmic_bytes_per_element_stage": STAGE_KERNEL_BYTES,
                     "overhead_bytes_per_element_stage": STAGE_OVERHEAD_BYTES,
                     "avg_launch_ms": avg_stage_s * 1e3,
                     "whole_step": {"bytes_per_element_stage": STEP_BYTES_PER_ELEMENT_STAGE,
                                    "achieved": step_achieved, "frac": step_achieved / peak,
                                    "ms_per_step": ms_max / args.steps},
                     "stage_all_kernels_ms": stage_total_ms / max(stage_total_n, 1),
                     "per_kernel_ms": {k: v[0] / max(v[1], 1) for k, v in prof.items() if v[1]}},
    }
    if args.other_variant_steps > 0:
        line["other_variant"] = other_variant_arm(deck, stream, args, world, dist if world > 1 else None, local)
    if args.partition_steps > 0:
        line["partitioned"] = partitioned_arm(deck, args, world, dist, local)
    if not args.no_mixed:
        mixed = mixed_arm(deck, stream, args, world, dist if world > 1 else None, local)
        mixed["speedup_vs_fp64"] = mixed["value"] / value  # against the headline FP64 build
        if "other_variant" in line:
            mixed["speedup_vs_other_fp64_build"] = mixed["value"] / line["other_variant"]["value"]
        line["mixed"] = mixed
    if args.config3_steps > 0:
        line["config3"] = config3_arm(args, stream, local, world, dist if world > 1 else None)
    if args.ensemble_members > 0:
        line["ensemble"] = ensemble_arm(args, stream, local, world, dist if world > 1 else None)
    if args.adjoint_steps > 0 and world == 1:
        line["adjoint"] = adjoint_arm(args, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the checker: the headline build and the oracle from the deck's
        # initial state for the same steps; the oracle's run is also the
        # timed CPU baseline sample
        k = args.cpu_steps
        with HydroStep(deck, device=local, **vkw) as hp:
            hp.set_stream(stream.cuda_stream)
            hp.run(1, k)
            hp.synchronize()
            gstate = hp.state()
        threads = os.cpu_count() or 1
        v, secs, ostate = cpu_baseline(path, k, threads)
        line["cpu_baseline"] = {"value": v, "unit": "DOF-stage/s", "cores": threads, "kind": "port",
                                "sample": f"steps 2-{k} of the same {ne}-element deck from its initial state "
                                          f"({secs:.1f} s), FP64 oracle, OpenMP"}
        line["parity"] = parity(gstate, ostate, k, args.variant)
    hs.close()
    deck.close()
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
