#!/usr/bin/env python3
"""Benchmark of the MIMICA dynamical-core path on B200.

Metric: Mcell-updates/s = interior cells x integrator steps / time / 1e6, one
"step" = one full integrator step of the reference's scheme (two Heun stages,
each: scalar advection of density + 5 density-weighted scalars, momentum
advection/pgf/buoyancy, stage update, anelastic projection).

Workload (default): the shallow-cumulus-like domain, 512 x 512 x 256 interior cells,
dx = dy = 25 m, stretched dz (10 m -> 100 m), 3 momentum + density + 5 scalars
(theta_l, qt, qr, nr, aerosol number), scalar scheme WENO (the reference's
WENO3-switch), FD4 momentum, dt = 1 s, plain FP64 form.  Synthetic seeded inputs
(no dataset exists for this benchmark); the working set (~16 GB) exceeds the
126 MB L2, so no flush is needed between timed steps.

Both arithmetic forms are measured by default: the plain FP64 form is the headline
(`value`, bit-exact with the CPU restatement of the reference routines), and the mixed
form (FP32 stencils, fluxes and spectra; FP64 state, tendencies, tridiagonal elimination
and divergence residual, with refinement of the Poisson solve) is reported in the
`mixed` object: its throughput, roofline, and its per-field relative L2 error against the
FP64 form after `--err-steps` steps from the same initial state.

`python bench.py --gpus N --steps K --warmup W` prints one JSON line.
`--impl reference` times the reference's algorithm on the host cores instead
(the CPU restatement, OpenMP over all cores, bounded sample).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    except Exception:
        return PEAKS_FALLBACK, "fallback"


# ---------------- algorithmic bytes (FP64 state), per interior cell ----------------
def alg_bytes(nf_scalar: int, nsubp: int, sgs: bool = False) -> dict:
    """Minimal HBM traffic per interior cell of each kernel group (bytes).

    K1 (all scalar fields incl. density), per launch averaged over the two stages:
      stage 1: per field read psi_n, write psi*, T (24 B); momentum 24 B; two buoyancy
               stage tendencies written (16 B)
      stage 2: per field read psi*, psi_n, T, write psi_new (32 B); momentum 24 B; 16 B
    K2 (momentum), per launch: stage 1: read m_n (24), p (8), dens/es/qt + their stage
      tendencies (40), write m*, T (48); stage 2: read m*, m_n, T (72), p 8, 40, write m_new 24.
    Projection pass (FP64 spectra, half spectrum ~8 B/cell per complex plane):
      fft_x_fwd_div: read momentum 24, write spectrum 8; y/tridiag/y/x_inv: 4 x (8+8);
      correction: read dp 8, m 24, p 8, write m 24, p 8.
    """
    f = nf_scalar
    k1 = (f * 24 + 24 + 16 + f * 32 + 24 + 16) / 2.0
    k2 = ((24 + 8 + 40 + 48) + (72 + 8 + 40 + 24)) / 2.0
    proj = 32 + 64 + 72
    out = {"k1_scalar_advection": k1, "k2_momentum": k2, "fft_x_fwd_div": 32.0,
           "fft_y_tridiag_fft_y_fft_x_inv": 64.0, "correction_halo": 72.0}
    step = 2 * (k1 + k2) + 2 * nsubp * proj
    if sgs:
        # SGS diffusion, once per step: the viscosity kernel reads u, v, w, es, qt, dens and
        # writes the six deformation components, dens*fkv and the diffusivity; the momentum
        # stresses read dens*fkv and dij and write 3 tendencies; the scalar fluxes read the
        # diffusivity and f-1 scalars and write f-1 tendencies.  K1 and K2 read the stored
        # tendencies in both stages (f-1 and 3 fields).
        s = f - 1
        out["sgs_viscosity"] = 48.0 + 64.0
        out["sgs_momentum"] = 56.0 + 24.0
        out["sgs_scalars"] = 8.0 + 16.0 * s
        k1 += 8.0 * s
        k2 += 24.0
        out["k1_scalar_advection"], out["k2_momentum"] = k1, k2
        step = 2 * (k1 + k2) + 2 * nsubp * proj + out["sgs_viscosity"] + out["sgs_momentum"] + out["sgs_scalars"]
    out["step"] = step
    return out


# DRAM bytes per interior cell of one launch (mean of the two stages), from ncu captures
# of the WENO cumulus workload with density + 5 scalars, SGS off, plain FP64, at
# 384x384x64 (the mixed form moved the same bytes at 256x256x64).  Per-launch traffic
# grows in proportion to the cells processed: K1 207.4 B/cell at 256x256x64 and 211.3 at
# 384x384x64, K2 140.0 and 143.9.
MEASURED_TRAFFIC_PER_CELL = {"k1_scalar_advection": 211.3, "k2_momentum": 143.9}
TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one stage-1 and one stage-2 launch at "
                  "384x384x64 (profiles/k1_k2_traffic_cumulus.md), per interior cell, times this launch's cells")
# The same for an ensemble member (dry warm bubble, WENO, density + theta + one passive
# scalar, SGS off) at 256x256x96, plain FP64 (the mixed form: K1 116.4, K2 131.4)
MEMBER_TRAFFIC_PER_CELL = {"k1_scalar_advection": 118.4, "k2_momentum": 128.9}
MEMBER_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one stage-1 and one stage-2 launch of "
                         "a 256x256x96 warm-bubble member (profiles/k1_k2_traffic_warmbubble256x96.md), per interior "
                         "cell, times this launch's cells")


class ClockSampler:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


PAGEABLE_FALLBACKS = []   # shapes for which page-locked allocation failed (reported in e2e)


def host_buffers() -> str:
    return "page-locked" if not PAGEABLE_FALLBACKS else f"{len(PAGEABLE_FALLBACKS)} pageable (cudaMallocHost failed)"


def pinned_like(shape):
    """numpy array in page-locked host memory (cudaMallocHost); pageable if that fails,
    which the e2e object reports."""
    rt = C.CDLL("libcudart.so")
    n = int(np.prod(shape)) * 8
    p = C.c_void_p()
    if rt.cudaMallocHost(C.byref(p), C.c_size_t(n)) != 0:
        PAGEABLE_FALLBACKS.append(tuple(shape))
        return np.zeros(shape)
    buf = (C.c_double * int(np.prod(shape))).from_address(p.value)
    return np.frombuffer(buf, dtype=np.float64).reshape(shape)


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def dist_max(x: float, ws: int) -> float:
    if ws <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def dist_sum(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def dist_barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def bench_sgs(args, d):
    """SGS settings of the --sgs option (the BOMEX template's pran, zdec, momsf; uniform
    surface fluxes of its prescribed magnitude: 8.4 W/m2 sensible, 153 W/m2 latent heat,
    u* = 0.28 m/s)."""
    if args.sgs == "none":
        return None
    from fdd3260_b200 import config
    one = np.ones((d.ny, d.nx))
    return config.Sgs(pran=-0.4, zdec=2400.0, momsf=1, zrough=1.0, min_w=0.1,
                      esflux=7.0e-3 * one, qvflux=5.2e-5 * one, mflux=-(0.28 ** 2) * one)


def sgs_label(args):
    return {"none": "off", "smagorinsky": "Smagorinsky-Lilly, pran=-0.4, zdec=2400 m, surface fluxes"}[args.sgs]


def timed_cpu_sample(orc, st, seconds):
    """One timed warm-up step (page faults, OpenMP pool), then as many steps as fill about
    `seconds` of wall time (1 to 20), timed as one call: returns (steps, elapsed s)."""
    t0 = time.perf_counter()
    orc.stepping(st, nsteps=1, ntime0=1)
    warm = time.perf_counter() - t0
    n = int(min(20, max(1, math.ceil(seconds / max(warm, 1e-3)))))
    t0 = time.perf_counter()
    orc.stepping(st, nsteps=n, ntime0=1)
    return n, time.perf_counter() - t0


def cpu_domain(args, mx, nz, scheme):
    """The workload's domain at a reduced horizontal size, built entirely on the CPU: the grid
    metrics and base state come from the oracle's restatement of the reference's init
    routines, so this path never loads the CUDA library."""
    from fdd3260_b200 import config
    from oracle import oracle as O
    d = config.cumulus_domain(mx, mx, nz, scheme=scheme, init=O.Init(omp=True), muscl_limiter=args.limiter)
    d.sgs = bench_sgs(args, d)
    return d


def cpu_reference(args, d_full, scheme, omp=True):
    """The reference's algorithm timed on the host cores: the CPU restatement, bounded
    sample = a horizontally reduced domain with the same dz profile, spacing and fields.
    The sample runs as many steps as fill about args.cpu_seconds of wall time."""
    from fdd3260_b200 import config
    from oracle import oracle as O
    mx = args.cpu_sample_xy
    d = cpu_domain(args, mx, d_full.nz, scheme)
    st = config.cumulus_state(d, seed=1000, n_extra=3)
    orc = O.Oracle(d, omp=omp)
    nsamp_steps, dt = timed_cpu_sample(orc, st, args.cpu_seconds)
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)) if omp else 1
    val = d.cells * nsamp_steps / dt / 1e6
    return val, cores, (f"{mx}x{mx}x{d.nz} interior cells, {nsamp_steps} step(s) in {dt:.1f} s, same dz/dt/fields "
                        f"as the workload")


def reference_arm(args, cfg, metric, ws):
    """--impl reference: the reference's algorithm (the oracle's timed OpenMP build; the
    Fortran reference cannot be built on these hosts) on all host cores, exactly W warm-up
    and K timed integrator steps.  Each step is one step of a bounded sample of the workload:
    the same dz profile, spacing, fields and scheme on a horizontally reduced domain, whose
    size is halved from --ref-sample-xy until W + K steps fit in about --ref-seconds.
    ms_per_step is the sample's own time per step.  Nothing here loads the CUDA library."""
    from fdd3260_b200 import config
    from oracle import oracle as O
    mx = args.ref_sample_xy
    while True:
        d = cpu_domain(args, mx, args.nz, args.scheme)
        st = config.cumulus_state(d, seed=1000, n_extra=3)
        orc = O.Oracle(d, omp=True)
        t0 = time.perf_counter()
        st, _, _ = orc.stepping(st, nsteps=1, ntime0=1)      # warm-up step 1 (page faults, thread pool)
        one = time.perf_counter() - t0
        if one * (args.warmup + args.steps) <= args.ref_seconds or mx <= 32:
            break
        mx //= 2
    if args.warmup > 1:
        st, _, _ = orc.stepping(st, nsteps=args.warmup - 1, ntime0=2)
    t0 = time.perf_counter()
    orc.stepping(st, nsteps=args.steps, ntime0=1 + args.warmup)
    dt = time.perf_counter() - t0
    cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    v = d.cells * args.steps / dt / 1e6
    sample = (f"bounded sample of the workload: {mx}x{mx}x{d.nz} interior cells ({d.cells} cells, "
              f"{d.cells / cfg['interior_cells']:.4f} of the workload) with the same dz profile, spacing, fields and "
              f"scheme; {args.warmup} warm-up + {args.steps} timed steps, {dt:.1f} s timed; ms_per_step is per step of "
              f"the sample")
    line = {"impl": "reference", "metric": metric, "value": v, "unit": "Mcell-updates/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64)", "config": cfg,
            "sample": {"maxx": mx, "maxy": mx, "nz": d.nz, "cells": d.cells, "reduced_size": mx != args.maxx},
            "cpu_baseline": {"value": v, "unit": "Mcell-updates/s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "Mcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mimica", choices=["mimica", "reference"])
    ap.add_argument("--scheme", default="weno", choices=["weno", "ppm", "muscl", "lw", "quick"])
    ap.add_argument("--maxx", type=int, default=512)
    ap.add_argument("--nz", type=int, default=256)
    ap.add_argument("--limiter", default="minmod", choices=["minmod", "VL", "MC", "default"],
                    help="MUSCL limiter (the reference's muscllimiter; module default minmod)")
    ap.add_argument("--cpu-sample-xy", type=int, default=64)
    ap.add_argument("--ref-sample-xy", type=int, default=256,
                    help="--impl reference: horizontal size of the sample (halved until W+K steps fit --ref-seconds)")
    ap.add_argument("--ref-seconds", type=float, default=150.0)
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="wall time the CPU sample is sized to (steps of the 64x64xnz sample, 1 to 20)")
    ap.add_argument("--e2e-steps", type=int, default=6)
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--form", default="both", choices=["both", "fp64", "mixed"],
                    help="both (default): the plain FP64 form is the headline, the mixed form (FP32 "
                         "stencils/fluxes/spectra, FP64 state) is reported beside it with its error against "
                         "the FP64 form; fp64 / mixed: one form only")
    ap.add_argument("--workload", default="cumulus", choices=["cumulus", "ensemble", "capacity", "acoustic"],
                    help="cumulus: the 512x512x256 shallow-cumulus domain (default); ensemble: 64 independent "
                         "warm-bubble domains of seeded uneven sizes, batched per GPU, sharded over ranks; "
                         "capacity: one 1024x1024x256 domain with 3 momentum + density + 12 scalars (mixed form); "
                         "acoustic: the compressible model's acoustic sub-steps (prognostic_pressure) on "
                         "--maxx x --maxx x --nz")
    ap.add_argument("--sgs", default="none", choices=["none", "smagorinsky"],
                    help="smagorinsky: SGS turbulence diffusion on (Smagorinsky-Lilly, pran=-0.4, zdec=2400 m, "
                         "surface heat, moisture and momentum fluxes), as the BOMEX template runs it")
    ap.add_argument("--members", type=int, default=64)
    ap.add_argument("--ens-mode", choices=["grouped", "streams"], default="grouped",
                    help="ensemble graphs: one launch per kernel of a stage over all members, or per-member streams")
    ap.add_argument("--autotune", default="on", choices=["on", "off"],
                    help="pick the projection plan and K1's segments by timing before the timed steps")
    ap.add_argument("--traj-steps", type=int, default=200, help="steps of the trajectory adjoint leg (0: off)")
    ap.add_argument("--traj-ckpt", type=int, default=25)
    ap.add_argument("--exact-nsubp", type=int, default=3,
                    help="passes of the exact projection legs (fp64_exact, mixed_exact); 0 or 1: not run")
    ap.add_argument("--err-steps", type=int, default=50,
                    help="steps of the accuracy leg (mixed vs FP64 fields from the same initial state)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3

    if args.impl == "reference":
        # the CPU arm needs no process group: rank 0 runs it, the other ranks exit at once
        ws, rank, local = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0")), 0
        if rank != 0:
            return
    else:
        ws, rank, local = dist_init()
    if args.workload == "ensemble":
        return run_ensemble(args, ws, rank, local)
    if args.workload == "capacity":
        return run_capacity(args, ws, rank, local)
    if args.workload == "acoustic":
        return run_acoustic(args, ws, rank, local)
    metric = "Mcell-updates/s per integrator step (2-stage Heun + projection)"
    lim = f" ({args.limiter} limiter)" if args.scheme == "muscl" else ""
    cfg = {"workload": f"shallow-cumulus domain {args.maxx}x{args.maxx}x{args.nz}, dx=dy=25 m, stretched dz 10->100 m, "
                       f"3 momentum + density + 5 scalars, {args.scheme.upper()}{lim} (reference scheme), FD4 momentum, "
                       f"dt=1 s, nsubp=1",
           "fields": "theta_l 298->310 K, qt 17->4 g/kg, qr/nr/aerosol smooth decreasing profiles; "
                     "seeded Gaussian perturbations below 500 m; u=-8+N(0,0.5), v=N(0,0.5) m/s",
           "form": {"both": "plain FP64 (headline) + mixed", "fp64": "plain FP64",
                    "mixed": "mixed (FP32 stencils, fluxes and spectra; FP64 state)"}[args.form],
           "scheme": args.scheme, "sgs": sgs_label(args), "interior_cells": args.maxx * args.maxx * args.nz,
           "l2": "inputs larger than L2 (~16 GB working set)", "parallelism": f"replicas x{ws}"}
    if args.scheme == "muscl":
        cfg["limiter"] = args.limiter

    if args.impl == "reference":
        return reference_arm(args, cfg, metric, ws)

    from fdd3260_b200 import Mimica, _lib, config
    d = config.cumulus_domain(args.maxx, args.maxx, args.nz, scheme=args.scheme, muscl_limiter=args.limiter)
    d.sgs = bench_sgs(args, d)

    st = config.cumulus_state(d, seed=1000 + rank, n_extra=3)
    use_graph = not args.no_graph
    dev = local if ws > 1 else 0
    forms = ["fp64", "mixed"] if args.form == "both" else [args.form]
    # the exact projection: the reference's own nsubp loop (pressure_solver.f90:100-111),
    # each pass solving for the physical divergence of the corrected momentum (caldiv,
    # gradients.f90:986-1052), run to exact_nsubp passes; in the mixed form every pass is an
    # FP32 solve against an FP64 divergence, with no refinement against the Poisson operator.
    # fp64_exact is only run for its fields (the reference for mixed_exact's error).
    if args.form == "both" and args.exact_nsubp > 1 and args.err_steps > 0:
        forms += ["fp64_exact", "mixed_exact"]
    spec = {"fp64": (_lib.MG_PREC_FP64, 1, d.refine_iters), "mixed": (_lib.MG_PREC_MIXED, 1, d.refine_iters),
            "fp64_exact": (_lib.MG_PREC_FP64, args.exact_nsubp, 0),
            "mixed_exact": (_lib.MG_PREC_MIXED, args.exact_nsubp, 0)}
    res = {}
    ref = {}
    for form in forms:
        d.precision, d.nsubp, d.refine_iters = spec[form]
        m = Mimica(d, nscal=len(st.scal), iqt=st.iqt, device=dev)
        r = {}
        # accuracy leg: err_steps steps from the initial state, fields downloaded; the mixed
        # form is compared with the plain FP64 form (bit-exact with the CPU restatement of
        # the reference routines), the mixed exact form with the FP64 exact form
        if args.err_steps > 0 and len(forms) >= 2:
            m.upload(st)
            md, _ = m.stepping(args.err_steps, ntime0=1, diagnostics=True, graph=use_graph)
            out = m.download()
            r["maxdiv"] = md
            if form == "fp64":
                ref["fp64"] = out
                # FP64 twin: the same run from u perturbed by 1e-9 relative (seeded).  The
                # reference's WENO3 switch is discontinuous, so any perturbation of about
                # this size flips faces and the trajectories separate along the flow's own
                # sensitivity; this is the floor against which the mixed error is read.
                tw = config.State(st.u * (1.0 + 1e-9 * np.random.default_rng(99).standard_normal(st.u.shape)),
                                  st.v, st.w, st.p, st.dens, st.scal, st.iqt)
                m.upload(tw)
                del tw
                m.stepping(args.err_steps, ntime0=1, graph=use_graph)
                twin = m.download()
                r["twin_error"] = field_errors(twin, ref["fp64"], st, args.err_steps)
                del twin
            elif form == "mixed":
                r["error_vs_fp64"] = field_errors(out, ref["fp64"], st, args.err_steps)
            elif form == "fp64_exact":
                r["departure_from_one_pass"] = field_errors(out, ref["fp64"], st, args.err_steps)
                ref["fp64_exact"] = out
            else:
                r["error_vs_fp64_exact"] = field_errors(out, ref["fp64_exact"], st, args.err_steps)
                r["departure_from_one_pass"] = field_errors(out, ref["fp64"], st, args.err_steps)
            del out
        if form != "fp64_exact":
            m.upload(st)
            r.update(time_form(args, m, d, st, use_graph, ws, local))
        if form == "fp64" and args.scheme == "weno":
            r["adjoint"] = adjoint_leg(m)
            if args.traj_steps > 0:
                r["adjoint"]["trajectory"] = trajectory_leg(args, dev)
        if form == forms[0]:
            r.update(e2e_leg(args, m, d, st, ws))
        r["device_bytes"] = m.device_bytes
        m.close()
        res[form] = r
    ref = None
    d.precision, d.nsubp, d.refine_iters = spec[forms[0]]

    cpu = None
    if rank == 0 and not args.skip_cpu:
        try:
            v, cores, sample = cpu_reference(args, d, args.scheme)
            cpu = {"value": v, "unit": "Mcell-updates/s", "cores": cores, "kind": "port", "sample": sample}
        except Exception as e:  # pragma: no cover
            cpu = {"value": None, "unit": "Mcell-updates/s", "cores": 0, "kind": "port", "sample": f"failed: {e}"}

    if rank == 0:
        head = res[forms[0]]
        line = {"metric": metric, "value": head["value"], "unit": "Mcell-updates/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if forms[0] == "fp64" else "f32 fluxes/spectra, f64 state",
                "data": "synthetic (seeded PCG64)", "config": cfg,
                "clocks": head["clocks"], "gpu_launches": head["gpu_launches"],
                "e2e": head["e2e"], "roofline": head["roofline"], "kernel_share": head["kernel_share"],
                "cpu_baseline": cpu, "graph": use_graph, "device_bytes": head["device_bytes"],
                "projection_plan": head["projection_plan"]}
        if "mixed" in res and forms[0] != "mixed":
            mx = res["mixed"]
            line["mixed"] = {"form": "FP32 stencils, fluxes and spectra; FP64 state, tendencies, tridiagonal, "
                                     f"residual; refinement passes <= {d.refine_iters}, tol {d.refine_tol} 1/s",
                             "value": mx["value"], "unit": "Mcell-updates/s", "ms_per_step": mx["ms_per_step"],
                             "speedup_vs_fp64": mx["value"] / head["value"], "roofline": mx["roofline"],
                             "kernel_share": mx["kernel_share"], "clocks": mx["clocks"],
                             "gpu_launches": mx["gpu_launches"], "projection_plan": mx["projection_plan"]}
            if "error_vs_fp64" in mx:
                line["mixed"]["error_vs_fp64"] = mx["error_vs_fp64"]
                line["mixed"]["fp64_twin_1e-9_error"] = head.get("twin_error")
                line["mixed"]["maxdiv"] = mx["maxdiv"]
                line["mixed"]["maxdiv_fp64"] = head.get("maxdiv")
        if "mixed_exact" in res:
            mx, fx = res["mixed_exact"], res["fp64_exact"]
            line["mixed_exact"] = {
                "form": f"exact projection: {args.exact_nsubp} passes of the reference's nsubp loop, each an FP32 "
                        "solve for the FP64 physical divergence of the corrected momentum; FP32 stencils, fluxes "
                        "and spectra, FP64 state",
                "value": mx["value"], "unit": "Mcell-updates/s", "ms_per_step": mx["ms_per_step"],
                "speedup_vs_fp64": mx["value"] / head["value"], "roofline": mx["roofline"],
                "kernel_share": mx["kernel_share"], "clocks": mx["clocks"], "gpu_launches": mx["gpu_launches"],
                "maxdiv": mx["maxdiv"], "maxdiv_fp64_exact": fx["maxdiv"],
                "error_vs_fp64_exact": mx["error_vs_fp64_exact"],
                "departure_from_one_pass": mx["departure_from_one_pass"],
                "fp64_exact_departure_from_one_pass": fx["departure_from_one_pass"]}
        if "adjoint" in head:
            line["adjoint"] = head["adjoint"]
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_ensemble(args, ws, rank, local):
    """Batched ensemble: the members are sharded over the ranks by cell count (no
    collective on the data path); each rank advances its members with one graph launch
    per step pair; value = all ranks' cell updates / max over ranks of the device time."""
    from fdd3260_b200 import Mimica, _lib
    from fdd3260_b200 import ensemble as E
    specs = E.ensemble_specs(args.members, seed=3000)
    total_cells = sum(s.cells for s in specs)
    form = "mixed" if args.form == "mixed" else "fp64"
    prec = _lib.MG_PREC_MIXED if form == "mixed" else _lib.MG_PREC_FP64
    dev = local if ws > 1 else 0
    members, states, plans = [], [], {}

    def build(mine):
        for sp in mine:
            d, st = E.member_problem(sp, precision=prec)
            m = Mimica(d, nscal=len(st.scal), iqt=st.iqt, device=dev)
            m.upload(st)
            members.append(m)
            states.append(st)
        ens = E.Ensemble(members, mode=args.ens_mode)
        if args.autotune == "on":
            plans.update(ens.autotune(reps=3))
        return ens

    clk = ClockSampler(local)
    sh = E.shard_and_time(specs, rank, ws, build, args.warmup, args.steps, barrier=lambda: dist_barrier(ws),
                          reduce_max=lambda x: dist_max(x, ws), reduce_sum=lambda x: dist_sum(x, ws), timed_region=clk)
    ens, parts, t_ms = sh["stepper"], sh["parts"], sh["t_ms"]
    value = total_cells * args.steps / (t_ms / 1e3) / 1e6
    launches = ens.launches_per_step
    # the other recording mode on the same members, same step count, for comparison
    other = "streams" if args.ens_mode == "grouped" else "grouped"
    cmp_ = None
    try:
        ens.mode = other
    except Exception as ex:   # members that cannot share grouped launches
        cmp_ = {"mode": other, "unavailable": str(ex)}
    if cmp_ is None:
        t1 = 1 + args.warmup + args.steps
        ens.step(2, ntime0=t1)   # records the pair graph at the timed parity
        dist_barrier(ws)
        ms_o = dist_max(ens.time_steps(args.steps, ntime0=t1 + 2), ws)
        cmp_ = {"mode": other, "value": total_cells * args.steps / (ms_o / 1e3) / 1e6,
                "ms_per_step": ms_o / args.steps, "gpu_launches_per_step": ens.launches_per_step}
        ens.mode = args.ens_mode
    # roofline of the dominant kernel, from an eager profiled pass of this rank's largest member
    big = max(range(len(members)), key=lambda q: members[q].domain.cells)
    mb = members[big]
    L = mb._L
    L.mg_profile_enable(mb._h, 1)
    mb.stepping(2, ntime0=1 + args.warmup + args.steps)
    buf = C.create_string_buffer(8192)
    L.mg_profile_report(mb._h, buf, 8192)
    L.mg_profile_enable(mb._h, 0)
    kern = {ln.split()[0]: (int(ln.split()[1]), float(ln.split()[2])) for ln in buf.value.decode().splitlines()}
    ab = alg_bytes(1 + len(states[big].scal), mb.domain.nsubp)
    pk, pk_src = peaks()
    dom = max((k for k in kern if k in ab), key=lambda k: kern[k][1])
    avg_ms = kern[dom][1] / kern[dom][0]
    achieved = ab[dom] * mb.domain.cells / (avg_ms / 1e3) / 1e9
    # the traffic captures are of a warm-bubble member (two scalars) and of the 5-scalar
    # cumulus workload; the profiled member's own field count and SGS setting decide which
    # applies
    nsc = len(states[big].scal)
    plain = args.scheme == "weno" and getattr(mb.domain, "sgs", None) is None
    table, src = ((MEMBER_TRAFFIC_PER_CELL, MEMBER_TRAFFIC_SOURCE) if nsc == 2 else
                  (MEASURED_TRAFFIC_PER_CELL, TRAFFIC_SOURCE) if nsc == 5 else (None, None))
    measured = plain and table is not None and dom in table
    traffic = table[dom] * mb.domain.cells if measured else None
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "traffic": traffic, "traffic_unit": "bytes per launch",
            "traffic_source": src if measured else "no capture of this configuration",
            "peak_source": pk_src, "algorithmic_bytes_per_cell": ab[dom], "avg_launch_ms": avg_ms,
            "measured_on": f"largest member of rank 0 ({mb.domain.maxx}x{mb.domain.maxy}x{mb.domain.nz}), eager",
            "step_frac": ab["step"] * total_cells * args.steps / (t_ms / 1e3) / 1e9 / pk["hbm_gbs"] / ws}
    # end to end: every member's state uploaded, one ensemble step, every state downloaded
    # into the same page-locked buffers
    from fdd3260_b200 import config
    hosts = []
    for m, st in zip(members, states):
        h = config.State(*[pinned_like(m.domain.shape) for _ in range(5)], [pinned_like(m.domain.shape) for _ in st.scal],
                         st.iqt)
        for a, b in zip([h.u, h.v, h.w, h.p, h.dens, *h.scal], [st.u, st.v, st.w, st.p, st.dens, *st.scal]):
            a[...] = b
        hosts.append(h)
    dist_barrier(ws)
    t0 = time.perf_counter()
    nbytes = 0
    for s_ in range(args.e2e_steps):
        for m, h in zip(members, hosts):
            m.upload(h)
        ens.step(1, ntime0=1)
        for m, h in zip(members, hosts):
            m.download(out=h)
        nbytes = sum((5 + len(st.scal)) * m.domain.nx * m.domain.ny * m.domain.nz * 8 for m, st in zip(members, states))
    e2e_s = dist_max(time.perf_counter() - t0, ws)
    nbytes_all = dist_sum(nbytes, ws)
    ens.close()
    cpu = None
    if rank == 0 and not args.skip_cpu:
        from oracle import oracle as O
        sp = min(specs, key=lambda q: q.cells)
        d, st = E.member_problem(sp)
        orc = O.Oracle(d, omp=True)
        n, dt = timed_cpu_sample(orc, st, args.cpu_seconds)
        cores = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
        cpu = {"value": d.cells * n / dt / 1e6, "unit": "Mcell-updates/s", "cores": cores, "kind": "port",
               "sample": f"smallest member {d.maxx}x{d.maxy}x{d.nz}, {n} step(s) in {dt:.1f} s"}
    for m in members:
        m.close()
    if rank == 0:
        line = {"metric": "Mcell-updates/s per integrator step (2-stage Heun + projection), batched ensemble",
                "value": value, "unit": "Mcell-updates/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": t_ms / args.steps, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f64" if form == "fp64" else "f32 fluxes/spectra, f64 state",
                "data": "synthetic (seeded PCG64)",
                "config": {"workload": f"ensemble of {len(specs)} dry warm bubbles, nx=ny in {E.NX_CHOICES}, "
                                       f"nz in {E.NZ_CHOICES} (seeded), dx=dy=50 m, dz=40 m, WENO, FD4, dt=0.5 s",
                           "total_cells": total_cells, "members_per_rank": [len(p) for p in parts],
                           "form": form, "parallelism": f"members sharded over {ws} rank(s), no collective",
                           "l2": "inputs larger than L2", "ensemble_mode": args.ens_mode},
                "other_mode": cmp_,
                "clocks": clk.summary(), "gpu_launches": launches * args.steps,
                "e2e": {"value": total_cells * args.e2e_steps / e2e_s / 1e6, "unit": "Mcell-updates/s",
                        "h2d_bytes_per_step": nbytes_all, "d2h_bytes_per_step": nbytes_all,
                        "timing": f"host wall clock, synchronised, host buffers: {host_buffers()}",
                        "host_buffers": host_buffers()},
                "roofline": roof, "cpu_baseline": cpu, "graph": True,
                "projection_plans": {k: {f: v[f] for f in ("x_radix", "y_radix", "x_threads", "y_threads", "tri_block",
                                                           "ms_default", "ms_tuned") if f in v}
                                     for k, v in plans.items()}}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_capacity(args, ws, rank, local):
    """The capacity run: one 1024 x 1024 x 256 domain (dx = dy = 20 m, the cumulus tanh dz,
    dt = 0.5 s) with 3 momentum fields, density and 12 scalars (theta_l, qt and 10 lognormal
    tracers, sigma_log = 1), WENO, in the mixed form with the refined Poisson solve (or
    --form fp64).  The state is generated and uploaded one field at a time, so the host
    never holds more than one 2.2 GB field; the context holds the rest on the device."""
    from types import SimpleNamespace

    from fdd3260_b200 import Mimica, _lib, config
    form = "fp64" if args.form == "fp64" else "mixed"
    d = config.cumulus_domain(1024, 1024, 256, dx=20.0, dy=20.0, dt0=0.5, scheme=args.scheme,
                              muscl_limiter=args.limiter)
    d.precision = _lib.MG_PREC_MIXED if form == "mixed" else _lib.MG_PREC_FP64
    nscal = 12
    dev = local if ws > 1 else 0
    m = Mimica(d, nscal=nscal, iqt=1, device=dev)
    t0 = time.perf_counter()
    for f in range(_lib.MG_FIELD_SCAL + nscal):
        m.upload_field(f, config.cumulus_field(d, f, seed=4000 + rank))
    t_up = time.perf_counter() - t0
    st = SimpleNamespace(scal=[None] * nscal)
    r = time_form(args, m, d, st, not args.no_graph, ws, local)
    md, _ = m.stepping(1, ntime0=2 + args.warmup + args.steps, diagnostics=True, graph=False)
    dev_bytes = m.device_bytes
    m.close()
    if rank == 0:
        line = {"metric": "Mcell-updates/s per integrator step (2-stage Heun + projection), capacity run",
                "value": r["value"], "unit": "Mcell-updates/s", "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64" if form == "fp64" else "f32 fluxes/spectra, f64 state",
                "data": "synthetic (seeded PCG64, one stream per field)",
                "config": {"workload": "capacity domain 1024x1024x256, dx=dy=20 m, stretched dz 10->100 m, "
                                       f"3 momentum + density + 12 scalars, {args.scheme.upper()}, FD4, dt=0.5 s",
                           "form": form, "interior_cells": d.cells, "parallelism": f"replicas x{ws}",
                           "l2": "inputs larger than L2"},
                "clocks": r["clocks"], "gpu_launches": r["gpu_launches"], "roofline": r["roofline"],
                "kernel_share": r["kernel_share"], "projection_plan": r["projection_plan"],
                "device_bytes": dev_bytes, "maxdiv_after": md, "upload_s": t_up,
                "e2e": None, "e2e_note": "not measured: 15 fields of 2.2 GB cross the bus each way per step",
                "cpu_baseline": None}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


# algorithmic HBM bytes per interior cell of one acoustic sub-step (FP64), with nscal
# passive scalars: the scalar kernel (advection, integ_scal, equation of state,
# divergence) reads dens, es, uadv, vadv, wadv, sdens, ses, sqt, tdens, tes, tqt, qt, u,
# v, w and writes dens', es', tdens, tes, tqt, qt, p, cs2, div (24 fields); the momentum
# kernel reads p, div, dens, su, sv, sw, tu, tv, tw, u, v, w and writes tu, tv, tw, u, v,
# w (18); each passive scalar reads sscal, tscal, scal and writes tscal, scal (5)
# measured DRAM bytes per interior cell of one sub-step with one passive scalar:
# ac_scal_kernel 230 + ac_mom_kernel 138 (ncu, 256x256x64)
ACOUSTIC_TRAFFIC_PER_CELL = 230.0 + 138.0


def acoustic_alg_bytes(nscal: int) -> int:
    return 8 * (24 + 18 + 5 * nscal)


def run_acoustic(args, ws, rank, local):
    """The compressible model's acoustic sub-steps (prognostic_pressure.f90, dry ISENTROPIC
    CONSERVATIVE build) on one domain per rank: ntau = 8 sub-steps of stage 1 per call,
    W untimed and K timed calls on the resident fields (device time, CUDA events),
    value = all ranks' cell sub-steps / max over ranks of the time."""
    from fdd3260_b200 import Mimica, acoustic, config
    dev = local if ws > 1 else 0
    d = config.warm_bubble_domain(args.maxx, args.maxx, args.nz, dx=50.0, dy=50.0, dz=40.0, dt0=0.5,
                                  scheme=args.scheme)
    nscal, ntau = 1, 8
    inp, st = acoustic.acoustic_case(d, seed=31 + rank, im=1, ntau=ntau, nscal=nscal)
    with Mimica(d, nscal=1, device=dev) as m:
        dist_barrier(ws)
        with ClockSampler(local) as clk:
            _, ms = m.prognostic_pressure(inp, st, reps=args.steps, warmup=args.warmup)
        # end to end: one call from host arrays (upload, ntau sub-steps, download)
        t0 = time.perf_counter()
        m.prognostic_pressure(inp, st)
        e2e_s = time.perf_counter() - t0
    ms = dist_max(ms, ws)
    e2e_s = dist_max(e2e_s, ws)
    cells = d.cells
    value = ws * cells * ntau / (ms / 1e3) / 1e6
    pk, pk_src = peaks()
    ab = acoustic_alg_bytes(nscal)
    achieved = ab * cells * ntau / (ms / 1e3) / 1e9
    nio = 16 + 3 * nscal   # host arrays uploaded (inputs and state) and 14 + 2 nscal downloaded
    cpu = None
    if rank == 0 and not args.skip_cpu:
        from oracle import oracle as O
        ds = config.warm_bubble_domain(64, 64, args.nz, dx=50.0, dy=50.0, dz=40.0, dt0=0.5, scheme=args.scheme)
        si, ss = acoustic.acoustic_case(ds, seed=31, im=1, ntau=ntau, nscal=nscal)
        orc = O.Oracle(ds)
        orc.prognostic_pressure(si, ss)
        n, t0 = 0, time.perf_counter()
        while time.perf_counter() - t0 < min(args.cpu_seconds, 20.0) and n < 20:
            orc.prognostic_pressure(si, ss)
            n += 1
        dt = time.perf_counter() - t0
        cpu = {"value": ds.cells * ntau * n / dt / 1e6, "unit": "Mcell-substeps/s", "cores": 1, "kind": "port",
               "sample": f"64x64x{args.nz} interior cells, {n} call(s) of {ntau} sub-steps in {dt:.1f} s"}
    if rank == 0:
        line = {"metric": "Mcell-substeps/s of the compressible acoustic sub-steps (prognostic_pressure)",
                "value": value, "unit": "Mcell-substeps/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": ms, "step": f"one call: {ntau} acoustic sub-steps", "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded PCG64)",
                "config": {"workload": f"compressible acoustic sub-steps {args.maxx}x{args.maxx}x{args.nz}, "
                                       f"dx=dy=50 m, dz=40 m, dt0=0.5 s, ntau={ntau}, stage 1, density + es + qt + "
                                       f"{nscal} passive scalar, "
                                       f"{'QUICK' if args.scheme == 'quick' else 'Lax-Wendroff'} faces without limiter",
                           "interior_cells": cells, "parallelism": f"replicas x{ws}", "l2": "inputs larger than L2"},
                "clocks": clk.summary(), "gpu_launches": args.steps * (1 + ntau * 5),
                "roofline": {"bound": "hbm", "kernel": "acoustic sub-step (2 kernels + ghost refreshes and level sums)",
                             "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                             "frac": achieved / pk["hbm_gbs"],
                             "traffic": ACOUSTIC_TRAFFIC_PER_CELL * cells if nscal == 1 else None,
                             "traffic_unit": "bytes per sub-step",
                             "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of ac_scal_kernel and "
                                               "ac_mom_kernel at 256x256x64 with 1 passive scalar "
                                               "(profiles/acoustic_substep_256x256x64.md), per interior cell, times "
                                               "this domain's cells",
                             "peak_source": pk_src, "algorithmic_bytes_per_cell": ab},
                "e2e": {"value": ws * cells * ntau / e2e_s / 1e6, "unit": "Mcell-substeps/s",
                        "h2d_bytes_per_step": nio * d.nx * d.ny * d.nz * 8,
                        "d2h_bytes_per_step": (14 + 2 * nscal) * d.nx * d.ny * d.nz * 8,
                        "timing": "host wall clock of one mg_prognostic_pressure call from pageable numpy arrays"},
                "cpu_baseline": cpu}
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def adjoint_leg(m, reps: int = 3) -> dict:
    """Device time of the hand-written tangent-linear and adjoint kernels against their
    forward operators, on copies of the resident state (mg_time_adjoint)."""
    out = (C.c_double * 5)()
    rc = m._L.mg_time_adjoint(m._h, reps, out)
    if rc:
        return {"error": rc}
    f = list(out)
    return {"advection_fwd_ms": f[0], "advection_tl_ms": f[1], "advection_ad_ms": f[2],
            "advection_ad_over_fwd": f[2] / f[0], "projection_fwd_ms": f[3], "projection_ad_ms": f[4],
            "projection_ad_over_fwd": f[4] / f[3],
            "note": "operator level: one density-weighted field (WENO) and one anelastic_pressure call"}


def trajectory_leg(args, dev) -> dict:
    """Checkpointed trajectory adjoint against the forward model on the adjoint workload:
    128 x 128 x 96 cells at 40 m, a dry warm bubble (u, v, w, theta; density carried),
    traj_steps steps with a checkpoint every traj_ckpt steps.  Device times with CUDA
    events: the production step (graph), the composition the linearisation follows, its
    tangent linear, and the adjoint including its forward sweep and recomputation."""
    from fdd3260_b200 import Mimica, config
    d = config.warm_bubble_domain(128, 128, 96, dx=40.0, dy=40.0, dz=40.0, dt0=0.5)
    st = config.warm_bubble_state(d, seed=1002, centre=(2560.0, 2560.0, 800.0), radius=600.0, nscal_passive=0)
    n, ck = args.traj_steps, args.traj_ckpt
    with Mimica(d, nscal=len(st.scal), device=dev) as m:
        m.upload(st)
        m.time_traj(2, 1)   # warm-up: plans, buffers, first launches
        t = m.time_traj(n, ck)
        t1 = m.time_traj(n, n)   # one segment: no recomputation (memory permitting)
        m.upload(st)
        ms = C.c_double(0.0)
        m.stepping(3, ntime0=1, graph=True)
        rc = m._L.mg_time_steps(m._h, n, 4, 1, C.byref(ms))
        if rc:
            raise RuntimeError(f"mg_time_steps failed: {rc}")
    fwd = ms.value
    return {"workload": "warm bubble 128x128x96 at 40 m, dry (u, v, w, theta, density), WENO3 switch, FD4",
            "steps": n, "ckpt": ck, "step_ms": fwd, "composition_ms": t["forward_ms"], "tl_ms": t["tl_ms"],
            "adjoint_ms": t["adjoint_ms"], "adjoint_over_fwd": t["adjoint_ms"] / fwd,
            "adjoint_over_composition": t["adjoint_ms"] / t["forward_ms"], "tl_over_fwd": t["tl_ms"] / fwd,
            "adjoint_device_gb": t["adjoint_device_bytes"] / 1e9,
            "one_segment": {"ckpt": n, "adjoint_ms": t1["adjoint_ms"], "adjoint_over_fwd": t1["adjoint_ms"] / fwd,
                            "adjoint_device_gb": t1["adjoint_device_bytes"] / 1e9},
            "note": "adjoint_ms includes the forward sweep that stores checkpoints and the segment recomputation"}


def field_errors(out, ref, st0, nsteps: int) -> dict:
    """Per-field relative L2 error over the interior: against the FP64 field, and against
    the change the FP64 form made over the run."""
    rel, relc = {}, {}
    names = [("u", out.u, ref.u, st0.u), ("v", out.v, ref.v, st0.v), ("w", out.w, ref.w, st0.w),
             ("p", out.p, ref.p, st0.p), ("dens", out.dens, ref.dens, st0.dens)]
    names += [(f"s{i}", a, b, c) for i, (a, b, c) in enumerate(zip(out.scal, ref.scal, st0.scal))]
    for name, a, b, c in names:
        a, b, c = a[:, 3:-2, 3:-2], b[:, 3:-2, 3:-2], c[:, 3:-2, 3:-2]
        e = float(np.linalg.norm(a - b))
        rel[name] = e / max(float(np.linalg.norm(b)), 1e-300)
        relc[name] = e / max(float(np.linalg.norm(b - c)), 1e-300)
    return {"steps": nsteps, "rel_l2": rel, "rel_l2_of_change": relc}


def time_form(args, m, d, st, use_graph, ws, local) -> dict:
    L = m._L
    plan = m.autotune(reps=3) if args.autotune == "on" else dict(m.tune_get(), source="default")
    # W warm-up steps; the last two form a pair at the timed region's step parity, so the
    # pair graph the timed steps replay (the momentum direction order alternates with the
    # step's parity) is recorded inside the warm-up
    m.stepping(args.warmup - 2, ntime0=1, graph=use_graph)
    m.stepping(2, ntime0=args.warmup - 1, graph=use_graph)
    m.synchronize()
    # timed region (device time, CUDA events on the library stream), clocks sampled meanwhile
    dist_barrier(ws)
    ms = C.c_double(0.0)
    with ClockSampler(local) as clk:
        rc = L.mg_time_steps(m._h, args.steps, 1 + args.warmup, 1 if use_graph else 0, C.byref(ms))
    if rc:
        raise RuntimeError(f"mg_time_steps failed: {rc}")
    t_ms = dist_max(ms.value, ws)
    value = d.cells * args.steps / (t_ms / 1e3) / 1e6 * ws
    launches_per_step = m.launches_per_call

    # per-kernel device times (separate eager pass, events around each launch group)
    L.mg_profile_enable(m._h, 1)
    m.stepping(2, ntime0=1 + args.warmup + args.steps)
    buf = C.create_string_buffer(8192)
    L.mg_profile_report(m._h, buf, 8192)
    L.mg_profile_enable(m._h, 0)
    kern = {}
    for ln in buf.value.decode().splitlines():
        name, n, tot = ln.split()
        kern[name] = {"launches": int(n), "total_ms": float(tot)}
    ab = alg_bytes(1 + len(st.scal), d.nsubp, d.sgs is not None)
    pk, pk_src = peaks()
    dom = max((k for k in kern if k in ab), key=lambda k: kern[k]["total_ms"])
    avg_ms = kern[dom]["total_ms"] / kern[dom]["launches"]
    achieved = ab[dom] * d.cells / (avg_ms / 1e3) / 1e9
    measured = args.scheme == "weno" and len(st.scal) == 5 and d.sgs is None and dom in MEASURED_TRAFFIC_PER_CELL
    traffic = MEASURED_TRAFFIC_PER_CELL[dom] * d.cells if measured else None
    roof = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": achieved / pk["hbm_gbs"], "traffic": traffic, "traffic_unit": "bytes per launch",
            "traffic_source": TRAFFIC_SOURCE if measured else "no capture of this configuration",
            "peak_source": pk_src, "algorithmic_bytes_per_cell": ab[dom], "avg_launch_ms": avg_ms,
            "step_alg_bytes_per_cell": ab["step"],
            "step_frac": ab["step"] * d.cells * args.steps / (t_ms / 1e3) / 1e9 / pk["hbm_gbs"]}
    kshare = {k: round(v["total_ms"] / sum(x["total_ms"] for x in kern.values()), 4) for k, v in kern.items()}
    return {"value": value, "ms_per_step": t_ms / args.steps, "clocks": clk.summary(),
            "gpu_launches": launches_per_step * args.steps, "roofline": roof, "kernel_share": kshare,
            "projection_plan": plan}


def e2e_leg(args, m, d, st, ws) -> dict:
    """End to end through the public API with page-locked host buffers: every step uploads
    its state, steps once and downloads the result.  Two ways:
      serial     one context, upload -> step -> download, step after step;
      pipelined  two contexts (two device states, two streams) driven by two host threads,
                 the second started one upload later, so that one context's download
                 (device to host) overlaps the other's upload (host to device) on the
                 full-duplex bus.  Every step still moves its whole state both ways.
    `value` is the pipelined figure; the serial one is reported beside it."""
    import threading

    from fdd3260_b200 import Mimica, config

    def host_state():
        host = {n: pinned_like(d.shape) for n in ("u", "v", "w", "p", "dens")}
        hscal = [pinned_like(d.shape) for _ in st.scal]
        for n in ("u", "v", "w", "p", "dens"):
            host[n][...] = getattr(st, n)
        for a, b in zip(hscal, st.scal):
            a[...] = b
        return config.State(host["u"], host["v"], host["w"], host["p"], host["dens"], hscal, st.iqt)

    hstate = host_state()
    m.upload(hstate)
    m.stepping(1, ntime0=1)
    m.synchronize()
    dist_barrier(ws)
    t0 = time.perf_counter()
    for s in range(args.e2e_steps):
        m.upload(hstate)
        m.stepping(1, ntime0=2 + s)
        m.download(out=hstate)
    m.synchronize()
    serial_s = dist_max(time.perf_counter() - t0, ws)
    nbytes = (5 + len(st.scal)) * d.nx * d.ny * d.nz * 8
    # pipelined: a second context with the same plan
    m2 = Mimica(d, nscal=len(st.scal), iqt=st.iqt, device=m.device)
    try:
        m2.tune_set(m.tune_get())
        h2 = host_state()
        m2.upload(h2)
        m2.stepping(1, ntime0=1)
        m2.synchronize()
        uploaded = threading.Event()
        errs = []

        def drive(mm, hs, first):
            try:
                for s in range(args.e2e_steps):
                    mm.upload(hs)
                    if first and s == 0:
                        uploaded.set()
                    mm.stepping(1, ntime0=2 + s)
                    mm.download(out=hs)
                mm.synchronize()
            except Exception as ex:   # pragma: no cover
                errs.append(ex)
                uploaded.set()

        dist_barrier(ws)
        t0 = time.perf_counter()
        ta = threading.Thread(target=drive, args=(m, hstate, True))
        tb = threading.Thread(target=lambda: (uploaded.wait(), drive(m2, h2, False)))
        ta.start()
        tb.start()
        ta.join()
        tb.join()
        pipe_s = dist_max(time.perf_counter() - t0, ws)
        if errs:
            raise errs[0]
    finally:
        m2.close()
    serial = d.cells * args.e2e_steps * ws / serial_s / 1e6
    pipelined = 2 * d.cells * args.e2e_steps * ws / pipe_s / 1e6
    return {"e2e": {"value": pipelined, "unit": "Mcell-updates/s",
                    "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "serial_value": serial,
                    "timing": "host wall clock, synchronised; every step uploads its whole state from the host "
                              "buffers and downloads its result; value: two contexts in two host threads, one upload "
                              f"apart, {2 * args.e2e_steps} steps; serial_value: one context, {args.e2e_steps} steps; "
                              f"host buffers: {host_buffers()}",
                    "host_buffers": host_buffers()}}


if __name__ == "__main__":
    main()
