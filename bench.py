#!/usr/bin/env python
"""Benchmark of the COMCOT time-stepping hot path on B200.

Workload (default, the configuration the headline metric is quoted on):
C2 -- one linear spherical layer of 2401 x 2001 cells at 1 arc-minute,
dt = 1 s, OPEN boundary on four sides, max-eta recorder and 32 gauges,
seeded synthetic bathymetry (200 seamounts, 2 % land) and dipole source.
A "step" is one outer time step over the whole grid.

value  : cell-updates/s of the batched engine (one fused launch per step,
         state resident in HBM, CUDA-graph replay), device-timed with CUDA
         events on the engine's stream, max over ranks.
e2e    : the same metric through the reference C ABI with host buffers:
         gcomcot_init_layer_ uploads H, Z and the R arrays from host memory,
         then every step runs MASS/OPEN/MOMENT/MAX_AMP through the legacy
         entry points and reads the 32 gauge stencils back to the host, and the
         final surface and max-eta are downloaded.
--impl reference : the reference algorithm's CPU implementation (the
         restated Fortran solvers, all host threads) on the same workload.

Multi-GPU: every rank steps its own replica (independent forecasts shard
with no exchange); value is the sum over ranks (weak scaling).
"""
from __future__ import annotations

import argparse
import json
import os
import pathlib
import statistics
import subprocess
import sys
import threading
import time

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "gpu-comcot_b200"))
os.environ.setdefault("GCOMCOT_QUIET", "1")  # the JSON line is the only stdout

import numpy as np  # noqa: E402

from comcot_b200 import replicas, synth  # noqa: E402

METRIC = "cell-updates/s"
WORKLOADS = {"c1": "C1: 361x301 2' linear spherical, Gaussian hump, OPEN, max-eta, dt 2 s",
             "c2": "C2: 2401x2001 1' linear spherical, OPEN, max-eta, 32 gauges, dt 1 s"}
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_CELL = 36  # Z1,M1,N1,H in + Z2,M2,N2 out (28 B) + max-eta read/write (8 B)


def env_rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(
        os.environ.get("LOCAL_RANK", "0"))


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            d = json.loads(p.read_text())
            return float(d["hbm_gbs"]), "measured"
        except Exception:
            pass
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(name="fused_linear_step_c2.txt", key="traffic_bytes_per_launch"):
    """DRAM bytes (read + write) per launch of a kernel, from its committed ncu summary"""
    f = ROOT / "profiles" / name
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if parts[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(case, budget_s=15.0):
    """FP32 oracle (the restated reference Fortran), one thread, bounded sample."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    o = oracle.OracleRun(case)
    t0 = time.perf_counter()
    o.run(1, threads=1)
    one = time.perf_counter() - t0
    n = max(1, min(case.nsteps, int(budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    o.run(n, threads=1)
    dt = time.perf_counter() - t0
    cells = case.root.nx * case.root.ny
    return {"value": cells * n / dt, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{n} outer steps of the full {case.root.nx}x{case.root.ny} grid, serial oracle "
                      f"(restated Fortran MASS_S/OPEN/MOMT_S + max-eta), {dt:.1f} s"}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    threads = os.cpu_count() or 1
    make_case = synth.config_c1 if args.workload == "c1" else synth.config_c2
    case = make_case(nsteps=args.warmup + args.steps)
    o = oracle.OracleRun(case)
    o.run(max(1, min(args.warmup, 3)), threads=threads)
    t0 = time.perf_counter()
    o.run(1, threads=threads)
    one = time.perf_counter() - t0
    k = max(1, min(args.steps, int(60.0 / max(one, 1e-6))))
    t0 = time.perf_counter()
    o.run(k, threads=threads)
    dt = time.perf_counter() - t0
    cells = case.root.nx * case.root.ny
    v = cells * k / dt
    line = {"metric": METRIC, "value": v, "unit": METRIC, "n_gpus": args.gpus, "steps": k,
            "warmup": args.warmup, "ms_per_step": 1e3 * dt / k, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOADS.get(args.workload, WORKLOADS["c2"])},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": METRIC, "cores": threads, "kind": "port",
                             "sample": f"{k} outer steps of the full grid (of {args.steps} requested; "
                                       f"bounded to ~60 s), restated Fortran solvers on {threads} threads"},
            "e2e": {"value": v, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_c4(args, torch, dist, rank, world, local):
    """C4: 64 dipole scenarios on one 1201x1001 2' grid with shared bathymetry,
    stepped by the batched engine (one fused launch per step over all members,
    CUDA-graph replay), against the plain path: one scenario at a time through
    the reference C ABI with one kernel per phase."""
    from comcot_b200.abi import ReferenceSession
    from comcot_b200.engine import Engine
    from comcot_b200.synth import Case

    L = synth.config_c4_grid()
    nscen = args.scenarios
    run_steps = args.steps  # steps of one forecast (3600 = 2 h at dt 2 s)
    srcs = synth.ensemble_sources(L.x, L.y, nscen, seed=40 + rank)
    case = Case("C4", [L], run_steps)
    tune_reps = 2
    from comcot_b200 import _lib
    ncand = _lib.load().gc_engine_num_candidates()  # tile variants x tile-height rules
    extra = ncand * (tune_reps + 1) + args.warmup  # the autotuner's steps
    eng = Engine(budget=120 << 30)
    eng.config(variant=args.variant, use_graphs=1, chunk=64)
    cls = eng.add_class(L)
    ids = [eng.add(case, z0=z, cls=cls, nsteps=run_steps + extra, gauges=[], arrival_thr=0.05) for z in srcs]
    if args.variant < 0:
        eng.autotune(tune_reps)
    variant = eng.variant()  # variant + variants x tile-height rule
    eng.step(args.warmup)
    eng.prepare()  # step-chunk graph built before the timed region
    eng.sync()
    stream = torch.cuda.ExternalStream(eng.stream())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = eng.launches()
    ev0.record(stream)
    eng.step(run_steps)
    ev1.record(stream)
    ev1.synchronize()
    ck = clocks.stop()
    launches = eng.launches() - l0
    ms = ev0.elapsed_time(ev1)
    ms = replicas.reduce_max(ms, dist, 'cuda')
    cells = L.nx * L.ny
    value_cells = cells * nscen * run_steps * world / (ms * 1e-3)
    scen_per_hour = nscen * world * 3600.0 / (ms * 1e-3)
    eng.close()
    # plain path: a sample of scenarios, each alone through the reference ABI
    plain = None
    if rank == 0 and args.plain_sample > 0:
        t_tot = 0.0
        k = min(args.plain_sample, nscen)
        for q in range(k):
            c1 = Case("C4p", [L], run_steps)
            L.Z0 = srcs[q]
            s = ReferenceSession(c1, fusion=False, init_layers=False)
            st = torch.cuda.ExternalStream(s.stream())
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.init_layers()
            torch.cuda.synchronize()
            a.record(st)
            s.drive(run_steps, maxamp=True)
            b.record(st)
            b.synchronize()
            t_tot += a.elapsed_time(b) * 1e-3
            s.close()
        per = t_tot / k
        plain = {"scenarios_per_hour": 3600.0 / per, "s_per_scenario": per,
                 "sample": f"{k} of {nscen} scenarios run alone, full length, extrapolated per scenario",
                 "path": "reference C ABI, one kernel per phase (mass, open, momentum, max)"}
    peak, peak_kind = peaks()
    bpc = 24.0 + 4.0 / nscen + 8.0  # per member-cell: Z,M,N in/out, shared H, max-eta r/w
    achieved = bpc * cells * nscen / (ms * 1e-3 / run_steps) / 1e9
    line = {"metric": "ensemble scenarios/hour", "value": scen_per_hour, "unit": "scenarios/hour",
            "n_gpus": world, "steps": run_steps, "warmup": args.warmup, "ms_per_step": ms / run_steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"C4: {nscen} dipole scenarios on 1201x1001 2' linear spherical, shared H, "
                                   f"dt 2 s, {run_steps} steps, max-eta + arrival",
                       "parallelism": f"scenario replicas x{world}", "tile_variant": variant,
                       "l2": f"working set {nscen} x 7 fields x 4.9 MB >> 126 MB L2"},
            "cell_updates_per_s": value_cells,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": (None if profiled_traffic("fused_ensemble_step_c4.txt",
                                                              "traffic_bytes_per_member_launch") is None
                                     else nscen * profiled_traffic("fused_ensemble_step_c4.txt",
                                                                   "traffic_bytes_per_member_launch")),
                         "peak_kind": f"{peak_kind} (copy bandwidth)",
                         "algorithmic_bytes_per_launch": bpc * cells * nscen},
            "clocks": ck, "gpu_launches": launches}
    if plain:
        line["plain_path"] = plain
        line["speedup_vs_plain"] = scen_per_hour / plain["scenarios_per_hour"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_c3(args, torch, dist, rank, world, local):
    """C3: two-level nested run -- 1201x1001 2' linear spherical outer grid and
    a 601x501 nonlinear Cartesian child (wet/dry, Manning n = 0.025, ratio 5)
    coupled by JNQ/NEWQ edge fluxes and JNZ feedback every outer step.  value:
    the batched engine's nested path (per-phase kernels in a captured graph);
    e2e: the reference C ABI call sequence with host buffers."""
    from comcot_b200.abi import ReferenceSession
    from comcot_b200.engine import Engine

    total = args.warmup + args.steps
    case = synth.config_c3(nsteps=total)
    P, Cl = case.layers
    cells = P.nx * P.ny + Cl.nx * Cl.ny * Cl.rel_time
    eng = Engine(budget=8 << 30)
    eng.config(variant=args.variant, use_graphs=1, chunk=64)
    eng.add(case)
    eng.step(args.warmup)
    eng.prepare()  # step-chunk graph built before the timed region
    eng.sync()
    stream = torch.cuda.ExternalStream(eng.stream())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = eng.launches()
    ev0.record(stream)
    eng.step(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    ck = clocks.stop()
    launches = eng.launches() - l0
    ms = ev0.elapsed_time(ev1)
    ms = replicas.reduce_max(ms, dist, 'cuda')
    eng.close()
    value = cells * args.steps * world / (ms * 1e-3)
    e2e = None
    if not args.no_e2e:
        case_e = synth.config_c3(nsteps=args.steps)
        s = ReferenceSession(case_e, fusion=True, arrival=True, init_layers=False)
        st = torch.cuda.ExternalStream(s.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        s.init_layers()
        s.drive(args.steps, maxamp=True)
        z, zc, zm = s.getz(1), s.getz(2), s.getzmax(1)
        b.record(st)
        b.synchronize()
        e2e_ms = a.elapsed_time(b)
        s.close()
        fp, fc = P.nx * P.ny * 4, Cl.nx * Cl.ny * 4
        e2e = {"value": cells * args.steps * world / (e2e_ms * 1e-3), "unit": METRIC,
               # the outer grid's H and Z, the child's H, Z, HP and HQ, and the 8-float row records
               "h2d_bytes_per_step": int((2 * fp + 4 * fc + (P.ny + Cl.ny) * 8 * 4) / args.steps),
               "d2h_bytes_per_step": int((2 * fp + fc) / args.steps), "ms_per_step": e2e_ms / args.steps,
               "path": "gcomcot_set_layer_params_/init_layer x2 + per step mass/openbd/all_grid/momt/maxamp/"
                       "update + getz x2/getzmax"}
        del z, zc, zm
    peak, peak_kind = peaks()
    # algorithmic bytes of one outer step: outer grid 28 B + max-eta 8 B + arrival 8 B per cell;
    # child 28 B per cell per sub-step (Z, M, N, H in; Z, M, N out; DZ = Z + H) + JNZ 8 B per child cell
    bstep = 44.0 * P.nx * P.ny + (28.0 * Cl.rel_time + 8.0) * Cl.nx * Cl.ny
    achieved = bstep / (ms * 1e-3 / args.steps) / 1e9
    line = {"metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"C3: 1201x1001 2' linear spherical + {Cl.nx}x{Cl.ny} nonlinear Cartesian "
                                   f"child (r=5, rel_time {Cl.rel_time}, Manning 0.025), dt 2 s",
                       "cells_per_step": cells, "parallelism": f"replicas x{world}",
                       "l2": "working set ~60 MB per step fits the 126 MB L2; no flush (L2 resident)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_kind": f"{peak_kind} (copy bandwidth)",
                         "algorithmic_bytes_per_step": bstep},
            "clocks": ck, "gpu_launches": launches}
    if e2e:
        line["e2e"] = e2e
    if rank == 0 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle

        o = oracle.OracleRun(synth.config_c3(nsteps=total))
        t0 = time.perf_counter()
        o.run(1, threads=1)
        one = time.perf_counter() - t0
        n = max(1, min(total, int(15.0 / max(one, 1e-6))))
        t0 = time.perf_counter()
        o.run(n, threads=1)
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": cells * n / dt, "unit": METRIC, "cores": 1, "kind": "port",
                                "sample": f"{n} outer steps of both layers, serial oracle, {dt:.1f} s"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def run_c5(args, torch, dist, rank, world, local):
    """C5 serving: a seeded Poisson stream of forecast requests (mean 2 req/s;
    outer grids 481x401, 961x801 or 1921x1601 at 2'; 30 % nested with a
    301x251 ratio-5 nonlinear child; 30-120 simulated minutes at dt 2 s; a
    dipole source and 16 gauges each) served by continuous batching with
    admission by HBM footprint.  Reported: p50/p99 time-to-forecast under the
    arrival load, scenarios/hour at saturation, and the same for the plain
    one-request-at-a-time path (its per-class service times measured through
    the reference C ABI with one kernel per phase, then queued FIFO on the
    same arrival times)."""
    from comcot_b200 import serving
    from comcot_b200.abi import ReferenceSession
    from comcot_b200.engine import Engine

    tpl = synth.config_c5_templates()
    # one trace for the whole job; each rank serves its round-robin share
    trace = replicas.shard(synth.poisson_trace(n=args.requests, rate=args.rate, seed=5), rank, world)

    def make_requests():
        return [serving.Request(k, t, synth.c5_request_case(tpl, size, nsteps, nested, seed))
                for k, (t, size, nsteps, nested, seed) in enumerate(trace)]

    reqs = make_requests()
    # tile variant: tuned once on a warm batch of the largest class (not timed)
    variant = args.variant
    if variant < 0:
        big = [r for r in reqs if r.case.root.nx == 1921 and len(r.case.layers) == 1][:4]
        from comcot_b200 import _lib
        with Engine(budget=16 << 30) as eng:
            for r in big:
                eng.add(r.case, nsteps=3 * _lib.load().gc_engine_num_candidates() + 8)
            eng.autotune(2)
            variant = eng.variant()  # variant + variants x tile-height rule
    budget = int(args.budget_gb * (1 << 30))
    # warm-up: a few requests through the server (module load, first graphs)
    with serving.ForecastServer(budget, chunk=args.chunk, variant=variant) as srv:
        warm = [serving.Request(k, 0.0, synth.c5_request_case(tpl, sz, 64, k % 2 == 1, 900 + k))
                for k, sz in enumerate(synth.C5_SIZES)]
        srv.serve(warm, speed=float("inf"))
    torch.cuda.synchronize()
    cell_updates = sum(r.case.nsteps * sum(L.nx * L.ny * L.rel_time for L in r.case.layers) for r in reqs)
    # 1) the arrival load, in real time
    clocks = ClockSampler(local)
    clocks.start()
    with serving.ForecastServer(budget, chunk=args.chunk, variant=variant) as srv:
        l0 = srv.eng.launches()
        srv.serve(reqs, speed=1.0)
        launches = srv.eng.launches() - l0
        max_active, refused = srv.max_active, srv.refused
    ck = clocks.stop()
    lat = np.array([r.latency for r in reqs])
    span = max(r.t_done for r in reqs)
    pl = serving.percentiles(lat)
    # 2) saturation: every request at t = 0
    reqs_sat = make_requests()
    torch.cuda.synchronize()
    with serving.ForecastServer(budget, chunk=args.chunk, variant=variant) as srv:
        t0 = time.perf_counter()
        srv.serve(reqs_sat, speed=float("inf"))
        sat_s = time.perf_counter() - t0
        sat_active = srv.max_active
    capacity = len(reqs_sat) * 3600.0 / sat_s
    # 3) plain path: per class service time through the reference C ABI, one kernel per phase
    plain = None
    if not args.no_plain:
        svc_class = {}
        for size in synth.C5_SIZES:
            for nested in (False, True):
                c = synth.c5_request_case(tpl, size, 200, nested, 7)
                s = ReferenceSession(c, fusion=False, arrival=True, init_layers=False)
                st = torch.cuda.ExternalStream(s.stream())
                ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
                torch.cuda.synchronize()
                ev[0].record(st)
                s.init_layers()
                ev[1].record(st)
                s.drive(20, maxamp=True)
                ev[2].record(st)
                s.drive(180, maxamp=True)
                ev[3].record(st)
                ev[3].synchronize()
                t_init = ev[0].elapsed_time(ev[1]) * 1e-3
                t_step = ev[2].elapsed_time(ev[3]) * 1e-3 / 180
                t0 = time.perf_counter()
                s.getzmax(1)
                s.getarrival(1)
                t_read = time.perf_counter() - t0
                s.close()
                svc_class[(size, nested)] = (t_init + t_read, t_step)
        service = [svc_class[(size, nested)][0] + nsteps * svc_class[(size, nested)][1]
                   for (_t, size, nsteps, nested, _seed) in trace]
        plat, _ = serving.fifo_latencies([t for (t, *_rest) in trace], service)
        plain = {"p50_s": float(np.percentile(plat, 50)), "p99_s": float(np.percentile(plat, 99)),
                 "scenarios_per_hour": 3600.0 / float(np.mean(service)),
                 "method": "per class (size x nested) service time = init + reads + nsteps x measured step "
                           "time through the reference C ABI (one kernel per phase); FIFO queue on the same "
                           "arrival times"}
    line = {"metric": "p99 time-to-forecast", "value": pl["p99"], "unit": "s", "n_gpus": world,
            "steps": int(sum(r.case.nsteps for r in reqs)), "warmup": len(warm),
            "ms_per_step": None, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"C5: {len(reqs)} requests, Poisson {args.rate} req/s, outer "
                                   "481x401/961x801/1921x1601 at 2', 30% nested 301x251 r=5 nonlinear child, "
                                   "30-120 min at dt 2 s, 16 gauges", "hbm_budget_gb": args.budget_gb,
                       "graph_chunk": args.chunk, "tile_variant": variant, "parallelism": f"replicas x{world}"},
            "p50_s": pl["p50"], "p99_s": pl["p99"], "mean_s": float(lat.mean()), "max_s": float(lat.max()),
            "scenarios_per_hour_under_load": len(reqs) * 3600.0 / span,
            "scenarios_per_hour_saturated": capacity, "saturated_seconds": sat_s,
            "cell_updates_per_s_saturated": cell_updates / sat_s,
            "max_active": max_active, "max_active_saturated": sat_active, "admission_waits": refused,
            "clocks": ck, "gpu_launches": launches,
            "e2e": {"value": pl["p99"], "unit": "s",
                    "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                    "note": "time-to-forecast is end to end: the request's initial surface and gauges go "
                            "host->device at admission, max-eta, arrival and gauge series device->host at "
                            "completion"}}
    if plain:
        line["plain_path"] = plain
        line["capacity_vs_plain"] = capacity / plain["scenarios_per_hour"]
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 7200 for c2, 3600 for c4)")
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--variant", type=int, default=-1, help="fixed tile variant (skips the autotuner)")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the headline single grid; c3: the nested run; c4: the 64-scenario ensemble; "
                         "c5: the forecast-serving load")
    ap.add_argument("--requests", type=int, default=400, help="C5: requests in the trace")
    ap.add_argument("--rate", type=float, default=2.0, help="C5: mean arrivals per second")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="C5: HBM admission budget")
    ap.add_argument("--chunk", type=int, default=32, help="C5: steps between harvests")
    ap.add_argument("--no-plain", action="store_true", help="C5: skip the plain-path service times")
    ap.add_argument("--scenarios", type=int, default=64)
    ap.add_argument("--plain-sample", type=int, default=4, help="C4: scenarios run on the plain path")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = 7200 if args.workload == "c2" else 3600
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)

    import torch

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod

    from comcot_b200.abi import ReferenceSession
    from comcot_b200.engine import Engine

    if args.workload == "c4":
        return run_c4(args, torch, dist, rank, world, local)
    if args.workload == "c3":
        return run_c3(args, torch, dist, rank, world, local)
    if args.workload == "c5":
        return run_c5(args, torch, dist, rank, world, local)

    return run_single(args, torch, dist, rank, world, local)


def run_single(args, torch, dist, rank, world, local):
    """C1 / C2: one linear spherical grid (value: the engine, device-resident;
    e2e: the reference C ABI with host buffers; cpu_baseline: the serial oracle)."""
    from comcot_b200.abi import ReferenceSession
    from comcot_b200.engine import Engine

    tune_reps = 3
    from comcot_b200 import _lib

    lib = _lib.load()
    ncand = lib.gc_engine_num_candidates()  # the autotuner's candidates: tile variants x tile-height rules
    total = ncand * (tune_reps + 1) + args.warmup + args.steps + 8
    make_case = synth.config_c1 if args.workload == "c1" else synth.config_c2
    case = make_case(nsteps=total)
    cells = case.root.nx * case.root.ny

    # ---------------- device-resident throughput (engine) ----------------
    eng = Engine(budget=8 << 30)
    eng.config(variant=args.variant, use_graphs=1, chunk=64)
    eng.add(case)
    if args.variant < 0:
        eng.autotune(tune_reps)
    variant = eng.variant()  # variant + variants x tile-height rule
    eng.step(args.warmup)
    eng.prepare()  # step-chunk graph built before the timed region
    eng.sync()
    stream = torch.cuda.ExternalStream(eng.stream())
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    l0 = eng.launches()
    ev0.record(stream)
    eng.step(args.steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    ck = clocks.stop()
    if dist:
        dist.barrier()
    launches = eng.launches() - l0  # fused steps + the graphs' step-counter kernels
    ms = ev0.elapsed_time(ev1)
    ms = replicas.reduce_max(ms, dist, 'cuda')
    value = cells * args.steps * world / (ms * 1e-3)
    eng.close()

    # ---------------- end to end through the reference C ABI ----------------
    e2e = None
    if not args.no_e2e:
        case_e = make_case(nsteps=args.steps)
        s = ReferenceSession(case_e, fusion=True, init_layers=False)
        st = torch.cuda.ExternalStream(s.stream())
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        s.init_layers()
        s.drive(args.steps, maxamp=True)
        z = s.getz(1)
        zm = s.getzmax(1)
        b.record(st)
        b.synchronize()
        e2e_ms = a.elapsed_time(b)
        e2e_ms = replicas.reduce_max(e2e_ms, dist, 'cuda')
        nx, ny = case_e.root.nx, case_e.root.ny
        field = nx * ny * 4
        # H and Z as fields plus the 8-float row record per row; the R fields are read on the host
        h2d = (2 * field + ny * 8 * 4) / args.steps
        d2h = len(case_e.gauges) * 16 + 2 * field / args.steps
        e2e = {"value": cells * args.steps * world / (e2e_ms * 1e-3), "unit": METRIC,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e2e_ms / args.steps,
               "path": "gcomcot_init_layer_ + per step mass/openbd/momt/maxamp/get_z x32/update + getz/getzmax"}
        launches_e2e = s.launches()
        s.close()
        del z, zm

    peak, peak_kind = peaks()
    bytes_launch = BYTES_PER_CELL * cells
    achieved = bytes_launch / (ms * 1e-3 / args.steps) / 1e9
    traffic = profiled_traffic()
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload],
                   "cells": cells, "parallelism": f"replicas x{world}",
                   "l2": ("working set 156 MB per step (8 fields x 19.5 MB) > 126 MB L2; no flush"
                          if args.workload == "c2" else "working set 3.5 MB: L2 resident (no flush)"),
                   "tile_variant": variant, "graph_chunk": 64},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic,
                     "peak_kind": f"{peak_kind} (copy bandwidth)",
                     "algorithmic_bytes_per_launch": bytes_launch},
        "clocks": ck,
        "gpu_launches": launches,
    }
    if e2e:
        line["e2e"] = e2e
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(make_case(nsteps=total))
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
