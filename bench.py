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
e2e    : the same metric through the reference C ABI with host buffers, over
         one whole C2 forecast (7200 steps) whatever --steps is:
         gcomcot_init_layer_ uploads H, Z and the R arrays from host memory,
         then every step runs MASS/OPEN/MOMENT/MAX_AMP through the legacy
         entry points and reads the 32 gauge stencils back to the host, and the
         final surface and max-eta are downloaded.
parity : after the timed runs, the state each of them produced (the engine's
         member after every step it ran, the reference-ABI session after its
         forecast) against the FP32 oracle run for the same number of steps
         on the host's cores: max relative error of eta, M/N, max-eta and the
         gauge series, wet mask and arrival steps compared exactly, and bit
         equality.
nested, ensemble, serving (default C2 run, one GPU): compact records of the
         C3 nested step, the C4 64-scenario ensemble against the plain
         one-scenario path, and the C5 serving load on a shortened trace,
         each with its own timing, roofline, clocks and parity sample.
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
FORECAST_STEPS = {"c1": 3600, "c2": 7200}  # one whole forecast of the config
FALLBACK_HBM_GBS = 6650.0
BYTES_PER_CELL = 36  # per launch: Z1,M1,N1,H in + Z,M,N out (28 B) + max-eta read/write (8 B)
TOL = 1e-4           # max|d eta| <= 1e-4 max|eta|, max|d(M,N)| <= 1e-4 max|M,N|
GX = np.float32(1e-5)


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


def pair_note(rl, one_step_gbs, profile):
    """a two-step launch reads and writes each cell once for two steps, so its
    HBM fraction is of half the one-step bytes; it is bounded by instruction
    issue instead.  Adds the HBM fraction a one-step kernel would need for
    the same steps/s, and the limiter."""
    if rl.get("steps_per_launch") == 2:
        rl["one_step_equivalent_gbs"] = one_step_gbs
        rl["one_step_equivalent_frac"] = one_step_gbs / rl["peak"]
        rl["limiter"] = (f"instruction issue (two steps per HBM pass: same bytes per launch as one step); "
                         f"issue-slot and stall figures in profiles/{profile}")
    return rl


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        """Starts polling and returns after the first sample (3 s at most):
        nvidia-smi's start-up opens the driver and would otherwise overlap
        the first launches of a short timed region."""
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "100",
                 "-i", str(self.gpu)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
            return
        t_end = time.time() + 3.0
        while not self.lines and time.time() < t_end and self.proc.poll() is None:
            time.sleep(0.01)

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


# ---------------------------------------------------------------------------
# parity: the state a benchmarked run produced against the FP32 oracle
# ---------------------------------------------------------------------------
def _oracle():
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle

    return oracle


def oracle_states(case, checkpoints, threads=None):
    """Runs the FP32 oracle on `case` and snapshots every layer (and the gauge
    series so far) after each step count in `checkpoints`."""
    oracle = _oracle()
    threads = threads or os.cpu_count() or 1
    o = oracle.OracleRun(case)
    out, done, ts = {}, 0, []
    for s in sorted(set(int(c) for c in checkpoints if c > 0)):
        ts.append(o.run(s - done, threads=threads))
        done = s
        out[s] = {"layers": [{k: (None if v is None else v.copy()) for k, v in o.layer(q).items()}
                             for q in range(len(case.layers))],
                  "ts": np.concatenate(ts, axis=0)}
    return out


def _rel(a, b):
    scale = max(float(np.abs(b).max()), 1e-30)
    return float(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).max()) / scale


def _same_bits(a, b):
    return bool(np.array_equal(np.ascontiguousarray(a, np.float32).view(np.uint32),
                               np.ascontiguousarray(b, np.float32).view(np.uint32)))


def parity_record(got, ref, steps, H=None, ts=None, ts_ref=None, child=None, child_ref=None, child_H=None,
                  what=""):
    """got / ref: dicts with any of z, m, n, zmax (float) and arrival (int);
    child / child_ref likewise for a nested child.  Floating fields at the
    stated tolerance and bit for bit; wet mask and arrival exactly."""
    rec = {"what": what, "steps": int(steps), "tolerance": TOL}
    ok, bits = True, True
    if "z" in got:
        rec["max_rel_eta"] = _rel(got["z"], ref["z"])
        ok &= rec["max_rel_eta"] <= TOL
        bits &= _same_bits(got["z"], ref["z"])
    mn = [k for k in ("m", "n") if k in got]
    if mn:
        rec["max_rel_mn"] = max(_rel(got[k], ref[k]) for k in mn)
        ok &= rec["max_rel_mn"] <= TOL
        bits &= all(_same_bits(got[k], ref[k]) for k in mn)
    if "zmax" in got and ref.get("zmax") is not None:
        rec["max_rel_zmax"] = _rel(got["zmax"], ref["zmax"])
        ok &= rec["max_rel_zmax"] <= TOL
        bits &= _same_bits(got["zmax"], ref["zmax"])
    if "arrival" in got and ref.get("arrival") is not None:
        rec["arrival_equal"] = bool(np.array_equal(got["arrival"], ref["arrival"]))
        ok &= rec["arrival_equal"]
        bits &= rec["arrival_equal"]
    if H is not None and "z" in got:
        rec["masks_equal"] = bool(np.array_equal(got["z"] + H > GX, ref["z"] + H > GX))
        ok &= rec["masks_equal"]
    if ts is not None and ts_ref is not None and ts.size:
        rec["max_rel_gauges"] = _rel(ts, ts_ref)
        ok &= rec["max_rel_gauges"] <= TOL
        bits &= _same_bits(ts, ts_ref)
    if child is not None:
        rec["child_max_rel_eta"] = _rel(child["z"], child_ref["z"])
        rec["child_max_rel_mn"] = max(_rel(child[k], child_ref[k]) for k in ("m", "n"))
        ok &= rec["child_max_rel_eta"] <= TOL and rec["child_max_rel_mn"] <= TOL
        bits &= all(_same_bits(child[k], child_ref[k]) for k in ("z", "m", "n"))
        if child_H is not None:
            rec["child_masks_equal"] = bool(np.array_equal(child["z"] + child_H > GX,
                                                           child_ref["z"] + child_H > GX))
            ok &= rec["child_masks_equal"]
    rec["within_tolerance"] = bool(ok)
    rec["bitwise"] = bool(bits)
    return rec


def timed_engine_steps(torch, eng, steps, warmup, dist, local):
    """The warm-up steps, then exactly `steps` timed steps with CUDA events on
    the engine's stream, between a barrier and a synchronize on both sides.
    The step-chunk graph and the clock sampler are set up first, so the
    warm-up runs directly before the timed region: a B200 left idle for a
    fraction of a second starts the next short region measurably slower.
    Returns (ms, launches, clocks); ms is the max over ranks."""
    eng.prepare()  # step-chunk graph built before the timed region
    clocks = ClockSampler(local)
    clocks.start()
    eng.step(warmup)
    eng.sync()
    stream = torch.cuda.ExternalStream(eng.stream())
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = eng.launches()
    ev0.record(stream)
    eng.step(steps)
    ev1.record(stream)
    ev1.synchronize()
    torch.cuda.synchronize()
    ck = clocks.stop()
    if dist:
        dist.barrier()
    launches = eng.launches() - l0
    ms = replicas.reduce_max(ev0.elapsed_time(ev1), dist, 'cuda')
    return ms, launches, ck


def steps_per_launch(variant):
    """2 when the engine's chosen candidate is the two-step kernel
    (candidates past the one-step variants x their tile-height rules)"""
    from comcot_b200 import _lib

    return 2 if variant >= 2 * _lib.load().gc_engine_num_variants() else 1


def merge_parity(records):
    """one summary over several parity records"""
    return {"within_tolerance": all(r["within_tolerance"] for r in records),
            "bitwise": all(r["bitwise"] for r in records), "runs": records}


def gauge_series(stencils, gauges):
    from comcot_b200.serving import gauge_series as gs

    return gs(stencils, gauges)


# ---------------------------------------------------------------------------
# CPU baselines
# ---------------------------------------------------------------------------
def cpu_baseline(case, budget_s=15.0):
    """FP32 oracle (the restated reference Fortran), one thread, bounded sample."""
    oracle = _oracle()
    o = oracle.OracleRun(case)
    t0 = time.perf_counter()
    o.run(1, threads=1)
    one = time.perf_counter() - t0
    n = max(1, min(case.nsteps, int(budget_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    o.run(n, threads=1)
    dt = time.perf_counter() - t0
    cells = case.cells_per_step()
    return {"value": cells * n / dt, "unit": METRIC, "cores": 1, "kind": "port",
            "sample": f"{n} outer steps of the full {case.root.nx}x{case.root.ny} grid"
                      f"{' and its child' if len(case.layers) > 1 else ''}, serial oracle "
                      f"(restated Fortran solvers + max-eta), {dt:.1f} s"}


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    oracle = _oracle()
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


# ---------------------------------------------------------------------------
# C4: the batched ensemble
# ---------------------------------------------------------------------------
def bench_c4(torch, dist, world, local, steps, warmup, nscen, plain_sample, variant, rank_seed=0,
             parity_members=2):
    """C4: `nscen` dipole scenarios on one 1201x1001 2' grid with shared
    bathymetry, stepped by the batched engine (one fused launch per step over
    all members, CUDA-graph replay), against the plain path: one scenario at a
    time through the reference C ABI with one kernel per phase."""
    from comcot_b200 import _lib
    from comcot_b200.abi import ReferenceSession
    from comcot_b200.engine import Engine
    from comcot_b200.synth import Case

    L = synth.config_c4_grid()
    srcs = synth.ensemble_sources(L.x, L.y, nscen, seed=40 + rank_seed)
    case = Case("C4", [L], steps)
    tune_reps = 2
    ncand = _lib.load().gc_engine_num_candidates()  # tile variants x tile-height rules
    # the autotuner's steps (two-step candidates run pairs), its second round
    # (the three fastest, three 64-step graph chunks each), and the warm-up
    extra = ncand * (2 * tune_reps + 2) + 3 * 3 * 64 + warmup
    eng = Engine(budget=120 << 30)
    eng.config(variant=variant, use_graphs=1, chunk=64)
    cls = eng.add_class(L)
    ids = [eng.add(case, z0=z, cls=cls, nsteps=steps + extra, gauges=[], arrival_thr=0.05) for z in srcs]
    if variant < 0:
        eng.autotune(tune_reps)
    chosen = eng.variant()  # variant + variants x tile-height rule
    ms, launches, ck = timed_engine_steps(torch, eng, steps, warmup, dist, local)
    eng.sync()
    sample = sorted({0, nscen - 1})[:parity_members]
    got = {q: (eng.steps_done(ids[q]), eng.read(ids[q], fields=("z", "m", "n", "zmax", "arrival"))) for q in sample}
    eng.close()
    cells = L.nx * L.ny
    # scenarios/hour of whole 3600-step forecasts at the measured step rate
    scen_per_hour = nscen * world * 3600.0 / (ms * 1e-3 / steps * 3600.0)
    value_cells = cells * nscen * steps * world / (ms * 1e-3)
    # plain path: a sample of scenarios, each alone through the reference ABI
    plain, plain_state = None, None
    if plain_sample > 0:
        t_tot = 0.0
        k = min(plain_sample, nscen)
        host = {}
        for q in range(k):
            Lq = synth.LayerSpec(**{**L.__dict__, "Z0": np.ascontiguousarray(srcs[q], dtype=np.float32)})
            s = ReferenceSession(Case("C4p", [Lq], steps), fusion=False, init_layers=False, arrival=False,
                                 host_cache=host)
            st = torch.cuda.ExternalStream(s.stream())
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.init_layers()
            torch.cuda.synchronize()
            a.record(st)
            s.drive(steps, maxamp=True)
            b.record(st)
            b.synchronize()
            t_tot += a.elapsed_time(b) * 1e-3
            if q == 0:
                (pm, pn) = s.getmn(1)
                plain_state = {"z": s.getz(1), "m": pm, "n": pn, "zmax": s.getzmax(1)}
            s.close()
        per_step = t_tot / k / steps
        plain = {"scenarios_per_hour": 3600.0 / (per_step * 3600.0), "s_per_step": per_step,
                 "sample": f"{k} of {nscen} scenarios run alone for {steps} steps each, per-step time scaled "
                           f"to a 3600-step forecast",
                 "path": "reference C ABI, one kernel per phase (mass, open, momentum, max)"}
    # parity of the benchmarked state: sampled members and the first plain scenario
    recs = []
    for q in sample:
        done, g = got[q]
        Lq = synth.LayerSpec(**{**L.__dict__, "Z0": np.ascontiguousarray(srcs[q], dtype=np.float32)})
        cq = Case("C4", [Lq], max(done, steps))
        chk = [done] + ([steps] if (q == 0 and plain_state is not None) else [])
        st = oracle_states(cq, chk)
        recs.append(parity_record(g, st[done]["layers"][0], done, H=L.H, what=f"engine member {q}"))
        if q == 0 and plain_state is not None:
            recs.append(parity_record(plain_state, st[steps]["layers"][0], steps, H=L.H,
                                      what="plain path scenario 0 (reference ABI, per phase)"))
    peak, peak_kind = peaks()
    spl = steps_per_launch(chosen)
    bpc = 24.0 + 4.0 / nscen + 8.0  # per member-cell and launch: Z,M,N in/out, shared H, max-eta r/w
    achieved = bpc * cells * nscen / (ms * 1e-3 / steps * spl) / 1e9
    tr = profiled_traffic("pair_ensemble_step_c4.txt" if spl == 2 else "fused_ensemble_step_c4.txt",
                          "traffic_bytes_per_member_launch")
    rec = {"metric": "ensemble scenarios/hour", "value": scen_per_hour, "unit": "scenarios/hour",
           "steps": steps, "warmup": warmup, "ms_per_step": ms / steps, "cell_updates_per_s": value_cells,
           "config": {"workload": f"C4: {nscen} dipole scenarios on 1201x1001 2' linear spherical, shared H, "
                                  f"dt 2 s, max-eta + arrival; scenarios/hour of 3600-step forecasts",
                      "tile_variant": chosen,
                      "l2": f"working set {nscen} x 7 fields x 4.9 MB >> 126 MB L2"},
           "roofline": pair_note({"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                  "frac": achieved / peak, "traffic": None if tr is None else nscen * tr,
                                  "peak_kind": f"{peak_kind} (copy bandwidth)",
                                  "algorithmic_bytes_per_launch": bpc * cells * nscen, "steps_per_launch": spl},
                                 achieved * spl, "pair_ensemble_step_c4.txt"),
           "clocks": ck, "gpu_launches": launches, "parity": merge_parity(recs)}
    if plain:
        rec["plain_path"] = plain
        rec["speedup_vs_plain"] = scen_per_hour / plain["scenarios_per_hour"]
    return rec


def run_c4(args, torch, dist, rank, world, local):
    rec = bench_c4(torch, dist, world, local, args.steps, args.warmup, args.scenarios,
                   args.plain_sample if rank == 0 else 0, args.variant, rank_seed=rank)
    line = {"metric": rec["metric"], "value": rec["value"], "unit": rec["unit"], "n_gpus": world,
            "steps": rec["steps"], "warmup": rec["warmup"], "ms_per_step": rec["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    line.update({k: v for k, v in rec.items() if k not in line})
    line["config"]["parallelism"] = f"scenario replicas x{world}"
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# C3: the nested run
# ---------------------------------------------------------------------------
def bench_c3(torch, dist, world, local, steps, warmup, variant, e2e_steps=0, cpu=False):
    """C3: two-level nested run -- 1201x1001 2' linear spherical outer grid and
    a 601x501 nonlinear Cartesian child (wet/dry, Manning n = 0.025, ratio 5)
    coupled by JNQ/NEWQ edge fluxes and JNZ feedback every outer step.  value:
    the batched engine's nested path (per-phase child kernels in a captured
    graph); e2e: the reference C ABI call sequence with host buffers over
    e2e_steps outer steps."""
    from comcot_b200.abi import ReferenceSession
    from comcot_b200.engine import Engine

    total = warmup + steps
    case = synth.config_c3(nsteps=total)
    P, Cl = case.layers
    cells = P.nx * P.ny + Cl.nx * Cl.ny * Cl.rel_time
    eng = Engine(budget=8 << 30)
    eng.config(variant=variant, use_graphs=1, chunk=64)
    mid = eng.add(case)
    ms, launches, ck = timed_engine_steps(torch, eng, steps, warmup, dist, local)
    eng.sync()
    done = eng.steps_done(mid)
    got = eng.read(mid, fields=("z", "m", "n", "zmax", "arrival", "child"))
    eng.close()
    value = cells * steps * world / (ms * 1e-3)
    e2e, e2e_state = None, None
    if e2e_steps > 0:
        case_e = synth.config_c3(nsteps=e2e_steps)
        s = ReferenceSession(case_e, fusion=True, arrival=True, init_layers=False)
        st = torch.cuda.ExternalStream(s.stream())
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        s.init_layers()
        s.drive(e2e_steps, maxamp=True)
        z, zc, zm = s.getz(1), s.getz(2), s.getzmax(1)
        b.record(st)
        b.synchronize()
        e2e_ms = a.elapsed_time(b)
        (m, n), (mc, nc) = s.getmn(1), s.getmn(2)
        e2e_state = ({"z": z, "m": m, "n": n, "zmax": zm, "arrival": s.getarrival(1)},
                     {"z": zc, "m": mc, "n": nc})
        s.close()
        fp, fc = P.nx * P.ny * 4, Cl.nx * Cl.ny * 4
        e2e = {"value": cells * e2e_steps * world / (e2e_ms * 1e-3), "unit": METRIC, "steps": e2e_steps,
               # the outer grid's H and Z, the child's H, Z, HP and HQ, and the 8-float row records
               "h2d_bytes_per_step": int((2 * fp + 4 * fc + (P.ny + Cl.ny) * 8 * 4) / e2e_steps),
               "d2h_bytes_per_step": int((2 * fp + fc) / e2e_steps), "ms_per_step": e2e_ms / e2e_steps,
               "path": "gcomcot_set_layer_params_/init_layer x2 + per step mass/openbd/all_grid/momt/maxamp/"
                       "update + getz x2/getzmax"}
    # parity of the benchmarked states
    chk = [done] + ([e2e_steps] if e2e_state else [])
    ost = oracle_states(synth.config_c3(nsteps=max(chk)), chk)
    child = {k: got["child_" + k] for k in ("z", "m", "n")}
    recs = [parity_record(got, ost[done]["layers"][0], done, H=P.H, child=child,
                          child_ref=ost[done]["layers"][1], child_H=Cl.H, what="engine nested member")]
    if e2e_state:
        recs.append(parity_record(e2e_state[0], ost[e2e_steps]["layers"][0], e2e_steps, H=P.H, child=e2e_state[1],
                                  child_ref=ost[e2e_steps]["layers"][1], child_H=Cl.H,
                                  what="reference ABI session (e2e)"))
    peak, peak_kind = peaks()
    # algorithmic bytes of one outer step: outer grid 28 B + max-eta 8 B + arrival 8 B per cell;
    # child 28 B per cell per sub-step (Z, M, N, H in; Z, M, N out; DZ = Z + H) + JNZ 8 B per child cell
    bstep = 44.0 * P.nx * P.ny + (28.0 * Cl.rel_time + 8.0) * Cl.nx * Cl.ny
    achieved = bstep / (ms * 1e-3 / steps) / 1e9
    rec = {"metric": METRIC, "value": value, "unit": METRIC, "steps": steps, "warmup": warmup,
           "ms_per_step": ms / steps,
           "config": {"workload": f"C3: 1201x1001 2' linear spherical + {Cl.nx}x{Cl.ny} nonlinear Cartesian "
                                  f"child (r=5, rel_time {Cl.rel_time}, Manning 0.025), dt 2 s",
                      "cells_per_step": cells,
                      "l2": "working set ~60 MB per step fits the 126 MB L2; no flush (L2 resident)"},
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "traffic": None, "peak_kind": f"{peak_kind} (copy bandwidth)",
                        "algorithmic_bytes_per_step": bstep},
           "clocks": ck, "gpu_launches": launches, "parity": merge_parity(recs)}
    if e2e:
        rec["e2e"] = e2e
    if cpu:
        rec["cpu_baseline"] = cpu_baseline(synth.config_c3(nsteps=total))
    return rec


def run_c3(args, torch, dist, rank, world, local):
    rec = bench_c3(torch, dist, world, local, args.steps, args.warmup, args.variant,
                   e2e_steps=0 if args.no_e2e else 3600, cpu=(rank == 0 and not args.no_cpu_baseline))
    line = {"metric": METRIC, "value": rec["value"], "unit": METRIC, "n_gpus": world, "steps": rec["steps"],
            "warmup": rec["warmup"], "ms_per_step": rec["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    line.update({k: v for k, v in rec.items() if k not in line})
    line["config"]["parallelism"] = f"replicas x{world}"
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# C5: serving
# ---------------------------------------------------------------------------
def bench_c5(torch, local, nreq, rate, budget_gb, chunk, variant, plain=True, rank=0, world=1, dist=None):
    """C5 serving: a seeded Poisson stream of forecast requests (mean `rate`
    req/s; outer grids 481x401, 961x801 or 1921x1601 at 2'; 30 % nested with
    a 301x251 ratio-5 nonlinear child; 30-120 simulated minutes at dt 2 s; a
    dipole source and 16 gauges each) served by continuous batching with
    admission by HBM footprint.  Reported: p50/p99 time-to-forecast under the
    arrival load, scenarios/hour at saturation, and the same measured for the
    plain path (one request at a time through the reference C ABI, one kernel
    per phase) on the same trace."""
    from comcot_b200 import _lib, serving
    from comcot_b200.engine import Engine

    tpl = synth.config_c5_templates()
    # one trace for the whole job; each rank serves its round-robin share
    trace = replicas.shard(synth.poisson_trace(n=nreq, rate=rate, seed=5), rank, world)

    def make_requests():
        return [serving.Request(k, t, synth.c5_request_case(tpl, size, nsteps, nested, seed))
                for k, (t, size, nsteps, nested, seed) in enumerate(trace)]

    reqs = make_requests()
    # tile variant: tuned once (not timed) on a warm batch of one request of
    # each outer size, so that the launch forms are those of a mixed batch
    # (the work list, not the one-class launch)
    if variant < 0:
        batch = [synth.c5_request_case(tpl, sz, 64, False, 77 + k) for k, sz in enumerate(synth.C5_SIZES)]
        with Engine(budget=16 << 30) as eng:
            for c in batch:
                eng.add(c, nsteps=6 * _lib.load().gc_engine_num_candidates() + 3 * 3 * 32 + 8)
            eng.autotune(2)
            variant = eng.variant()  # variant + variants x tile-height rule
    budget = int(budget_gb * (1 << 30))
    # warm-up: a few requests through the server (module load, first graphs)
    with serving.ForecastServer(budget, chunk=chunk, variant=variant) as srv:
        warm = [serving.Request(k, 0.0, synth.c5_request_case(tpl, sz, 64, k % 2 == 1, 900 + k))
                for k, sz in enumerate(synth.C5_SIZES)]
        srv.serve(warm, speed=float("inf"))
    torch.cuda.synchronize()
    cell_updates = sum(r.case.nsteps * r.case.cells_per_step() for r in reqs)
    # 1) the arrival load, in real time
    clocks = ClockSampler(local)
    clocks.start()
    with serving.ForecastServer(budget, chunk=chunk, variant=variant) as srv:
        l0 = srv.eng.launches()
        srv.serve(reqs, speed=1.0)
        launches = srv.eng.launches() - l0
        max_active, refused = srv.max_active, srv.refused
    ck = clocks.stop()
    lat = np.array([r.latency for r in reqs])
    span = max(r.t_done for r in reqs)
    pl = serving.percentiles(lat)
    ranks = None
    if dist is not None and world > 1:
        # every rank's latencies to rank 0 through the group's store, with a
        # bounded wait: a rank that died is reported, not waited for
        store = replicas.default_store(dist)
        if store is not None:
            hb = replicas.Heartbeat(store, rank, world)
            got, missing, stale = replicas.collect(store, rank, world, {"lat": lat.tolist(), "span": span},
                                                   timeout_s=300.0, hb=hb)
            if rank == 0:
                lat = np.concatenate([np.asarray(g["lat"], dtype=np.float64) for g in got.values()])
                span = max(g["span"] for g in got.values())
                pl = serving.percentiles(lat)
                served = len(lat)
                ranks = {"ranks_reporting": sorted(got), "ranks_missing": missing, "ranks_stale": stale,
                         "requests_unserved": nreq - served}
    # 2) saturation: every request at t = 0
    reqs_sat = make_requests()
    torch.cuda.synchronize()
    with serving.ForecastServer(budget, chunk=chunk, variant=variant) as srv:
        t0 = time.perf_counter()
        srv.serve(reqs_sat, speed=float("inf"))
        sat_s = time.perf_counter() - t0
        sat_active = srv.max_active
    capacity = len(reqs_sat) * 3600.0 / sat_s
    # 3) the plain path, measured on the same trace: one request at a time
    plain_rec, preqs = None, None
    if plain:
        ps = serving.PlainServer(fusion=False)
        preqs = make_requests()
        ps.prepare(preqs)
        torch.cuda.synchronize()
        ps.serve(preqs, speed=1.0)
        plat = np.array([r.latency for r in preqs])
        service = np.array([r.t_done - r.t_admit for r in preqs])
        pp = serving.percentiles(plat)
        plain_rec = {"p50_s": pp["p50"], "p99_s": pp["p99"], "mean_s": float(plat.mean()),
                     "scenarios_per_hour": 3600.0 / float(service.mean()),
                     "method": "measured: the same trace served one request at a time in arrival order "
                               "through the reference C ABI (layer upload, per-phase kernels, the gauge "
                               "stencils of every step gathered on the device by gcomcot_drive, products read "
                               "back)"}
    # parity: the smallest un-nested and nested requests of the trace, served in
    # the mix (and on the plain path) against the oracle
    recs = []
    for nested in (False, True):
        cand = [r for r in reqs if (len(r.case.layers) > 1) == nested and r.status == "done"]
        if not cand:
            continue
        r = min(cand, key=lambda q: q.case.nsteps * q.case.cells_per_step())
        ost = oracle_states(r.case, [r.case.nsteps])[r.case.nsteps]
        ref, ts_ref = ost["layers"][0], ost["ts"]
        res = r.result
        recs.append(parity_record({"zmax": res["zmax"], "arrival": res["arrival"]}, ref, r.case.nsteps,
                                  ts=res["ts"][: r.case.nsteps], ts_ref=ts_ref,
                                  what=f"served in the mix: request {r.rid} "
                                       f"({r.case.root.nx}x{r.case.root.ny}{' nested' if nested else ''})"))
        if preqs is not None:
            pr = preqs[r.rid].result
            recs.append(parity_record({"zmax": pr["zmax"], "arrival": pr["arrival"]}, ref, r.case.nsteps,
                                      ts=pr["ts"], ts_ref=ts_ref, what=f"plain path: request {r.rid}"))
    rec = {"metric": "p99 time-to-forecast", "value": pl["p99"], "unit": "s",
           "steps": int(sum(r.case.nsteps for r in reqs)),
           "config": {"workload": f"C5: {len(reqs)} requests, Poisson {rate} req/s, outer "
                                  "481x401/961x801/1921x1601 at 2', 30% nested 301x251 r=5 nonlinear child, "
                                  "30-120 min at dt 2 s, 16 gauges", "hbm_budget_gb": budget_gb,
                      "graph_chunk": chunk, "tile_variant": variant},
           "p50_s": pl["p50"], "p99_s": pl["p99"], "mean_s": float(lat.mean()), "max_s": float(lat.max()),
           "scenarios_per_hour_under_load": len(lat) * 3600.0 / span,
           "scenarios_per_hour_saturated": capacity, "saturated_seconds": sat_s,
           "cell_updates_per_s_saturated": cell_updates / sat_s,
           "max_active": max_active, "max_active_saturated": sat_active, "admission_waits": refused,
           "clocks": ck, "gpu_launches": launches, "parity": merge_parity(recs)}
    if ranks:
        rec["replicas"] = ranks
    if plain_rec:
        rec["plain_path"] = plain_rec
        rec["capacity_vs_plain"] = capacity / plain_rec["scenarios_per_hour"]
        rec["p99_vs_plain"] = plain_rec["p99_s"] / pl["p99"]
    return rec


def run_c5(args, torch, dist, rank, world, local):
    rec = bench_c5(torch, local, args.requests, args.rate, args.budget_gb, args.chunk, args.variant,
                   plain=not args.no_plain, rank=rank, world=world, dist=dist)
    line = {"metric": rec["metric"], "value": rec["value"], "unit": "s", "n_gpus": world, "steps": rec["steps"],
            "warmup": 3, "ms_per_step": None, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic"}
    line.update({k: v for k, v in rec.items() if k not in line})
    line["config"]["parallelism"] = f"replicas x{world}"
    line["e2e"] = {"value": rec["p99_s"], "unit": "s", "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                   "note": "time-to-forecast is end to end: the request's initial surface and gauges go "
                           "host->device at admission, max-eta, arrival and gauge series device->host at "
                           "completion"}
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# C1 / C2: one grid (the headline)
# ---------------------------------------------------------------------------
def run_single(args, torch, dist, rank, world, local):
    """C1 / C2: one linear spherical grid (value: the engine, device-resident;
    e2e: the reference C ABI with host buffers over one whole forecast;
    parity of both against the oracle; cpu_baseline: the serial oracle)."""
    from comcot_b200 import _lib
    from comcot_b200.abi import ReferenceSession
    from comcot_b200.engine import Engine

    tune_reps = 3
    lib = _lib.load()
    ncand = lib.gc_engine_num_candidates()  # the autotuner's candidates: tile variants x tile-height rules
    # two-step candidates run pairs; the second round re-times the three
    # fastest over three 64-step graph chunks each
    total = ncand * (2 * tune_reps + 2) + 3 * 3 * 64 + args.warmup + args.steps + 8
    make_case = synth.config_c1 if args.workload == "c1" else synth.config_c2
    case = make_case(nsteps=total)
    cells = case.root.nx * case.root.ny

    # ---------------- device-resident throughput (engine) ----------------
    eng = Engine(budget=8 << 30)
    eng.config(variant=args.variant, use_graphs=1, chunk=64)
    mid = eng.add(case)
    if args.variant < 0:
        eng.autotune(tune_reps)
    variant = eng.variant()  # variant + variants x tile-height rule
    # launches: the step kernels + the graphs' step-counter kernels
    ms, launches, ck = timed_engine_steps(torch, eng, args.steps, args.warmup, dist, local)
    value = cells * args.steps * world / (ms * 1e-3)
    eng.sync()
    done = eng.steps_done(mid)
    got = eng.read(mid)
    eng.close()

    # ---------------- end to end through the reference C ABI ----------------
    e2e, e2e_state = None, None
    E = FORECAST_STEPS[args.workload]
    if not args.no_e2e:
        case_e = make_case(nsteps=E)
        s = ReferenceSession(case_e, fusion=True, init_layers=False)
        st = torch.cuda.ExternalStream(s.stream())
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        a.record(st)
        s.init_layers()
        stencils = s.drive(E, maxamp=True)
        z = s.getz(1)
        zm = s.getzmax(1)
        b.record(st)
        b.synchronize()
        e2e_ms = a.elapsed_time(b)
        e2e_ms = replicas.reduce_max(e2e_ms, dist, 'cuda')
        m, n = s.getmn(1)
        e2e_state = {"z": z, "m": m, "n": n, "zmax": zm}, gauge_series(stencils, case_e.gauges)
        nx, ny = case_e.root.nx, case_e.root.ny
        field = nx * ny * 4
        # H and Z as fields plus the 8-float row record per row; the R fields are read on the host
        h2d = (2 * field + ny * 8 * 4) / E
        d2h = len(case_e.gauges) * 16 + 2 * field / E
        e2e = {"value": cells * E * world / (e2e_ms * 1e-3), "unit": METRIC, "steps": E,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "ms_per_step": e2e_ms / E,
               "note": f"one whole forecast ({E} steps) end to end, whatever --steps is",
               "path": ("gcomcot_init_layer_ + gcomcot_drive (per step mass/openbd/momt/maxamp, the 32 gauge "
                        "stencils gathered on the device, update; stencils read back once per 1024 steps) "
                        "+ getz/getzmax")}
        s.close()

    peak, peak_kind = peaks()
    spl = steps_per_launch(variant)
    bytes_launch = BYTES_PER_CELL * cells  # per launch: one step, or two in the two-step kernel
    achieved = bytes_launch / (ms * 1e-3 / args.steps * spl) / 1e9
    traffic = profiled_traffic("pair_linear_step_c2.txt" if spl == 2 else "fused_linear_step_c2.txt")
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload],
                   "cells": cells, "parallelism": f"replicas x{world}",
                   "l2": ("working set 156 MB per step (8 fields x 19.5 MB) > 126 MB L2; no flush"
                          if args.workload == "c2" else "working set 3.5 MB: L2 resident (no flush)"),
                   "tile_variant": variant, "graph_chunk": 64},
        "roofline": pair_note({"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                               "frac": achieved / peak, "traffic": traffic,
                               "peak_kind": f"{peak_kind} (copy bandwidth)",
                               "algorithmic_bytes_per_launch": bytes_launch, "steps_per_launch": spl},
                              achieved * spl, "pair_linear_step_c2.txt"),
        "clocks": ck,
        "gpu_launches": launches,
    }
    if e2e:
        line["e2e"] = e2e
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return 0
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(make_case(nsteps=total))
    # ---------------- parity of the benchmarked runs ----------------
    chk = [done] + ([E] if e2e_state else [])
    ost = oracle_states(make_case(nsteps=max(chk)), chk)
    recs = [parity_record(got, ost[done]["layers"][0], done, H=case.root.H, ts=got["ts"][: done - 1],
                          ts_ref=ost[done]["ts"][: done - 1], what="engine member (the timed run)")]
    if e2e_state:
        recs.append(parity_record(e2e_state[0], ost[E]["layers"][0], E, H=case.root.H, ts=e2e_state[1],
                                  ts_ref=ost[E]["ts"], what="reference ABI session (the e2e run)"))
    line["parity"] = merge_parity(recs)
    # ---------------- the other workloads, compact (one GPU) ----------------
    if world == 1 and args.workload == "c2" and not args.no_sub:
        # at least 256 steps, so that a short headline run still times the
        # sub-records over whole step-chunk graphs
        sub_steps = max(256, min(args.steps, 3600))
        for key, fn in (("nested", lambda: bench_c3(torch, None, 1, local, sub_steps, args.warmup, -1)),
                        ("ensemble", lambda: bench_c4(torch, None, 1, local, sub_steps, args.warmup, 64, 2, -1)),
                        ("serving", lambda: bench_c5(torch, local, args.sub_requests, args.rate, args.budget_gb,
                                                     args.chunk, -1))):
            try:
                rec = fn()
            except Exception as exc:  # a sub-record never hides the headline line
                rec = {"error": f"{type(exc).__name__}: {exc}"}
            line[key] = rec
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None, help="timed steps (default 7200 for c2, 3600 otherwise)")
    ap.add_argument("--warmup", type=int, default=100)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sub", action="store_true", help="c2: skip the nested/ensemble/serving records")
    ap.add_argument("--variant", type=int, default=-1, help="fixed tile variant (skips the autotuner)")
    ap.add_argument("--workload", default="c2", choices=["c1", "c2", "c3", "c4", "c5"],
                    help="c2: the headline single grid; c3: the nested run; c4: the 64-scenario ensemble; "
                         "c5: the forecast-serving load")
    ap.add_argument("--requests", type=int, default=400, help="C5: requests in the trace")
    ap.add_argument("--sub-requests", type=int, default=40, help="c2: requests in the serving record's trace")
    ap.add_argument("--rate", type=float, default=2.0, help="C5: mean arrivals per second")
    ap.add_argument("--budget-gb", type=float, default=120.0, help="C5: HBM admission budget")
    ap.add_argument("--chunk", type=int, default=32, help="C5: steps between harvests")
    ap.add_argument("--no-plain", action="store_true", help="C5: skip the plain path")
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

    if args.workload == "c4":
        return run_c4(args, torch, dist, rank, world, local)
    if args.workload == "c3":
        return run_c3(args, torch, dist, rank, world, local)
    if args.workload == "c5":
        return run_c5(args, torch, dist, rank, world, local)
    return run_single(args, torch, dist, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
