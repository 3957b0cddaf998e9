"""Benchmark: FP64 particle.turns/s of bmad_standard ring tracking on B200.

Workload (the configuration the metric is quoted on): the 64-cell FODO ring
with apertures (elliptical 20 x 10 mm on every quadrupole, rectangular
30 x 15 mm at the RF), 1,000,000 particles from a seeded 6D Gaussian at 3x the
base emittances, FP64.  One step = one persistent-kernel pass of
`--turns-per-step` turns over the whole bunch (a segment of the 10,000-turn
run).  value = particle.turns tracked (particles alive at the start of each
turn) / device time, summed over ranks.

Usage:
    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU: launched by torch.distributed.run, one rank per GPU; each rank
tracks its own 1M-particle bunch (weak scaling, no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "bmad-ecosystem_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "FP64 particle*turns/s, bmad_standard ring tracking (1M particles, apertures)"
UNIT = "particle*turns/s"
N_PARTICLES = 1_000_000
# FP64 operations per particle.turn on this ring (add/sub/mul/div/sqrt = 1
# each) and libm calls per particle.turn, counted by the instrumented oracle
# build over the config-1 beam (tests/test_flop_count.py keeps these current).
FLOPS_PER_PARTICLE_TURN = 98807.0
LIBM_PER_PARTICLE_TURN = 2315.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="bgt", choices=["bgt", "reference"])
    ap.add_argument("--turns-per-step", type=int, default=20)
    ap.add_argument("--particles", type=int, default=N_PARTICLES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="use the library's default launch shape")
    ap.add_argument("--tuning", default="", help="threads_per_block,blocks_per_sm (skips the autotuner)")
    return ap.parse_args()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.samples = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def turns_tracked(state0_alive, ix_turn_lost, state, t0, t1):
    """particle.turns with the particle alive at the start of each turn in [t0, t1)."""
    alive_end = state == 1
    tracked = np.where(alive_end, t1 - t0, np.clip(ix_turn_lost + 1, t0, t1) - t0)
    return int(np.sum(np.where(state0_alive, tracked, 0)))


def run_reference(args, rank, world):
    """Reference arm: the reference's CPU path for this workload -- the C
    restatement of Bmad's bmad_standard track1 in the reference's loop
    structure (element-outer, OpenMP over particles), on all host threads."""
    if rank != 0:
        return
    from bgt import rings
    from oracle import oracle as O

    lat = rings.fodo_ring(apertures=True)
    eles = O.to_eles(lat)
    param = O.make_param(lat.species.mass, lat.species.charge)
    threads = os.cpu_count() or 1
    n_sample, t_sample = 2000, 10
    v0 = rings.gaussian_beam(rings.CONFIG1_BEAM, n=n_sample)

    def step():
        v = v0.copy()
        b = O.beta_of(lat.p0c, v[5], lat.species.mass)
        st = np.ones(n_sample, np.int32)
        ie = np.full(n_sample, -1, np.int32)
        it = np.full(n_sample, -1, np.int32)
        t = time.perf_counter()
        O.track_turns(eles, lat.p0c, param, v, b, st, ie, it, t_sample, n_threads=threads, element_outer=True)
        return time.perf_counter() - t, turns_tracked(np.ones(n_sample, bool), it, st, 0, t_sample)

    for _ in range(args.warmup):
        step()
    tot_t, tot_u = 0.0, 0
    for _ in range(args.steps):
        dt, u = step()
        tot_t += dt
        tot_u += u
    val = tot_u / tot_t
    sample = f"{n_sample} particles x {t_sample} turns of the config-1 ring per step"
    line = {"impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "fodo64 ring + apertures, config-1 beam (sampled)", "particles": n_sample,
                       "turns_per_step": t_sample, "parallelism": f"openmp x{threads}"},
            "cpu_baseline": {"value": val, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline():
    """Oracle (C restatement) on the host cores, a bounded sample."""
    from bgt import rings
    from oracle import oracle as O

    lat = rings.fodo_ring(apertures=True)
    eles = O.to_eles(lat)
    param = O.make_param(lat.species.mass, lat.species.charge)
    threads = os.cpu_count() or 1
    n, turns = 4000, 20
    v = rings.gaussian_beam(rings.CONFIG1_BEAM, n=n)
    b = O.beta_of(lat.p0c, v[5], lat.species.mass)
    st = np.ones(n, np.int32)
    ie = np.full(n, -1, np.int32)
    it = np.full(n, -1, np.int32)
    t = time.perf_counter()
    O.track_turns(eles, lat.p0c, param, v, b, st, ie, it, turns, n_threads=threads, element_outer=True)
    dt = time.perf_counter() - t
    return {"value": turns_tracked(np.ones(n, bool), it, st, 0, turns) / dt, "unit": UNIT, "cores": threads,
            "kind": "port", "sample": f"{n} particles x {turns} turns, element-outer OpenMP (reference loop order)"}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from bgt import lattice as L
    from bgt import rings
    from bgt.track import Tracker, fp64_peak_tflops

    lat = rings.fodo_ring(apertures=True)
    tr = Tracker(lat, device=local)
    n = args.particles
    spec = rings.CONFIG1_BEAM
    spec = rings.BeamSpec(n, spec.emit_x, spec.emit_y, spec.sigma_z, spec.sigma_pz, spec.seed + 1000 * rank)
    v0 = rings.gaussian_beam(spec)
    dev = torch.device("cuda", local)
    vec = torch.tensor(v0, dtype=torch.float64, device=dev).contiguous()
    beta = torch.tensor(L.beta_of(lat.p0c, v0[5], lat.species.mass), device=dev)
    state = torch.ones(n, dtype=torch.int32, device=dev)
    ixe = torch.full((n,), -1, dtype=torch.int32, device=dev)
    ixt = torch.full((n,), -1, dtype=torch.int32, device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    stream = torch.cuda.current_stream(dev)
    T = args.turns_per_step
    tune_info = None
    if args.tuning:
        tpb, bps = (int(x) for x in args.tuning.split(","))
        tr.set_tuning(threads_per_block=tpb, blocks_per_sm=bps)
    elif not args.no_autotune:
        from bgt import autotune

        autotune.tune(tr, v0, turns=2, sample=min(n, 300_000))
        res = autotune.last_results(tr, n)
        tune_info = {"sample": res["sample"], "turns": res["turns"],
                     "candidates_ms": [[round(ms, 3), t["threads_per_block"], t["blocks_per_sm"]]
                                       for ms, t in res["all"]]}

    def barrier():
        if dist:
            dist.barrier()

    turn = 0
    for _ in range(args.warmup):
        tr.track_turns_device(vec, beta, state, ixe, ixt, T, turn0=turn, stream=stream)
        turn += T
    torch.cuda.synchronize()

    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    units = 0
    launches0 = tr.launch_count
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            flush.fill_(float(k))  # evict L2 between timed steps (outside the events)
            alive0 = (state == 1).cpu().numpy()
            t0 = turn
            ev[k][0].record(stream)
            tr.track_turns_device(vec, beta, state, ixe, ixt, T, turn0=turn, stream=stream)
            ev[k][1].record(stream)
            turn += T
            torch.cuda.synchronize()
            units += turns_tracked(alive0, ixt.cpu().numpy(), state.cpu().numpy(), t0, turn)
        torch.cuda.synchronize()
    barrier()
    launches = tr.launch_count - launches0
    ms = sum(a.elapsed_time(b) for a, b in ev)
    t_local = ms / 1e3
    t_max = t_local
    units_all = units
    if dist:
        tt = torch.tensor([t_local], dtype=torch.float64, device=dev)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
        uu = torch.tensor([units], dtype=torch.float64, device=dev)
        dist.all_reduce(uu, op=dist.ReduceOp.SUM)
        units_all = int(uu.item())
    value = units_all / t_max

    # ---- end to end through the public API with host buffers ----
    e2e = None
    if not args.no_e2e:
        hb = tr.make_bunch(v0.copy())
        tr.track_turns(hb, 1)  # warm-up (staging buffers)
        hb = tr.make_bunch(v0.copy())
        e2e_units, e2e_t = 0, 0.0
        for k in range(max(1, min(args.steps, 5))):
            alive0 = hb.state == 1
            t0k = T * k
            barrier()
            ts = time.perf_counter()
            tr.track_turns(hb, T, turn0=t0k)
            e2e_t += time.perf_counter() - ts
            e2e_units += turns_tracked(alive0, hb.ix_turn_lost, hb.state, t0k, t0k + T)
        if dist:
            tt = torch.tensor([e2e_t], dtype=torch.float64, device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            e2e_t = float(tt.item())
            uu = torch.tensor([e2e_units], dtype=torch.float64, device=dev)
            dist.all_reduce(uu, op=dist.ReduceOp.SUM)
            e2e_units = int(uu.item())
        per = 6 * 8 + 8 + 3 * 4
        e2e = {"value": e2e_units / e2e_t, "unit": UNIT, "h2d_bytes_per_step": per * n,
               "d2h_bytes_per_step": per * n}

    if rank == 0:
        peak = fp64_peak_tflops(local)
        units_per_launch = units / max(1, launches)
        launch_s = t_local / max(1, launches)
        achieved = FLOPS_PER_PARTICLE_TURN * units_per_launch / launch_s / 1e12
        roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                    "frac": achieved / peak, "traffic": None,
                    "peak_source": "measured: DFMA throughput probe (bgt_fp64_peak_tflops) on this GPU; "
                                   "MEASURED_PEAKS.json has no FP64 figure",
                    "flops_per_unit": FLOPS_PER_PARTICLE_TURN, "libm_calls_per_unit": LIBM_PER_PARTICLE_TURN}
        cpu = None if args.no_cpu_baseline or world > 1 else cpu_baseline()
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": "fodo64 ring (770 elements) + apertures, config-1 beam",
                           "particles_per_gpu": n, "turns_per_step": T, "parallelism": f"particles x{world} GPUs",
                           "l2": "flushed between timed steps (256 MB write)"},
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clk.summary(), "tuning": tr.get_tuning(), "autotune": tune_info}
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
