"""Throughput benchmark: arena-ticks/s of the batched soccar simulator on B200.

One step = one env step of every arena, as the collector runs it: discrete actions in,
`tick_skip` physics ticks, AdvancedObs rows + action masks, the four stub rewards and the
terminal flags (goal, or 1,800 ticks since the reset), then the finished arenas reset to
random states.  Timing follows the measurement contract: W untimed warm-up steps, then K
steps, each bracketed by CUDA events on the stream the kernels run on, the L2 flushed
(256 MB write) between timed steps, max over ranks.  `--impl reference` times the
reference's own CPU implementation (RocketSim + RLGymCPP's env pieces, oracle/_ref) on the
host cores instead.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "emy-s-framework_b200")
ORACLE_LIB = os.path.join(ROOT, "oracle", "_ref", "librsref.so")
METRIC = "arena-ticks/s on 1 B200, learned-cull vs exact-BVH path; % of HBM roofline"
EPISODE_TICKS = 1800


def load_pkg():
    name = "emy_s_framework_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.stop_ev = threading.Event()
        self.thread = None

    def _run(self):
        while not self.stop_ev.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                     timeout=5).stdout.strip()
                if out:
                    self.samples.append([s.strip() for s in out.split(",")])
            except Exception:
                pass
            self.stop_ev.wait(0.2)

    def __enter__(self):
        self.thread = threading.Thread(target=self._run, daemon=True)
        self.thread.start()
        return self

    def __exit__(self, *exc):
        self.stop_ev.set()
        if self.thread:
            self.thread.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for s in self.samples:
            for k, name in enumerate(names):
                if len(s) > 5 + k and s[5 + k].lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.samples)}


# ------------------------------------------------------------------ workload

class Workload:
    """The timed configuration: soccar arenas started from seeded random states (RLGymCPP
    RandomState distribution), a fresh discrete action per car from the 90-entry table every
    env step, finished episodes reset to random states."""

    def __init__(self, args):
        self.num_arenas = args.arenas
        self.team_size = args.team_size
        self.tick_skip = args.tick_skip
        self.name = args.workload_name

    def config(self):
        return {"workload": self.name, "arenas": self.num_arenas, "team_size": self.team_size,
                "tick_skip": self.tick_skip, "narrowphase": "exact-bvh", "state": "fp32",
                "actions": "uniform over the 90-action table, new each env step",
                "obs": f"AdvancedObs {51 + 29 * 2 * self.team_size} floats + 90 masks per player",
                "rewards": "Goal, TouchBall, VelocityBallToGoal, VelocityPlayerToBall",
                "terminals": f"goal or {EPISODE_TICKS} ticks; finished arenas reset to random states",
                "l2": "flushed between timed steps (256 MB write)"}


# ------------------------------------------------------------------ our arm

def train_culler(batch, rsb, wl, rank):
    """Untimed: log body centres from short rollouts of this workload (random-state and
    high-contact starts), then train and calibrate the culler on the GPU."""
    rng = np.random.default_rng(0x5EED0005 + rank)
    t0 = time.perf_counter()
    for k in range(6):
        batch.reset_all(0x5EED3000 + k, rsb.RSB_RESET_RANDOM_STATE if k % 3 else rsb.RSB_RESET_HIGH_CONTACT)
        for _ in range(3):
            batch.set_actions(rng.integers(0, rsb.RSB_NUM_ACTIONS, batch.num_cars).astype(np.int32))
            batch.step(wl.tick_skip)
            batch.culler_log()
    rep = batch.culler_train(rsb.culler_config())
    rep["wall_s"] = time.perf_counter() - t0
    return rep


def run_ours(args, rank, world, dist):
    import torch

    pkg = load_pkg()
    rsb = pkg.rsb
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    wl = Workload(args)
    rewards = rsb.default_rewards(pkg.engine_library(), episode_max_ticks=EPISODE_TICKS)
    batch = rsb.Batch(pkg.engine_library(), wl.num_arenas, team_size=wl.team_size,
                      meshes_path=pkg.MESHES_DIR, device=dev, seed=0x5EED0000 + rank, rewards=rewards,
                      cull_mode=rsb.RSB_CULL_EXACT)
    batch.set_action_lut(rsb.default_action_lut(batch.lib))
    culler = train_culler(batch, rsb, wl, rank) if args.cull == "learned" else None

    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    gen = torch.Generator(device=f"cuda:{dev}")
    n_cars = max(1, batch.num_cars)
    actions = torch.empty(n_cars, dtype=torch.int32, device=dev)
    counter = [0]

    def one_step(ev=None):
        # the policy's actions arrive on the device; the whole env step stays there
        actions.random_(0, rsb.RSB_NUM_ACTIONS, generator=gen)
        batch.snapshot(stream=sp)
        batch.set_actions_device(actions.data_ptr(), batch.num_cars, stream=sp)
        if ev is not None:
            ev[0].record(stream)
        batch.step(wl.tick_skip, stream=sp)
        if ev is not None:
            ev[1].record(stream)
        batch.build_obs(stream=sp)
        batch.build_rewards_terminals(wl.tick_skip, stream=sp)
        counter[0] += 1
        batch.reset_done(0x5EED1000 + counter[0], rsb.RSB_RESET_RANDOM_STATE, stream=sp)

    def start(mode):
        # every path starts from the same seeded state and action stream
        batch.set_cull_mode(mode)
        batch.reset_all(0x5EED0001 + rank, rsb.RSB_RESET_RANDOM_STATE)
        gen.manual_seed(0x5EED0003 + rank)
        counter[0] = 0

    def timed(clocks_out):
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                one_step()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        s0 = batch.stats()
        times, step_times = [], []
        with ClockSampler(dev) as clocks, torch.cuda.stream(stream):
            torch.cuda.synchronize()
            for _ in range(args.steps):
                flush.fill_(1.0)  # evict the L2 between timed steps
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                e0.record(stream)
                one_step(ev)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                step_times.append(ev[0].elapsed_time(ev[1]))
            torch.cuda.synchronize()
        clocks_out.append(clocks.summary())
        s1 = batch.stats()
        total_ms = float(sum(times))
        if dist is not None:
            t = torch.tensor([total_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            total_ms = float(t.item())
            dist.barrier()
        value = wl.num_arenas * wl.tick_skip * args.steps * world / (total_ms / 1e3)
        queries = {k: s1[k] - s0[k] for k in ("narrowphase_queries", "culled_queries", "missed_contacts")}
        return value, total_ms, step_times, queries

    # exact-BVH path (also picks the step kernel's launch configuration)
    clocks = []
    start(rsb.RSB_CULL_EXACT)
    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            one_step()
    torch.cuda.synchronize()
    tune = batch.autotune(wl.tick_skip) if not args.no_autotune else []
    start(rsb.RSB_CULL_EXACT)
    ex_value, ex_ms, ex_steps, ex_q = timed(clocks)
    value, total_ms, step_times, queries = ex_value, ex_ms, ex_steps, ex_q
    learned = None
    if culler is not None:
        start(rsb.RSB_CULL_LEARNED)
        value, total_ms, step_times, queries = timed(clocks)
        # the same run once more with the skipped tests executed and checked
        start(rsb.RSB_CULL_LEARNED_AUDIT)
        s0 = batch.stats()
        with torch.cuda.stream(stream):
            for _ in range(args.warmup + args.steps):
                one_step()
        torch.cuda.synchronize()
        s1 = batch.stats()
        tested = queries["culled_queries"] + queries["narrowphase_queries"]
        learned = {"train": culler, "culled_fraction": queries["culled_queries"] / max(1, tested),
                   "static_tests": queries, "audit_missed_contacts": s1["missed_contacts"] - s0["missed_contacts"],
                   "audit_arenas_reverted": s1["arenas_reverted"],
                   "exact_bvh": {"value": ex_value, "ms_per_step": ex_ms / args.steps,
                                 "kernel_ms": statistics.mean(ex_steps), "static_tests": ex_q},
                   "learned_over_exact": value / ex_value}
        batch.set_cull_mode(rsb.RSB_CULL_LEARNED)

    # e2e through the public API with host buffers, as the collector's host path runs it:
    # host actions in (H2D), step, obs / masks / rewards / terminals back to the host (D2H),
    # then the finished arenas reset by index (H2D of the index list)
    e2e_times, h2d, d2h = [], [], []
    rng = np.random.default_rng(0x5EED0004 + rank)
    host_actions = rng.integers(0, rsb.RSB_NUM_ACTIONS, (16, n_cars)).astype(np.int32)
    for k in range(max(3, min(args.steps, 10))):
        t0 = time.perf_counter()
        batch.snapshot()
        batch.set_actions(host_actions[k % 16, :batch.num_cars])
        batch.step(wl.tick_skip)
        batch.build_obs()
        batch.build_rewards_terminals(wl.tick_skip)
        obs, masks, rew, term = batch.copy_obs(), batch.copy_masks(), batch.copy_rewards(), batch.copy_terminals()
        done = np.nonzero(term)[0].astype(np.int32)
        if done.size:
            batch.reset_arenas(done, 0x5EED2000 + k, rsb.RSB_RESET_RANDOM_STATE)
        e2e_times.append(time.perf_counter() - t0)
        h2d.append(4 * batch.num_cars + 4 * done.size)
        d2h.append(obs.nbytes + masks.nbytes + rew.nbytes + term.nbytes)
    e2e_value = wl.num_arenas * wl.tick_skip * world / statistics.median(e2e_times)

    # roofline of the step kernel (the dominant launch): algorithmic bytes = persistent
    # state read + written per launch (the library reports it), over the kernel's own time
    alg_bytes = batch.stats()["state_bytes_per_step"]
    kernel_s = statistics.mean(step_times) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / kernel_s / 1e9
    cfg = wl.config() | {"parallelism": f"arena-shards x{world}"}
    if learned is not None:
        cfg["narrowphase"] = "learned cull (exact BVH for every body the bound does not clear)"
    res = {
        "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random states)",
        "config": cfg,
        "roofline": {"bound": "hbm", "kernel": "stepKernel", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                     "bytes_per_launch": alg_bytes, "kernel_ms": kernel_s * 1e3,
                     "kernel_share": statistics.mean(step_times) / (total_ms / args.steps)},
        "e2e": {"value": e2e_value, "unit": "arena-ticks/s", "h2d_bytes_per_step": int(statistics.mean(h2d)),
                "d2h_bytes_per_step": int(statistics.mean(d2h))},
        # per env step: action expansion, (culler,) step, obs + masks, rewards + terminals, reset
        "gpu_launches": args.steps * (6 if learned is not None else 5),
        "learned_cull": learned,
        "autotune": tune,
        "clocks": clocks[-1],
        "clocks_exact": clocks[0],
    }
    return res


# ------------------------------------------------------------------ CPU reference

def cpu_reference(args, sample_s=10.0, threads=None):
    """The reference's CPU path for the same env step: RocketSim arenas stepped on all host
    threads, then RLGymCPP's GameState / AdvancedObs / DefaultAction masks / stub rewards /
    terminal conditions, then the finished arenas reset to random states."""
    pkg = load_pkg()
    rsb = pkg.rsb
    lib = rsb.load_library(ORACLE_LIB)
    threads = threads or os.cpu_count() or 1
    n = min(args.arenas, 64 * threads)
    wl = Workload(args)
    b = rsb.Batch(lib, n, team_size=wl.team_size, meshes_path=pkg.MESHES_DIR, threads=threads,
                  rewards=rsb.default_rewards(lib, episode_max_ticks=EPISODE_TICKS))
    b.reset_all(0x5EED0001, rsb.RSB_RESET_RANDOM_STATE)
    b.set_action_lut(rsb.default_action_lut(lib))
    rng = np.random.default_rng(0x5EED0003)
    pool = [rng.integers(0, rsb.RSB_NUM_ACTIONS, max(1, b.num_cars)).astype(np.int32) for _ in range(16)]

    def env_step(k):
        b.set_actions(pool[k % 16][:b.num_cars])
        b.step(wl.tick_skip)
        b.build_obs()
        b.build_rewards_terminals(wl.tick_skip)
        b.reset_done(k, rsb.RSB_RESET_RANDOM_STATE)

    env_step(0)
    steps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < sample_s:
        env_step(steps)
        steps += 1
    dt = time.perf_counter() - t0
    return {"value": n * wl.tick_skip * steps / dt, "unit": "arena-ticks/s", "cores": threads,
            "kind": "reference", "sample": f"{n} arenas x {steps} env steps of {wl.tick_skip} ticks "
                                          f"incl. obs/masks/rewards/terminals/resets ({dt:.1f} s)"}


def run_reference(args):
    cb = cpu_reference(args, sample_s=args.ref_seconds)
    wl = Workload(args)
    return {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": "arena-ticks/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded random states)",
            "config": wl.config(), "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "arena-ticks/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--arenas", type=int, default=65536)
    ap.add_argument("--team-size", type=int, default=3)
    ap.add_argument("--tick-skip", type=int, default=8)
    ap.add_argument("--workload-name", default=None)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--cull", default="learned", choices=["learned", "exact"])
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.workload_name is None:
        t = args.team_size
        args.workload_name = (f"soccar {t}v{t} x {args.arenas} arenas, tickSkip {args.tick_skip}: random discrete "
                              f"actions -> {args.tick_skip} ticks -> AdvancedObs + masks -> 4 stub rewards + "
                              "terminals -> random-state resets")

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod
    res = run_ours(args, rank, world, dist)
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            res["cpu_baseline"] = cpu_reference(args, sample_s=args.ref_seconds)
        print(json.dumps(res), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
