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


# ------------------------------------------------------------------ workloads

# The measured configurations (team sizes, arena counts, starts, action distribution and
# culling of the four GPU workloads; c3 is the headline: learned cull vs exact BVH).
PRESETS = {
    "c3": dict(arenas=65536, team=3, mixed=False, reset="random", bias=False, cull="learned", graph=False,
               desc="soccar 3v3 x 65536 arenas"),
    "c1": dict(arenas=8192, team=2, mixed=False, reset="random", bias=False, cull="exact", graph=False,
               desc="soccar 2v2 x 8192 arenas"),
    "c2": dict(arenas=32768, team=0, mixed=True, reset="random", bias=False, cull="exact", graph=True,
               desc="mixed 32768 arenas (1v1:2v2:3v3 = 1:1:1) in one launch, env step replayed as a CUDA graph"),
    "c4": dict(arenas=131072, team=1, mixed=False, reset="high_contact", bias=True, cull="learned", graph=False,
               desc="soccar 1v1 x 131072 arenas, high-contact starts, boost/jump-biased actions, 4096-tick rollout"),
}


class Workload:
    """One preset: arenas, team sizes, the reset distribution (starts and finished episodes),
    the action distribution (uniform over the 90-entry table, or biased so that boost and
    jump are each pressed with probability 0.6)."""

    def __init__(self, args):
        p = PRESETS[args.config]
        self.preset = args.config
        self.num_arenas = args.arenas or p["arenas"]
        self.team_size = args.team_size or p["team"]
        self.mixed = p["mixed"]
        self.reset = p["reset"]
        self.bias = p["bias"]
        self.graph = p["graph"] and not args.no_graph
        self.cull = args.cull or p["cull"]
        self.tick_skip = args.tick_skip
        self.desc = p["desc"]

        self.offset, self.global_arenas, self.strong = 0, self.num_arenas, False

    def team_sizes(self):
        if self.mixed:
            return np.array([1 + ((self.offset + a) % 3) for a in range(self.num_arenas)], np.int32)
        return None

    def shard(self, rank, world):
        """Strong scaling: this rank's contiguous range of the preset's arenas, the ranges
        balanced by car count (shard_range)."""
        full = np.array([1 + (a % 3) for a in range(self.global_arenas)], np.int32) if self.mixed else None
        lo, hi = shard_range(full, self.global_arenas, rank, world)
        self.offset, self.num_arenas, self.strong = lo, hi - lo, True

    def processed(self, world):
        """Arenas all ranks step per env step: every rank's own copy (weak), or the one set (strong)."""
        return self.global_arenas if self.strong else self.num_arenas * world

    def name(self):
        t = self.tick_skip
        return (f"{self.desc}, tickSkip {t}: discrete actions -> {t} ticks -> AdvancedObs + masks -> 4 stub rewards + "
                f"terminals -> {'high-contact' if self.reset == 'high_contact' else 'random-state'} resets")

    def reset_mode(self, rsb):
        return rsb.RSB_RESET_HIGH_CONTACT if self.reset == "high_contact" else rsb.RSB_RESET_RANDOM_STATE

    def action_weights(self, lut):
        """Per-action sampling weights: uniform, or boost / jump each with probability 0.6."""
        if not self.bias:
            return None
        b, j = lut["boost"].astype(bool), lut["jump"].astype(bool)
        w = np.zeros(len(lut))
        for bb in (False, True):
            for jj in (False, True):
                sel = (b == bb) & (j == jj)
                if sel.any():
                    w[sel] = (0.6 if bb else 0.4) * (0.6 if jj else 0.4) / sel.sum()
        return w / w.sum()

    def config(self):
        ts = "1v1/2v2/3v3 (1:1:1)" if self.mixed else f"{self.team_size}v{self.team_size}"
        shard = {"arenas_this_rank": self.num_arenas, "first_arena": self.offset} if self.strong else {}
        return {"workload": self.name(), "preset": self.preset, "arenas": self.global_arenas, **shard, "teams": ts,
                "tick_skip": self.tick_skip, "narrowphase": "exact-bvh", "state": "fp32",
                "actions": ("boost and jump each pressed with p=0.6" if self.bias else
                            "uniform over the 90-action table") + ", new each env step",
                "obs": "AdvancedObs 51+29*cars floats + 90 masks per player",
                "rewards": "Goal, TouchBall, VelocityBallToGoal, VelocityPlayerToBall",
                "terminals": f"goal or {EPISODE_TICKS} ticks; finished arenas reset on the device",
                "graph": self.graph, "l2": "flushed between timed steps (256 MB write)"}


def shard_range(team_sizes, num_arenas, rank, world):
    """Rank `rank`'s contiguous arena range [lo, hi) of `num_arenas` arenas split over `world`
    ranks with about the same number of cars each (team_sizes None: every arena the same size,
    so the same number of arenas each).  Arenas are independent, so a split needs no exchange."""
    if team_sizes is None:
        cuts = [num_arenas * r // world for r in range(world + 1)]
    else:
        cum = np.concatenate([[0], np.cumsum(2 * np.asarray(team_sizes, np.int64))])
        cuts = [int(np.searchsorted(cum, cum[-1] * r / world, side="left")) for r in range(world)] + [num_arenas]
        cuts = [min(max(c, 0), num_arenas) for c in cuts]
    return cuts[rank], cuts[rank + 1]


class DevArray:
    """A device pointer of the library seen as a CUDA array (for torch.as_tensor)."""

    def __init__(self, ptr, shape, typestr):
        self.__cuda_array_interface__ = {"data": (ptr, False), "shape": shape, "typestr": typestr, "version": 3}


def reduce_max(value, dist, device=None):
    """The largest value over the ranks (timing of the slowest rank)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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
    if getattr(args, "strong", False):
        wl.shard(rank, world)
    rewards = rsb.default_rewards(pkg.engine_library(), episode_max_ticks=EPISODE_TICKS)
    batch = rsb.Batch(pkg.engine_library(), wl.num_arenas, team_size=wl.team_size or None,
                      team_sizes=wl.team_sizes(), meshes_path=pkg.MESHES_DIR, device=dev, seed=0x5EED0000 + rank,
                      rewards=rewards, cull_mode=rsb.RSB_CULL_EXACT)
    lut = rsb.default_action_lut(batch.lib)
    batch.set_action_lut(lut)
    culler = train_culler(batch, rsb, wl, rank) if wl.cull == "learned" else None
    reset_mode = wl.reset_mode(rsb)

    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    n_cars = max(1, batch.num_cars)
    actions = torch.zeros(n_cars, dtype=torch.int32, device=dev)
    weights = wl.action_weights(lut)
    weights_t = torch.tensor(weights, dtype=torch.float32, device=dev) if weights is not None else None
    counter = [0]

    def sample_actions():
        if weights_t is not None:
            actions.copy_(torch.multinomial(weights_t, n_cars, replacement=True).to(torch.int32))
        else:
            torch.randint(0, rsb.RSB_NUM_ACTIONS, (n_cars,), device=dev, dtype=torch.int32, out=actions)

    def one_step(ev=None):
        # the policy's actions arrive on the device; the whole env step stays there
        sample_actions()
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
        batch.reset_done(0x5EED1000 + counter[0], reset_mode, stream=sp)

    def start(mode):
        # every path starts from the same seeded state and action stream
        batch.set_cull_mode(mode)
        batch.reset_all(0x5EED0001 + rank, reset_mode)
        torch.cuda.manual_seed(0x5EED0003 + rank)
        counter[0] = 0

    def warm():
        # untimed: settle steps (the per-step cost climbs for a few dozen steps after a
        # random-state reset while the airborne half of the cars lands), then the warm-up
        with torch.cuda.stream(stream):
            for _ in range(args.settle + args.warmup):
                one_step()
        torch.cuda.synchronize()

    def timed(steps, clocks_out, graph=None):
        if dist is not None:
            dist.barrier()
        s0 = batch.stats()
        times, step_times = [], []
        with ClockSampler(dev) as clocks, torch.cuda.stream(stream):
            torch.cuda.synchronize()
            for _ in range(steps):
                flush.fill_(1.0)  # evict the L2 between timed steps
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                e0.record(stream)
                if graph is not None:
                    graph.replay()
                else:
                    one_step(ev)
                e1.record(stream)
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
                if graph is None:
                    step_times.append(ev[0].elapsed_time(ev[1]))
            torch.cuda.synchronize()
        clocks_out.append(clocks.summary())
        s1 = batch.stats()
        total_ms = reduce_max(float(sum(times)), dist, dev)
        value = wl.processed(world) * wl.tick_skip * steps / (total_ms / 1e3)
        delta = {k: s1[k] - s0[k] for k in ("narrowphase_queries", "culled_queries", "missed_contacts", "solver_rows")}
        return value, total_ms, step_times, delta

    clocks = []
    # exact-BVH path (also picks the step kernel's launch configuration)
    start(rsb.RSB_CULL_EXACT)
    warm()
    tune = batch.autotune(wl.tick_skip) if not args.no_autotune else []
    extra = {}
    steps = args.steps
    if wl.preset == "c4" and not getattr(args, "summary", False):
        steps = max(steps, 4096 // wl.tick_skip)  # one 4096-tick rollout
    start(rsb.RSB_CULL_EXACT)
    warm()
    if wl.graph:
        # kernel time from a short eager segment, then the library's captured env step
        # (rsb_env_graph_capture) replayed once per step after the policy's action sampling;
        # the reset seed advances on the device at every replay
        _, _, kernel_steps, _ = timed(3, [])
        batch.env_graph_capture(actions.data_ptr(), wl.tick_skip, reset_mode, 0x5EED2000 + rank)

        class _Replay:
            @staticmethod
            def replay():
                sample_actions()
                batch.env_graph_launch(stream=sp)

        value, total_ms, _, queries = timed(steps, clocks, _Replay)
        step_times = kernel_steps
        extra["graph"] = {"api": "rsb_env_graph_capture / rsb_env_graph_launch", "launches_per_replay": 6,
                          "note": "action sampling (torch) launched outside the graph"}
        ex_value = value
    else:
        value, total_ms, step_times, queries = timed(steps, clocks)
        ex_value, ex_ms, ex_steps, ex_q = value, total_ms, step_times, queries
    learned = None
    if culler is not None:
        start(rsb.RSB_CULL_LEARNED)
        warm()
        value, total_ms, step_times, queries = timed(steps, clocks)
        # the same run once more with the skipped tests executed and checked (the shortened
        # summaries skip the audits: their lockstep event comparison checks the learned path)
        audit = not getattr(args, "summary", False)

        def audited(mode):
            if not audit:
                return None, None
            start(mode)
            a0 = batch.stats()
            with torch.cuda.stream(stream):
                for _ in range(args.settle + args.warmup + min(steps, 64)):
                    one_step()
            torch.cuda.synchronize()
            a1 = batch.stats()
            return a1["missed_contacts"] - a0["missed_contacts"], a1["arenas_reverted"]

        missed, reverted = audited(rsb.RSB_CULL_LEARNED_AUDIT)
        tested = queries["culled_queries"] + queries["narrowphase_queries"]
        # the same rollout with the bound that needs no training (voxel distance field)
        start(rsb.RSB_CULL_VOXEL)
        warm()
        vx_value, vx_ms, vx_steps, vx_q = timed(steps, [])
        vx_missed, _ = audited(rsb.RSB_CULL_VOXEL_AUDIT)
        vx_tested = vx_q["culled_queries"] + vx_q["narrowphase_queries"]
        learned = {"train": culler, "culled_fraction": queries["culled_queries"] / max(1, tested),
                   "static_tests": queries, "audit_missed_contacts": missed,
                   "audit_arenas_reverted": reverted,
                   "exact_bvh": {"value": ex_value, "ms_per_step": ex_ms / steps,
                                 "kernel_ms": statistics.mean(ex_steps), "static_tests": ex_q},
                   "learned_over_exact": value / ex_value,
                   "voxel_bound": {"value": vx_value, "ms_per_step": vx_ms / steps,
                                   "kernel_ms": statistics.mean(vx_steps),
                                   "culled_fraction": vx_q["culled_queries"] / max(1, vx_tested),
                                   "audit_missed_contacts": vx_missed,
                                   "over_exact": vx_value / ex_value}}
        batch.set_cull_mode(rsb.RSB_CULL_LEARNED)
    if wl.preset == "c4":
        # the full 4,096-tick rollout; the folded summary of the headline line runs it on a
        # quarter of the arenas
        extra["stress"] = stress_events(pkg, batch, wl, rank, dev, 4096 // wl.tick_skip,
                                        wl.num_arenas // 4 if getattr(args, "summary", False) else None)

    # e2e through the public API with host buffers, as the collector's host path runs it:
    # host actions in (H2D), step, obs / masks / rewards / terminals back to the host (D2H),
    # then the finished arenas reset by index (H2D of the index list)
    # (host buffers page-locked once, outside the timed steps, and reused, as a collector
    # keeps its host vectors)
    e2e_times, h2d, d2h = [], [], []
    rng = np.random.default_rng(0x5EED0004 + rank)
    host_actions = batch.pin(rng.integers(0, rsb.RSB_NUM_ACTIONS, (16, n_cars)).astype(np.int32))
    outs = batch.pinned_outputs()
    out_bytes = sum(outs[k].nbytes for k in ("obs", "masks", "terminals")) + 4 * batch.num_cars
    for k in range(max(3, min(args.steps, 10))):
        t0 = time.perf_counter()
        batch.snapshot()
        batch.set_actions(host_actions[k % 16, :batch.num_cars])
        batch.step(wl.tick_skip)
        batch.build_obs()
        batch.build_rewards_terminals(wl.tick_skip)
        batch.copy_outputs(outs)
        done = np.nonzero(outs["terminals"])[0].astype(np.int32)
        if done.size:
            batch.reset_arenas(done, 0x5EED2000 + k, reset_mode)
        e2e_times.append(time.perf_counter() - t0)
        h2d.append(4 * batch.num_cars + 4 * done.size)
        d2h.append(out_bytes)
    e2e_value = wl.processed(world) * wl.tick_skip / reduce_max(statistics.median(e2e_times), dist, dev)

    # state ring: a device capture (slot copies in HBM) and a restore, against the reference's
    # capture path (synchronise, download every car, ball and pad state)
    ring = None
    if wl.preset == "c3" and not args.no_ring:
        batch.ring_configure(depth=10, capture_every=1)
        cap_ms, res_ms = [], []
        for k in range(6):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.ring_capture(stream=sp)
            e1.record(stream)
            torch.cuda.synchronize()
            cap_ms.append(e0.elapsed_time(e1))
        for k in range(5):
            t0 = time.perf_counter()
            n_rest = batch.ring_restore(stream=sp)
            torch.cuda.synchronize()
            res_ms.append(1e3 * (time.perf_counter() - t0))
        host_ms = []
        for k in range(3):
            t0 = time.perf_counter()
            batch.get_cars(), batch.get_balls(), batch.get_pads()
            host_ms.append(1e3 * (time.perf_counter() - t0))
        slot_bytes = (23 + 86 * rsb.RSB_MAX_CARS_PER_ARENA + 2 * rsb.RSB_NUM_PADS) * 4 * wl.num_arenas
        cms = statistics.median(cap_ms[1:])
        ring = {"slot_bytes": slot_bytes, "capture_ms": cms, "capture_gbs": 2 * slot_bytes / cms / 1e6,
                "restore_ms_wall": statistics.median(res_ms), "arenas_per_restore": n_rest,
                "reference_style_host_capture_ms": statistics.median(host_ms)}
        batch.ring_configure(depth=0)

    # ball prediction (BallPredTracker's ball-only rollout, the one VantaObs reads at 1/2/3 s)
    # of every arena's ball, slices left on the device
    pred = None
    if wl.preset == "c3" and not args.no_pred:
        pred_ms = []
        for k in range(4):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            batch.predict_ball((120, 240, 360), to_host=False, stream=sp)
            e1.record(stream)
            torch.cuda.synchronize()
            pred_ms.append(e0.elapsed_time(e1))
        pms = statistics.median(pred_ms[1:])
        pred = {"arenas": wl.num_arenas, "ticks": 360, "slices": [120, 240, 360], "ms": pms,
                "ball_ticks_per_s": wl.num_arenas * 360 / pms * 1e3}

    # the observation kernel alone (AdvancedObs rows + DefaultAction masks), L2 flushed between
    # calls (the 256 MB flush write, then a 256 MB read of it, so that the write-back of the
    # flush's own dirty lines happens before the timed call, not inside it): its algorithmic
    # bytes are the rows and masks written plus the records it reads (ball 9 words + team
    # size, per car 22 words + its 24-byte action, 34 pads x 2 words)
    peak, peak_kind = measured_peaks()
    obs = None
    if not args.no_obs_roofline:
        obs_ms = []
        with torch.cuda.stream(stream):
            for k in range(8):
                flush.fill_(1.0)
                flush.sum()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                batch.build_obs(stream=sp)
                e1.record(stream)
                e1.synchronize()
                obs_ms.append(e0.elapsed_time(e1))
        oms = statistics.median(obs_ms[2:])
        out_b = batch.num_cars * (4 * batch.obs_stride + rsb.RSB_NUM_ACTIONS)
        in_b = wl.num_arenas * (10 * 4 + 34 * 2 * 4) + batch.num_cars * (22 * 4 + 24)
        ach = (out_b + in_b) / (oms / 1e3) / 1e9
        obs = {"bound": "hbm", "kernel": "obsKernel", "achieved": ach, "peak": peak, "unit": "GB/s",
               "frac": ach / peak, "bytes_per_call": out_b + in_b, "ms": oms, "traffic": None,
               "l2": "flushed by a 256 MB write, then a read of it, before each call"}

    # VantaObs rows (rsb_build_vanta_obs) of every player, without and with the ball-only
    # prediction rollout the builder runs (360 ticks, slices at 1 / 2 / 3 s), L2 flushed the same
    # way; bytes: the rows written
    vanta = None
    if wl.preset == "c3" and not args.no_obs_roofline:
        vanta = {"players": batch.num_cars, "row_floats": rsb.RSB_VANTA_OBS_SIZE}
        for pred_on in (0, 1):
            batch.vanta_configure(predict_ball=pred_on)
            vms = []
            with torch.cuda.stream(stream):
                for k in range(5):
                    flush.fill_(1.0)
                    flush.sum()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    batch.build_vanta_obs(stream=sp)
                    e1.record(stream)
                    e1.synchronize()
                    vms.append(e0.elapsed_time(e1))
            ms = statistics.median(vms[1:])
            key = "with_ball_prediction" if pred_on else "rows_only"
            vanta[key] = {"ms": ms, "rows_gbs": batch.num_cars * rsb.RSB_VANTA_OBS_SIZE * 4 / ms / 1e6}

    # the reference's own GPU batch (RocketSimCuda's stepArenaKernel and env kernels, built for
    # sm_100a) on the same settled state and a seeded action stream, timed the same way
    refgpu = None
    if wl.preset == "c3" and not args.no_ref_gpu and world == 1:
        refgpu = reference_gpu(batch, wl, lut, pkg.MESHES_DIR, args.steps, args.warmup, args.settle)

    # roofline of the step kernel (the dominant launch): algorithmic bytes = persistent
    # state read + written per launch (the library reports it), over the kernel's own time
    alg_bytes = batch.stats()["state_bytes_per_step"]
    # DRAM traffic of a settled 3v3 step-kernel launch, measured by ncu on 8,192 arenas
    # (dram__bytes_read.sum + dram__bytes_write.sum = 58,409 B per arena, the threads' local
    # memory), scaled by the arenas; no capture exists for other team sizes
    traffic = 58409 * wl.num_arenas if (wl.team_size == 3 and not wl.mixed) else None
    kernel_s = statistics.mean(step_times) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / kernel_s / 1e9
    cfg = wl.config() | {"parallelism": f"arena-shards x{world}"}
    if learned is not None:
        cfg["narrowphase"] = "learned cull (exact BVH for every body the bound does not clear)"
    res = {
        "metric": METRIC, "value": value, "unit": "arena-ticks/s", "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": total_ms / steps, "higher_is_better": True,
        "scaling": "strong" if wl.strong else "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded random states)", "config": cfg,
        "roofline": {"bound": "hbm", "kernel": "stepKernel", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                     "traffic_source": "ncu dram bytes of a settled 3v3 x 8192 launch, scaled by arenas"
                     if traffic else None,
                     "bytes_per_launch": alg_bytes, "kernel_ms": kernel_s * 1e3,
                     "kernel_share": statistics.mean(step_times) / (total_ms / steps)},
        "e2e": {"value": e2e_value, "unit": "arena-ticks/s", "h2d_bytes_per_step": int(statistics.mean(h2d)),
                "d2h_bytes_per_step": int(statistics.mean(d2h))},
        # per env step: action expansion, (culler,) step, obs + masks, rewards + terminals, reset
        "gpu_launches": steps * ((6 if learned is not None else 5) + (1 if wl.graph else 0)),
        "learned_cull": learned,
        "state_ring": ring,
        "ball_prediction": pred,
        "reference_gpu": refgpu,
        "obs_roofline": obs,
        "vanta_obs": vanta,
        "autotune": tune,
        "clocks": clocks[-1],
        "clocks_exact": clocks[0],
    } | extra
    return res


REF_GPU_LIB = os.path.join(ROOT, "oracle", "_ref", "librscudaref.so")


def reference_gpu(batch, wl, lut, meshes, steps, warmup, settle):
    """The reference's batched GPU simulator (rsc::RocketSimCudaBatch, compiled for sm_100a by
    oracle/Makefile) on this workload: its arenas start from its own kickoff reset, run the
    same number of untimed settle steps as the engine, then the timed env steps (snapshot,
    action indices, Step(tickSkip), AdvancedObs + masks, rewards + terminals) on a seeded
    uniform action stream, timed with CUDA events.  (Its per-car SetCarState costs two
    synchronous copies per car, over a minute at 393,216 cars, so the engine's states are not
    copied in.)  None when the comparator was not built."""
    import ctypes as C

    if not os.path.exists(REF_GPU_LIB) or wl.mixed:
        return None
    lib = C.CDLL(REF_GPU_LIB)
    lib.rscref_create.restype = C.c_void_p
    lib.rscref_create.argtypes = [C.c_int32, C.c_int32, C.c_char_p]
    lib.rscref_destroy.argtypes = [C.c_void_p]
    for f in ("rscref_set_lut", "rscref_set_states", "rscref_time_env_steps", "rscref_positions"):
        getattr(lib, f).restype = C.c_int32
    lib.rscref_set_lut.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.rscref_set_states.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rscref_time_env_steps.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                          C.POINTER(C.c_float)]
    lib.rscref_positions.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rscref_step.restype = lib.rscref_cars_ground.restype = C.c_int32
    lib.rscref_step.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
    lib.rscref_cars_ground.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    t0 = time.perf_counter()
    h = lib.rscref_create(wl.num_arenas, wl.team_size, meshes.encode())
    if not h:
        return {"unavailable": "the reference batch could not be created"}
    try:
        lut_c = np.ascontiguousarray(lut)
        if lib.rscref_set_lut(h, lut_c.ctypes.data, len(lut_c)):
            return {"unavailable": "uploading the action table to the reference batch failed"}
        setup_s = time.perf_counter() - t0
        rng = np.random.default_rng(0x5EED0005)
        warmup = settle + warmup
        acts = rng.integers(0, 90, (warmup + steps, batch.num_cars)).astype(np.int32)
        ms = C.c_float()
        if lib.rscref_time_env_steps(h, acts.ctypes.data, warmup, steps, wl.tick_skip, C.byref(ms)):
            return {"unavailable": "the reference's env step reported a CUDA error"}
        cp = np.zeros((batch.num_cars, 3), np.float32)
        bp = np.zeros((wl.num_arenas, 3), np.float32)
        lib.rscref_positions(h, cp.ctypes.data, bp.ctypes.data)
        value = wl.num_arenas * wl.tick_skip * steps / (ms.value / 1e3)
        lib.rscref_destroy(h)
        h = None
        drift = reference_gpu_drift(load_pkg(), lib, meshes)
        return {"value": value, "drift_vs_reference_cpu": drift, "unit": "arena-ticks/s", "ms_per_step": ms.value / steps, "steps": steps,
                "warmup": warmup, "setup_s": setup_s, "finite_state": bool(np.isfinite(cp).all() and
                                                                          np.isfinite(bp).all()),
                "kernel": "RocketSimCuda stepArenaKernel + env kernels (reference sources, sm_100a)",
                "start": f"its kickoff reset, {settle} settle + {warmup - settle} warm-up env steps; seeded uniform actions"}
    finally:
        if h:
            lib.rscref_destroy(h)


def reference_gpu_drift(pkg, lib, meshes, n=256, ticks=120, seed=0x5EED0006):
    """What the reference GPU batch trades for its speed: it and the engine run `ticks` single
    ticks beside the reference CPU RocketSim (the oracle) from identical car and ball states
    (cars on the ground at random places, headings and speeds; balls anywhere) with the same
    controls, redrawn every 8 ticks.  Reported: car position drift from the CPU reference at
    the end (median, 99th percentile, uu) and the share of car-ticks whose on-ground flag
    differs, for the reference GPU batch and for the engine.  Arenas whose cars the CPU
    reference visits in another order than the engine are left out of the engine's figures."""
    import ctypes as C

    rsb = pkg.rsb
    ora = rsb.Batch(rsb.load_library(ORACLE_LIB), n, team_size=3, meshes_path=meshes, threads=8)
    eng = rsb.Batch(pkg.engine_library(), n, team_size=3, meshes_path=meshes)
    h = lib.rscref_create(n, 3, meshes.encode())
    if not h:
        return {"unavailable": "the reference batch could not be created"}
    try:
        rng = np.random.default_rng(seed)
        cars = ora.get_cars()
        m = len(cars)
        yaw = rng.uniform(-np.pi, np.pi, m)
        cy, sy = np.cos(yaw), np.sin(yaw)
        cars["pos"]["x"], cars["pos"]["y"], cars["pos"]["z"] = rng.uniform(-3500, 3500, m), rng.uniform(-4500, 4500, m), 17.0
        for f, v in (("forward", (cy, sy, 0 * cy)), ("right", (-sy, cy, 0 * cy)), ("up", (0 * cy, 0 * cy, 1 + 0 * cy))):
            for k, comp in enumerate("xyz"):
                cars["rot"][f][comp] = v[k]
        sp = rng.uniform(0, 2300, m)
        cars["vel"]["x"], cars["vel"]["y"], cars["vel"]["z"] = cy * sp, sy * sp, 0.0
        cars["boost"] = rng.uniform(0, 100, m)
        cars["is_on_ground"] = 1
        balls = np.zeros(n, rsb.BALL_DTYPE)
        for k, f in enumerate(("forward", "right", "up")):
            balls["rot"][f]["xyz"[k]] = 1.0
        balls["pos"]["x"], balls["pos"]["y"], balls["pos"]["z"] = (rng.uniform(-3900, 3900, n), rng.uniform(-5000, 5000, n),
                                                                  rng.uniform(100, 1900, n))
        for c in "xyz":
            balls["vel"][c] = rng.uniform(-3000, 3000, n)
        for b in (ora, eng):
            b.set_cars(cars)
            b.set_balls(balls)
        if lib.rscref_set_states(h, cars.ctypes.data, balls.ctypes.data):
            return {"unavailable": "setting the reference batch's states failed"}
        order = np.zeros(n, bool)
        fn = ora.lib.rsbref_car_order
        fn.restype, fn.argtypes = C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p]
        buf = np.zeros(8, np.int32)
        for a in range(n):
            k = fn(ora._h, a, buf.ctypes.data)
            order[a] = k >= 0 and np.array_equal(buf[:k], np.arange(k)[::-1])
        keep = np.repeat(order, 6)
        cp = np.zeros((m, 3), np.float32)
        gr = np.zeros(m, np.uint8)
        bp = np.zeros((n, 3), np.float32)
        flag_ref = flag_eng = 0
        for t in range(ticks):
            if t % 8 == 0:
                ctl = np.zeros(m, rsb.CONTROLS_DTYPE)
                for f in ("throttle", "steer", "pitch", "yaw", "roll"):
                    ctl[f] = rng.integers(-1, 2, m).astype(np.float32)
                ctl["jump"], ctl["boost"], ctl["handbrake"] = rng.random(m) < 0.2, rng.random(m) < 0.4, rng.random(m) < 0.15
                ora.set_controls(ctl)
                eng.set_controls(ctl)
            ora.step(1)
            eng.step(1)
            if lib.rscref_step(h, ctl.ctypes.data, 1):
                return {"unavailable": "the reference batch's step reported a CUDA error"}
            oc, ec = ora.get_cars(), eng.get_cars()
            lib.rscref_cars_ground(h, cp.ctypes.data, gr.ctypes.data, bp.ctypes.data)
            flag_ref += int((gr != oc["is_on_ground"]).sum())
            flag_eng += int((ec["is_on_ground"] != oc["is_on_ground"])[keep].sum())
        opos = np.stack([oc["pos"][k] for k in "xyz"], 1).astype(np.float64)
        epos = np.stack([ec["pos"][k] for k in "xyz"], 1).astype(np.float64)
        d_ref = np.linalg.norm(cp - opos, axis=1)
        d_eng = np.linalg.norm(epos - opos, axis=1)[keep]
        return {"arenas": n, "team_size": 3, "ticks": ticks,
                "reference_gpu": {"drift_median_uu": float(np.median(d_ref)), "drift_p99_uu": float(np.percentile(d_ref, 99)),
                                  "on_ground_mismatch": flag_ref / (m * ticks)},
                "engine": {"drift_median_uu": float(np.median(d_eng)), "drift_p99_uu": float(np.percentile(d_eng, 99)),
                           "on_ground_mismatch": flag_eng / (int(keep.sum()) * ticks), "arenas": int(order.sum())}}
    finally:
        lib.rscref_destroy(h)
        ora.close()
        eng.close()


def stress_events(pkg, trained, wl, rank, dev, steps, arenas=None):
    """Goal and demo events of `steps` env steps (512 = one 4,096-tick rollout at tickSkip 8)
    on the exact and on the learned path, run in lockstep on two fresh batches of `arenas`
    arenas built the same way (same seeds, same actions), step by step (goals: terminal flag
    1; demoed cars: the demo flag of the obs rows); finished arenas reset on the device with
    the workload's reset mode, the same seed on both sides."""
    import torch
    rsb = pkg.rsb
    weights, margin = trained.culler_get()
    lut = rsb.default_action_lut(trained.lib)
    w = wl.action_weights(lut)
    n = arenas or wl.num_arenas
    mk = []
    for mode in (rsb.RSB_CULL_EXACT, rsb.RSB_CULL_LEARNED):
        b = rsb.Batch(pkg.engine_library(), n, team_size=wl.team_size or None,
                      team_sizes=wl.team_sizes(), meshes_path=pkg.MESHES_DIR, device=dev, seed=0x5EED0000 + rank,
                      rewards=rsb.default_rewards(pkg.engine_library(), episode_max_ticks=EPISODE_TICKS),
                      cull_mode=mode)
        b.set_action_lut(lut)
        if mode != rsb.RSB_CULL_EXACT:
            b.culler_set(weights, margin)
        b.reset_all(0x5EED0001 + rank, wl.reset_mode(rsb))
        obs = torch.as_tensor(DevArray(b.device_ptr(rsb.RSB_BUF_OBS), (b.num_cars, b.obs_stride), "<f4"), device=dev)
        term = torch.as_tensor(DevArray(b.device_ptr(rsb.RSB_BUF_TERMINALS), (n,), "|u1"), device=dev)
        mk.append((b, obs, term))
    rng = np.random.default_rng(0x5EED0006 + rank)
    seqs = [[], []]
    s0 = [b.stats() for b, _, _ in mk]
    for step in range(steps):
        idx = rng.choice(len(lut), mk[0][0].num_cars, p=w).astype(np.int32)
        for k, (b, obs, term) in enumerate(mk):
            b.set_actions(idx)
            b.step(wl.tick_skip)
            b.build_obs()
            b.build_rewards_terminals(wl.tick_skip)
            b.sync()
            seqs[k].append((int((term == 1).sum().item()), int((obs[:, 51 + 27] > 0.5).sum().item())))
            b.reset_done(0x5EED4000 + step, wl.reset_mode(rsb))
    same_state = (mk[0][0].get_cars().tobytes() == mk[1][0].get_cars().tobytes() and
                  mk[0][0].get_balls().tobytes() == mk[1][0].get_balls().tobytes())
    s1 = [b.stats() for b, _, _ in mk]
    ex, le = seqs
    dq = [{k: s1[i][k] - s0[i][k] for k in ("culled_queries", "narrowphase_queries", "solver_rows")} for i in (0, 1)]
    for b, _, _ in mk:
        b.close()
    return {"arenas": n, "steps_compared": len(ex), "ticks": len(ex) * wl.tick_skip,
            "goals_exact": sum(g for g, _ in ex), "goals_learned": sum(g for g, _ in le),
            "demoed_car_steps_exact": sum(d for _, d in ex), "demoed_car_steps_learned": sum(d for _, d in le),
            "event_agreement": sum(a == b for a, b in zip(ex, le)) / len(ex), "final_state_identical": same_state,
            "culled_queries": dq[1]["culled_queries"],
            "culled_fraction": dq[1]["culled_queries"] / max(1, dq[1]["culled_queries"] + dq[1]["narrowphase_queries"]),
            "solver_rows_per_arena_tick": dq[0]["solver_rows"] / (n * wl.tick_skip * len(ex))}


def config_summaries(args, rank, world, dist):
    """The three other workloads, shortened, folded into the headline line: c1 and c2 (c2
    replaying the library's captured env step) with the headline's timed steps, c4 with the
    same timed steps and its lockstep exact-vs-learned event comparison over one full
    4,096-tick rollout on a quarter of its arenas (32,768), so that the whole line ends within
    a few minutes (`--config c4` runs the rollout at full size).  Each carries the reference's
    CPU rate on a short sample of the same workload."""
    import gc
    out = {}
    for name in ("c1", "c2", "c4"):
        a = argparse.Namespace(**vars(args))
        a.config, a.arenas, a.team_size, a.cull, a.summary = name, None, None, None, True
        a.no_ring = a.no_pred = a.no_obs_roofline = a.no_ref_gpu = True
        r = run_ours(a, rank, world, dist)
        gc.collect()
        s = {"workload": r["config"]["workload"], "value": r["value"], "unit": r["unit"], "steps": r["steps"],
             "ms_per_step": r["ms_per_step"], "e2e": r["e2e"]["value"], "gpu_launches": r["gpu_launches"],
             "step_kernel_ms": r["roofline"]["kernel_ms"], "clocks": r["clocks"]}
        for k in ("graph", "stress"):
            if k in r:
                s[k] = r[k]
        if r.get("learned_cull"):
            lc = r["learned_cull"]
            s["learned_cull"] = {"learned_over_exact": lc["learned_over_exact"], "exact_value": lc["exact_bvh"]["value"],
                                 "culled_fraction": lc["culled_fraction"],
                                 "audit_missed_contacts": lc["audit_missed_contacts"],
                                 "voxel_over_exact": lc["voxel_bound"]["over_exact"],
                                 "voxel_culled_fraction": lc["voxel_bound"]["culled_fraction"]}
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            ref = cpu_reference(a, sample_s=4.0)
            s["reference_cpu"] = {"value": ref["value"], "cores": ref["cores"], "sample": ref["sample"]}
            s["vs_reference_cpu"] = r["value"] / ref["value"]
        out[name] = s
    return out


# ------------------------------------------------------------------ GAE over a rollout buffer

GAE_METRIC = "GAE elements/s on 1 B200 (rsb_compute_gae over a flat rollout buffer)"
GAE_LIB_REF = os.path.join(ROOT, "oracle", "_ref", "libgaeref.so")
GAE_LIB_PORT = os.path.join(ROOT, "oracle", "_ref", "libgaeoracle.so")
GAE_PLAYERS, GAE_STEPS = 65536 * 6, 32
GAE_STD, GAE_CLIP = 1.7, 4.0


def gae_rollout(players, steps, seed):
    """A rollout buffer as the collector lays it out: each player's trajectory contiguous,
    a goal (NORMAL terminal) with probability 1/300 per step, every trajectory TRUNCATED at
    the rollout's end; rewards and values standard normal."""
    rng = np.random.default_rng(seed)
    term = np.zeros((players, steps), np.int8)
    term[rng.random((players, steps), dtype=np.float32) < 1.0 / 300.0] = 1
    term[:, -1] = 2
    term = term.ravel()
    T = term.size
    rews = rng.standard_normal(T, dtype=np.float32)
    vals = rng.standard_normal(T, dtype=np.float32)
    trunc = rng.standard_normal(int((term == 2).sum()), dtype=np.float32)
    return rews, term, vals, trunc


def gae_config(players, steps):
    return {"workload": f"GAE over {players} player trajectories x {steps} env steps (3v3 x 65536 arenas), "
                        f"player-major, goal terminal p=1/300 per step, truncated at the rollout end; "
                        f"gamma 0.99, lambda 0.95, returnStd {GAE_STD}, clipRange {GAE_CLIP}",
            "elements": players * steps, "layout": "flat float32 / int8 buffers in HBM",
            "l2": "flushed between timed calls (256 MB write); inputs + outputs 264 MB > L2"}


def gae_cpu_baseline(rews, term, vals, trunc):
    """The reference's own CPU recurrence for the device GAE (its parity test's CpuReference,
    built from the reference tree into oracle/_ref/libgaeref.so), one core, whole buffer; the
    C restatement of it when that library is absent."""
    import ctypes as C

    T = len(rews)
    outs = [np.zeros(T, np.float32) for _ in range(3)]
    clip = np.zeros(1, np.float32)
    p = lambda a: C.c_void_p(a.ctypes.data)  # noqa: E731
    if os.path.exists(GAE_LIB_REF):
        lib = C.CDLL(GAE_LIB_REF)
        f = lib.gaeref_cpu
        f.argtypes = [C.c_void_p] * 3 + [C.c_int32, C.c_void_p, C.c_int32, C.c_int32] + [C.c_float] * 4 + \
            [C.c_void_p] * 4
        t0 = time.perf_counter()
        f(p(rews), p(term), p(vals), len(vals), p(trunc), len(trunc), T, 0.99, 0.95, GAE_STD, GAE_CLIP,
          p(outs[0]), p(outs[1]), p(outs[2]), p(clip))
        kind = "reference"
    else:
        lib = C.CDLL(GAE_LIB_PORT)
        f = lib.gae_oracle
        f.argtypes = [C.c_void_p] * 4 + [C.c_int32] + [C.c_void_p] * 4 + [C.c_int32] + [C.c_float] * 4
        t0 = time.perf_counter()
        f(p(rews), p(term), p(vals), p(trunc), len(trunc), p(outs[0]), p(outs[1]), p(outs[2]), p(clip), T, 0.99,
          0.95, GAE_STD, GAE_CLIP)
        kind = "port"
    dt = time.perf_counter() - t0
    return {"value": T / dt, "unit": "elements/s", "cores": 1, "kind": kind,
            "sample": f"the whole {T}-element buffer once ({dt:.2f} s)"}


def run_gae(args, rank, world, dist, steps, warmup, reference_device=False):
    """Times rsb_compute_gae (or, for the reference arm, the reference's own
    rsc::ComputeGAEOnDevice built from its tree) on a device-resident rollout buffer."""
    import ctypes as C

    import torch

    pkg = load_pkg()
    rsb = pkg.rsb
    lib = pkg.engine_library()
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    rews, term, vals, trunc = gae_rollout(GAE_PLAYERS, GAE_STEPS, 0x5EED0006 + rank)
    T = len(rews)
    d_rews, d_term, d_vals, d_trunc = (torch.from_numpy(a).to(dev) for a in (rews, term, vals, trunc))
    d_out = torch.empty((3, T), dtype=torch.float32, device=dev)
    d_clip = torch.zeros(1, dtype=torch.float32, device=dev)
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    params = rsb.gae_params(lib, return_std=GAE_STD, clip_range=GAE_CLIP)
    if reference_device:
        ref = C.CDLL(GAE_LIB_REF)
        ref.gaeref_device.argtypes = [C.c_void_p] * 4 + [C.c_int32] + [C.c_void_p] * 4 + [C.c_int32] + \
            [C.c_float] * 4 + [C.c_void_p]
        ref.gaeref_device.restype = C.c_int32

        def call():
            ref.gaeref_device(d_rews.data_ptr(), d_term.data_ptr(), d_vals.data_ptr(), d_trunc.data_ptr(),
                              len(trunc), d_out[0].data_ptr(), d_out[1].data_ptr(), d_out[2].data_ptr(),
                              d_clip.data_ptr(), T, 0.99, 0.95, GAE_STD, GAE_CLIP, sp)
    else:
        def call():
            rsb.compute_gae_device(lib, d_rews.data_ptr(), d_term.data_ptr(), d_vals.data_ptr(), d_trunc.data_ptr(),
                                   len(trunc), d_out[0].data_ptr(), d_out[1].data_ptr(), d_out[2].data_ptr(),
                                   d_clip.data_ptr(), T, params, sp)
    with torch.cuda.stream(stream):
        for _ in range(warmup):
            call()
    torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    events = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    with ClockSampler(dev) as cs:
        with torch.cuda.stream(stream):
            for e0, e1 in events:
                flush.fill_(1.0)
                e0.record(stream)
                call()
                e1.record(stream)
        torch.cuda.synchronize()
    if dist is not None:
        dist.barrier()
    times = [e0.elapsed_time(e1) for e0, e1 in events]
    ms = reduce_max(statistics.mean(times), dist, dev)
    alg_bytes = T * (4 + 1 + 4 + 3 * 4) + 4 * len(trunc) + 4
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms / 1e3) / 1e9
    res = {"value": T * world / (ms / 1e3), "unit": "elements/s", "ms_per_call": ms, "elements": T,
           "roofline": {"bound": "hbm", "kernel": "gaeSegmentKernel (+ summary and scan)", "achieved": achieved,
                        "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        # ncu dram__bytes_read.sum + write.sum of gaeSegmentKernel on this buffer
                        "traffic": 213854464 if T == GAE_PLAYERS * GAE_STEPS else None,
                        "peak_kind": peak_kind, "bytes_per_call": alg_bytes},
           "gpu_launches": 3 * steps, "clocks": cs.summary()}
    if not reference_device:
        # e2e through the host entry point: copies in, kernels, copies out
        e2e = []
        for _ in range(max(3, min(steps, 5))):
            t0 = time.perf_counter()
            rsb.compute_gae(lib, rews, term, vals, trunc, params)
            e2e.append(time.perf_counter() - t0)
        res["e2e"] = {"value": T * world / reduce_max(statistics.median(e2e), dist, dev), "unit": "elements/s",
                      "h2d_bytes_per_step": T * 9 + 4 * len(trunc), "d2h_bytes_per_step": T * 12 + 4}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        res["cpu_baseline"] = gae_cpu_baseline(rews, term, vals, trunc)
    return res


# ------------------------------------------------------------------ CPU reference

def cpu_reference(args, sample_s=10.0, threads=None):
    """The reference's CPU path for the same env step: RocketSim arenas stepped on all host
    threads, then RLGymCPP's GameState / AdvancedObs / DefaultAction masks / stub rewards /
    terminal conditions, then the finished arenas reset.  (The CPU reference has no
    high-contact start; that preset's CPU sample starts from random states.)"""
    pkg = load_pkg()
    rsb = pkg.rsb
    lib = rsb.load_library(ORACLE_LIB)
    threads = threads or os.cpu_count() or 1
    wl = Workload(args)
    n = min(wl.num_arenas, 64 * threads)
    ts = wl.team_sizes()
    b = rsb.Batch(lib, n, team_size=wl.team_size or None, team_sizes=None if ts is None else ts[:n],
                  meshes_path=pkg.MESHES_DIR, threads=threads,
                  rewards=rsb.default_rewards(lib, episode_max_ticks=EPISODE_TICKS))
    b.reset_all(0x5EED0001, rsb.RSB_RESET_RANDOM_STATE)
    lut = rsb.default_action_lut(lib)
    b.set_action_lut(lut)
    rng = np.random.default_rng(0x5EED0003)
    w = wl.action_weights(lut)
    pool = [rng.choice(len(lut), max(1, b.num_cars), p=w).astype(np.int32) for _ in range(16)]

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


def gae_line(args, res, world, impl=None):
    line = {"metric": GAE_METRIC, "value": res["value"], "unit": "elements/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": res["ms_per_call"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded rollout buffer)",
            "config": gae_config(GAE_PLAYERS, GAE_STEPS)} | {k: v for k, v in res.items() if k not in (
                "value", "unit", "ms_per_call")}
    if impl:
        line["impl"] = impl
    return line


def run_reference(args):
    if args.config == "gae":
        # the reference's own implementation of this path is its device GAE
        # (RocketSimCuda/src/GAECuda.cu), built from its tree for sm_100a
        res = run_gae(args, 0, 1, None, args.steps, args.warmup, reference_device=True)
        line = gae_line(args, res, args.gpus, impl="reference")
        line["e2e"] = {"value": res["value"], "unit": "elements/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
        return line
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
    ap.add_argument("--strong", action="store_true",
                    help="split the preset's arenas over the ranks (balanced by car count) instead of one copy per rank")
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c3", choices=sorted(PRESETS) + ["gae"])
    ap.add_argument("--arenas", type=int, default=None)
    ap.add_argument("--team-size", type=int, default=None)
    ap.add_argument("--tick-skip", type=int, default=8)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--settle", type=int, default=40, help="untimed steps after each reset before warm-up")
    ap.add_argument("--no-graph", action="store_true")
    ap.add_argument("--cull", default=None, choices=["learned", "exact"])
    ap.add_argument("--ref-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-gae", action="store_true", help="skip the GAE measurement of the c3 line")
    ap.add_argument("--no-ring", action="store_true", help="skip the state-ring measurement of the c3 line")
    ap.add_argument("--no-pred", action="store_true", help="skip the ball-prediction measurement of the c3 line")
    ap.add_argument("--no-obs-roofline", action="store_true", help="skip timing the observation kernel alone")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="skip timing the reference's own GPU batch in the c3 line")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the shortened c1 / c2 / c4 summaries of the c3 line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

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
    if args.config == "gae":
        res = gae_line(args, run_gae(args, rank, world, dist, args.steps, args.warmup), world)
        if rank == 0:
            print(json.dumps(res), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    res = run_ours(args, rank, world, dist)
    # the next stage of the rollout: GAE over a rollout buffer of this size, device-resident
    if args.config == "c3" and not args.no_gae:
        res["gae"] = run_gae(args, rank, world, dist, steps=10, warmup=3)
    if args.config == "c3" and world == 1 and not args.no_configs:
        res["configs"] = config_summaries(args, rank, world, dist)
    if rank == 0:
        if not args.no_cpu_baseline and world == 1:
            res["cpu_baseline"] = cpu_reference(args, sample_s=args.ref_seconds)
        print(json.dumps(res), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
