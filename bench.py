#!/usr/bin/env python
"""Benchmark of the Oncolytica step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload scale|plain_small]
    python bench.py --impl reference ...        # the CPU reference arm

A step is one simulation step of the tumour-spheroid workload (fields, grid,
rule, contact).  The default workload ``scale`` is 1,000,000 agents with two
256^3 FP32 fields (O2 and drug).  ``value`` is agent-steps/s of the whole job
(sum over replicas / max device time over ranks) with the state resident in
HBM; ``e2e`` runs the same steps through Engine.run_step(collect_metrics=True,
wait=False) with a parameter upload from pinned host memory before each step
and the metric readback after it, each step's metrics read on the host once
the next step is queued (``value_waiting``: read before it is queued).  One
JSON line is printed by rank 0.

Multi-GPU: the step does not shard (the stencil and the agents share one
domain), so N GPUs run N independent replicas (different seeds), no
collective in the step ("replicas only"); the timed region is bracketed by
barriers and the slowest rank's device time is used.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from dataclasses import replace

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "agent-steps/s + voxel-updates/s, batched vs plain FP32 on 1 B200; p99 sim latency"
P99_TARGET_S = 8.0  # serving mix: p99 time to completion (see measure_serving)
UNIT = "agent-steps/s"


def parse() -> argparse.Namespace:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="scale")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0 = as many as --steps")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-graphs", action="store_true", help="eager launches instead of CUDA graphs of whole steps")
    ap.add_argument("--no-tune", action="store_true", help="default kernel shapes instead of measured ones")
    ap.add_argument("--sims", type=int, default=512, help="members of the batched workload (--workload batch)")
    ap.add_argument("--solo-sample", type=int, default=0, help="members also timed one at a time (--workload batch)")
    ap.add_argument("--storage", default="f32", choices=["f32", "bf16", "f16", "bf16_sr", "f16_sr"],
                    help="field storage of --workload batch")
    ap.add_argument("--extra-steps", type=int, default=10,
                    help="timed steps of the batched and 16-bit measurements added to the default line")
    ap.add_argument("--no-extras", action="store_true", help="leave the batched and 16-bit measurements out")
    ap.add_argument("--rate", type=float, default=20.0, help="request arrivals per second (--workload serve)")
    ap.add_argument("--duration", type=float, default=120.0, help="seconds of arrivals (--workload serve)")
    ap.add_argument("--serve-seconds", type=float, default=15.0,
                    help="seconds of arrivals of the serving run added to the default line")
    ap.add_argument("--storages", default="bf16_sr,f16_sr", help="field storages of --workload precision")
    ap.add_argument("--workload-base", default="scale",
                    help="the workload --workload precision runs; batch:K[,K...] = members K of the batched sweep")
    ap.add_argument("--error-steps", type=int, default=10,
                    help="steps of the field-error measurement added to the default line")
    ap.add_argument("--encoding", default="auto", choices=["auto", "value", "deficit", "offset3"],
                    help="16-bit element encoding of --workload batch")
    ap.add_argument("--contact", default="auto", choices=["auto", "flat", "nested"],
                    help="contact walk of the scale workload (auto: the tuner's choice)")
    ap.add_argument("--grid", type=int, default=256, help="field edge of --workload stencil")
    ap.add_argument("--stencil-pair", default="0,1024,512",
                    help="CTA sizes of the two-substep pass timed by --workload stencil (0: one substep per pass)")
    ap.add_argument("--encodings", default="value,deficit,offset3",
                    help="16-bit element encodings timed by --workload stencil")
    ap.add_argument("--l2-keep", default="0,30,45,60",
                    help="shares (%%) of the FP32 field kept in L2 timed by --workload stencil (one substep per pass)")
    return ap.parse_args()


def env_ranks() -> tuple[int, int, int]:
    return (int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)),
            int(os.environ.get("LOCAL_RANK", 0)))


def measured_peaks() -> dict:
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return {"hbm_gbs": float(d["hbm_gbs"]), "src": "measured"}
    return {"hbm_gbs": 6650.0, "src": "fallback"}


class ClockSampler:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id: str | None):
        self.gpu_id = gpu_id
        self.proc = None
        self.path = None

    def start(self) -> None:
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        cmd = ["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits", "-lms", "50"]
        if self.gpu_id:
            cmd += ["-i", self.gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.2)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                f = [x.strip() for x in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for name, v in zip(names, f[5:9]):
                    if v.lower() == "active":
                        reasons.add(name)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def read_traffic(kernel: str, nvox: int) -> int | None:
    """DRAM bytes per launch of `kernel` from a committed ncu summary
    (profiles/<kernel>*.txt line "dram_bytes_per_launch <bytes> voxels <n>"),
    scaled to this workload's voxels."""
    d = os.path.join(REPO, "profiles")
    if not os.path.isdir(d):
        return None
    for name in sorted(os.listdir(d)):
        if not (name.startswith(kernel) and name.endswith(".txt")):
            continue
        with open(os.path.join(d, name)) as fh:
            for line in fh:
                p = line.split()
                if len(p) >= 4 and p[0] == "dram_bytes_per_launch" and p[2] == "voxels":
                    return int(round(int(p[1]) * nvox / int(p[3])))
    return None


# ------------------------------------------------------------------ CPU (oracle) timing

def time_oracle_steps(orc, steps: int, nthreads: int = 0) -> dict:
    """``steps`` whole steps of the C oracle, each timed on the host clock:
    the field phase with every substep of every field, then the agent phase
    (sort, rule, contact).  Agent-steps count the live agents at each step's
    start, as the device counter does."""
    t_fields = t_agents = 0.0
    agents = 0
    for _ in range(steps):
        n = orc.rows
        agents += int((orc.dead[:n] == 0).sum())
        t0 = time.perf_counter()
        orc.fields(nthreads)
        t1 = time.perf_counter()
        orc.agents_part(nthreads)
        t2 = time.perf_counter()
        t_fields += t1 - t0
        t_agents += t2 - t1
    return {"t_fields": t_fields, "t_agents": t_agents, "agents": agents, "steps": steps}


def make_oracle(spec):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # the CPU restatement (checker and CPU baseline only)

    from oncolytica_b200 import workloads as W

    st = W.initial_state(spec)
    o2, drug = W.initial_fields(spec)
    return oracle.TumourOracle(spec, st, o2, drug, spec.capacity)


def reference_cpu_backend_record() -> dict | None:
    """The reference's own CPU backend (pure Python, one core) timed on a
    small configuration of the plain workload, as recorded by
    oracle/time_reference_cpu.py where the reference checkout exists (it does
    not travel with this repository)."""
    p = os.path.join(REPO, "oracle", "reference_cpu_backend.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        return json.load(fh)


def workload_config(spec, world: int = 1) -> dict:
    """The ``config`` object of a scale/plain_small line; the GPU arm and the
    reference arm print the same one."""
    nvox = int(np.prod(spec.field_dims))
    return {"workload": spec.name, "agents": spec.n_agents, "fields": "o2+drug" if spec.has_drug else "o2",
            "field_dims": list(spec.field_dims), "substeps": [spec.S_o2, spec.S_drug],
            "bins": list(spec.tissue_dims), "l2": "inputs larger than L2 (field state "
            f"{(5 if spec.has_drug else 3) * 4 * nvox / 1e6:.0f} MB)", "parallelism": f"replicas x{world}"}


def cpu_baseline(spec, steps: int = 3, warmup: int = 1) -> dict:
    """The C oracle on every host thread: ``warmup`` untimed then ``steps``
    timed whole steps of the workload from its initial state (the same
    procedure as the reference arm, shorter)."""
    orc = make_oracle(spec)
    cores = os.cpu_count() or 1
    time_oracle_steps(orc, warmup)
    r = time_oracle_steps(orc, steps)
    tot = r["t_fields"] + r["t_agents"]
    out = {"value": r["agents"] / tot, "unit": UNIT, "cores": cores, "kind": "port",
           "sample": f"{steps} whole step(s) of {spec.name} after {warmup} warm-up step(s): every substep of every "
                     f"field ({spec.S_o2}+{spec.S_drug}) and the full agent phase ({spec.n_agents} agents at the "
                     f"start: sort, rule, contact); C oracle, OpenMP on {cores} threads",
           "seconds": tot, "fields_s_per_step": r["t_fields"] / steps, "agents_s_per_step": r["t_agents"] / steps,
           "voxel_updates_per_s": spec.voxel_updates_per_step() * steps / r["t_fields"]}
    rec = reference_cpu_backend_record()
    if rec is not None:
        out["reference_cpu_backend"] = rec
    return out


def run_reference(args) -> None:
    rank, world, _ = env_ranks()
    if rank != 0:
        return
    from oncolytica_b200 import workloads as W

    spec = W.CONFIGS[args.workload]
    orc = make_oracle(spec)
    cores = os.cpu_count() or 1
    time_oracle_steps(orc, args.warmup)
    r = time_oracle_steps(orc, args.steps)
    tot = r["t_fields"] + r["t_agents"]
    value = r["agents"] / tot
    vox = spec.voxel_updates_per_step() * args.steps / tot
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (numpy default_rng, seed 0 + rank)", "config": workload_config(spec, world),
            "voxel_updates_per_s": vox,
            "phases_s_per_step": {"fields": r["t_fields"] / args.steps, "agents": r["t_agents"] / args.steps},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                             "sample": f"{args.steps} whole steps after {args.warmup} warm-up steps, every substep "
                                       "of every field and the full agent phase, host clock; the C oracle (the "
                                       "reference's algorithm restated: its own GPU path needs a graphics adapter, "
                                       "unavailable on this box)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm

def reduce_over_ranks(dist, t):
    """Combine one rank's ``[seconds_or_ms, units...]`` float64 tensor over all ranks.

    Returns ``(slowest time, t)`` where the time is the MAX of ``t[0]`` over ranks and ``t``
    now holds the SUM over ranks of every entry (its units are the whole job's). Every rank
    makes the same two collectives in the same order; with ``dist`` None (one rank) ``t`` is
    returned unchanged.
    """
    if dist is None:
        return float(t[0]), t
    mx = t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(mx[0]), t


def run_b200(args) -> None:
    import torch

    rank, world, local = env_ranks()
    if world != args.gpus and not (world == 1 and args.gpus == 1):
        print(f"warning: --gpus {args.gpus} but WORLD_SIZE={world}", file=sys.stderr)
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    from oncolytica_b200 import workloads as W

    base = W.CONFIGS[args.workload]
    spec = replace(base, seed=base.seed + rank)
    state0 = W.initial_state(spec)
    eng = W.build_engine(spec, state0)
    # kernel shapes and variants measured on this workload (state restored)
    from oncolytica_b200 import _lib, autotune

    tuning = autotune.tune_engine(eng) if not args.no_tune else {"tuning": None}
    if args.contact != "auto":
        # a fixed contact walk (profiling one variant); the other choices stay tuned
        t = dict(tuning["tuning"] or {"stencil_tile": [8, 8], "batch_tile_depth": 16, "stencil_pair": [0, 0]})
        t["contact_variant"] = {"flat": _lib.OLC_CONTACT_FLAT, "nested": _lib.OLC_CONTACT_NESTED}[args.contact]
        tuning = dict(tuning, tuning=t)
        autotune.apply_engine(eng, tuning)
    eng.set_graphs(not args.no_graphs)
    be = eng._backend_impl
    dev = torch.device("cuda", local)

    def tuned(e):
        autotune.apply_engine(e, tuning)
        return e
    props = torch.cuda.get_device_properties(dev)
    gpu_id = None
    try:
        gpu_id = "GPU-" + str(props.uuid)
    except Exception:
        pass

    # warm-up (untimed)
    eng.run_steps(args.warmup)
    gc.collect()
    torch.cuda.synchronize(dev)
    c0 = be.counters()
    stream = torch.cuda.current_stream(dev)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks = ClockSampler(gpu_id)
    if dist:
        dist.barrier()
    torch.cuda.synchronize(dev)
    clocks.start()
    start.record(stream)
    eng.run_steps(args.steps)
    end.record(stream)
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    if dist:
        dist.barrier()
    ms = start.elapsed_time(end)
    c1 = be.counters()
    # stage timing: a second engine from the same initial state replays the
    # same warm-up and steps eagerly with CUDA events between the stages (the
    # trajectory is deterministic, so it is the timed region's work); the
    # dominant kernel's launch time comes from here
    eng.close()
    del eng, be
    eng = tuned(W.build_engine(spec, state0))
    be = eng._backend_impl
    eng.run_steps(args.warmup)
    be.set_profiling(True)
    eng.run_steps(args.steps)
    prof = be.profile()
    be.set_profiling(False)
    assert be.counters()["agent_steps"] == c1["agent_steps"], "profiled window diverged from the timed one"
    agent_steps = c1["agent_steps"] - c0["agent_steps"]
    vox = spec.voxel_updates_per_step() * args.steps
    tot = torch.tensor([ms, float(agent_steps), float(vox)], dtype=torch.float64, device=dev)
    ms_max, tot = reduce_over_ranks(dist, tot)
    total_agent_steps, total_vox = float(tot[1]), float(tot[2])
    value = total_agent_steps / (ms_max / 1e3)

    # e2e through the public API on a fresh engine over the same warm-up and
    # steps as the timed region: params H2D before, metrics D2H after each step
    from oncolytica_b200.compiler.emit_cuda import pack_params

    eng.close()
    del eng, be
    gc.collect()
    eng = tuned(W.build_engine(spec, state0))
    eng.set_graphs(not args.no_graphs)
    be = eng._backend_impl
    eng.run_steps(args.warmup)
    params = eng._sim._params
    kw = {k: getattr(params, k) for k in eng._sim._params.__dataclass_fields__}
    e2e_steps = args.steps if args.e2e_steps <= 0 else max(1, min(args.e2e_steps, args.steps))
    torch.cuda.synchronize(dev)
    c2 = be.counters()
    if dist:
        dist.barrier()
    # each step: params H2D from pinned memory, the step, its metrics D2H;
    # step k's metrics are read on the host once step k+1 is queued
    t0 = time.perf_counter()
    pend = None
    for _ in range(e2e_steps):
        eng.update_params(**kw)
        h = eng.run_step(collect_metrics=True, wait=False)
        if pend is not None:
            pend.result()
        pend = h
    pend.result()
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - t0
    c3 = be.counters()
    e2e_agents = c3["agent_steps"] - c2["agent_steps"]
    # the same steps on a fresh engine with every step's metrics read before
    # the next is queued
    eng.close()
    del eng, be
    gc.collect()
    eng = tuned(W.build_engine(spec, state0))
    eng.set_graphs(not args.no_graphs)
    be = eng._backend_impl
    eng.run_steps(args.warmup)
    torch.cuda.synchronize(dev)
    c3w = be.counters()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        eng.update_params(**kw)
        eng.run_step(collect_metrics=True)
    torch.cuda.synchronize(dev)
    wait_s = time.perf_counter() - t0
    c4 = be.counters()
    assert c4["agent_steps"] - c3w["agent_steps"] == e2e_agents, "waiting e2e run diverged from the queued one"
    t2 = torch.tensor([e2e_s, float(e2e_agents)], dtype=torch.float64, device=dev)
    e2e_s, t2 = reduce_over_ranks(dist, t2)
    e2e_value = float(t2[1]) / e2e_s
    t3 = torch.tensor([wait_s, float(c4["agent_steps"] - c3w["agent_steps"])], dtype=torch.float64, device=dev)
    wait_s, t3 = reduce_over_ranks(dist, t3)
    e2e_wait_value = float(t3[1]) / wait_s
    h2d = len(pack_params(be.layout, params))
    d2h = 4 * max(1, len(be.layout.metrics))
    eng.close()
    del eng, be
    gc.collect()

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    # roofline of the dominant kernel (the 7-point substep)
    import numpy as np

    nvox = int(np.prod(spec.field_dims))
    peaks = measured_peaks()
    sub_ms = prof["ms_substeps"] / max(1, prof["substep_launches"])  # per substep (a pair counts two)
    alg_bytes = 8 * nvox  # read 4 B + write 4 B per voxel and launch (FP32)
    pair = tuple((tuning.get("tuning") or {}).get("stencil_pair", (0, 0)))
    paired = pair[0] > 0 and autotune.pair_applies(pair[0], spec.field_dims)
    if paired:
        # two substeps per launch: the odd substep of each field is a single
        # pass, so a pair launch takes the fields' time less those singles,
        # timed at the single-pass time per substep the tuner measured
        subs = [S for S in (spec.S_o2, spec.S_drug) if S]
        n_pairs = sum(S // 2 for S in subs)
        n_single = sum(S % 2 for S in subs)
        t = tuning["tuning"]
        single_ms = (tuning.get("measured_ms", {}).get("substeps", {})
                     .get(f"{t['stencil_tile'][0]}x{t['stencil_tile'][1]}", sub_ms * sum(subs)) / sum(subs))
        launch_ms = max(1e-6, (sub_ms * sum(subs) - n_single * single_ms) / max(1, n_pairs))
        kernel = f"k_substep_pair<{pair[0]}> (two 7-point FTCS substeps per pass, FP32, TMA plane ring)"
        traffic = read_traffic("k_substep_pair", nvox)
    else:
        launch_ms = sub_ms
        kernel = "k_substep_x4 (7-point FTCS, FP32, 4-wide rows, TMA tiles)"
        keep = (tuning.get("tuning") or {}).get("l2_keep_pct", 0)
        traffic = read_traffic("k_substep_x4_l2slab" if keep else "k_substep_x4_scale", nvox)
    achieved = alg_bytes / (launch_ms / 1e3) / 1e9
    steps_done = max(1, prof["steps"])
    stages = {k[3:]: prof[k] / steps_done for k in ("ms_sink", "ms_substeps", "ms_grid", "ms_rules",
                                                     "ms_contact", "ms_collect")}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (numpy default_rng, seed 0 + rank)",
"config": workload_config(spec, world),
        "voxel_updates_per_s": total_vox / (ms_max / 1e3),
        "agents_end": c1["n_agents"],
        "roofline": {"bound": "hbm", "kernel": kernel, "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                     "peak_src": peaks["src"], "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
                     "launch_ms": launch_ms, "substeps_per_launch": 2 if paired else 1,
                     # one-substep-per-pass stream model (8 B per voxel-substep): above 1.0
                     # only when passes carry more than one substep
                     "per_substep_us": sub_ms * 1e3,
                     "stream_model_frac_per_substep": alg_bytes / (sub_ms / 1e3) / 1e9 / peaks["hbm_gbs"]},
        "stages_ms_per_step": stages,
        # launches per step do not depend on the data: the profiled window of
        # the same length launches exactly what the timed graphs replay
        "gpu_launches": int(prof["kernel_launches"]),
        "graphs": not args.no_graphs,
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                "steps": e2e_steps,
                "api": "Engine.update_params + Engine.run_step(collect_metrics=True, wait=False); "
                       "step k's metrics read on the host (PendingReadback.result) after step k+1 is queued",
                "value_waiting": e2e_wait_value,
                "api_waiting": "Engine.update_params + Engine.run_step(collect_metrics=True): each step's "
                               "metrics read before the next step is queued (same steps, fresh engine)"},
        "clocks": clk,
        "status": c1["status"],
        "tuning": autotune.summary(tuning) if tuning["tuning"] else "defaults (--no-tune)",
    }
    if world == 1 and not args.no_extras:
        # the metric's other halves on the same GPU: the batched sweep (FP32
        # and BF16 with stochastic rounding) and 16-bit field storage of the
        # scale workload
        torch.cuda.empty_cache()
        line["batched"] = {st: measure_batch(args.sims, args.extra_steps, 3, graphs=not args.no_graphs,
                                             solo_sample=64 if st == "f32" else 0, storage=st)
                           for st in ("f32", "f16_sr")}
        # the batched forms against the plain FP32 path on the same sweep:
        # members sampled evenly over the sweep run one at a time on solo FP32
        # engines (CUDA graphs); their agent-steps/s is the plain path's rate
        solo = line["batched"]["f32"]["solo_vs_batch_sample"]
        for st, r in line["batched"].items():
            r["vs_plain_fp32"] = {"plain_fp32_agent_steps_per_s": solo["solo_agent_steps_per_s"],
                                  "members_sampled": solo["members"],
                                  "ratio": r["agent_steps_per_s"] / solo["solo_agent_steps_per_s"]}
        line["precision"] = {st: measure_storage(spec, st, args.extra_steps * 5, 3, graphs=not args.no_graphs)
                             for st in ("f16_sr", "bf16_sr", "f16")}
        # the precision tier's field error against FP64 on this workload (a
        # short run; --workload precision --steps 1000 runs the full length)
        if args.error_steps > 0:
            torch.cuda.empty_cache()
            line["field_error"] = measure_field_error(spec, ("bf16_sr", "f16_sr"), args.error_steps)
        torch.cuda.empty_cache()
        # the serving mix, shortened to args.serve_seconds of arrivals
        line["serving"] = measure_serving(args.rate, args.serve_seconds, seed=0, storage="f16_sr", solo_sample=4)
    if world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(spec)
    rec = recorded_runs()
    if rec:
        line["recorded"] = rec
    line["summary"] = summarise(line)
    assert_clean(line)
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def assert_clean(line: dict) -> None:
    """Every device status word a line reports must be 0 (no dropped child,
    no look-back or TMA wait that gave up, no capacity overflow)."""
    from oncolytica_b200._lib import status_names

    bad = []
    if line.get("status"):
        bad.append(("step", line["status"]))
    for st, r in (line.get("batched") or {}).items():
        if r.get("status"):
            bad.append((f"batched {st}", r["status"]))
    for st, r in (line.get("precision") or {}).items():
        if r.get("status"):
            bad.append((f"precision {st}", r["status"]))
    for st, v in ((line.get("field_error") or {}).get("status") or {}).items():
        if v:
            bad.append((f"field error {st}", v))
    if line.get("serving") and line["serving"].get("device_status"):
        bad.append(("serving", line["serving"]["device_status"]))
    if bad:
        raise RuntimeError("device status set: " + "; ".join(f"{w}: {s:#x} {status_names(s)}" for w, s in bad))


def recorded_runs() -> dict | None:
    """The long runs measured with their own commands (profiles/recorded_runs.json:
    the 1,000-step field error of the scale workload, the 500-step batched
    sweep against the plain FP32 path), copied into the line as recorded."""
    p = os.path.join(REPO, "profiles", "recorded_runs.json")
    if not os.path.exists(p):
        return None
    with open(p) as fh:
        return json.load(fh)


def summarise(line: dict) -> dict:
    """The headline figures of a line's nested measurements, short, printed
    last so that a log that keeps only the end of the line still shows them."""
    out = {"agent_steps_per_s": line["value"], "e2e": line["e2e"]["value"],
           "e2e_waiting": line["e2e"].get("value_waiting"), "roofline_frac": line["roofline"]["frac"]}
    if line.get("cpu_baseline"):
        out["cpu_port"] = line["cpu_baseline"]["value"]
    for st, r in (line.get("batched") or {}).items():
        out[f"batched_{st}_vs_plain_fp32"] = round(r["vs_plain_fp32"]["ratio"], 3)
    for st, r in (line.get("precision") or {}).items():
        out[f"{st}_ms_per_step"] = round(r["ms_per_step"], 4)
    fe = line.get("field_error")
    if fe:
        out[f"rel_l2_vs_fp64_after_{fe['steps']}_steps"] = {
            st: {f: float(f"{e['rel_l2']:.3g}") for f, e in r.items()} for st, r in fe["final"].items()}
    if line.get("serving"):
        sv = line["serving"]
        out["serving_p50_p99_s"] = [round(sv["ttc_p50_s"], 3), round(sv["ttc_p99_s"], 3)]
        if "p99_target_s" in sv:
            out["serving_p99_target_s"] = round(sv["p99_target_s"], 3)
            out["serving_p99_target_met"] = sv["p99_target_met"]
    rec = line.get("recorded")
    if rec:
        pr = rec["precision_scale_1000_steps"]["rel_l2_and_max_abs_after_1000_steps"]
        out["recorded_rel_l2_after_1000_steps"] = {st: {f: e["rel_l2"] for f, e in r.items()} for st, r in pr.items()}
        out["recorded_batched_500_steps_vs_plain_fp32"] = {
            k: v["vs_plain_fp32"] for k, v in rec["batched_sweep_500_steps"]["batched"].items()}
        mem = rec.get("batched_members_field_error_500_steps")
        if mem:
            # worst relative L2 over the checked sweep members, per storage (values stored)
            worst = {}
            for m in mem["by_member"].values():
                for st, r in m["rel_l2"].items():
                    worst[st] = max(worst.get(st, 0.0), *r.values())
            out["recorded_sweep_members_worst_rel_l2_500_steps_values"] = worst
    return out


def measure_storage(spec, storage: str, steps: int, warmup: int, graphs: bool = True) -> dict:
    """The scale workload with 16-bit field storage: whole-step device time
    (graphs) and the substep kernel's live launch time from a profiled replay
    of the same steps; roofline on 4 B per voxel-substep (2 B read + 2 B
    written)."""
    import torch

    from oncolytica_b200 import workloads as W

    sp = replace(spec, storage=storage)
    state0 = W.initial_state(sp)
    dev = torch.device("cuda", torch.cuda.current_device())
    eng = W.build_engine(sp, state0)
    eng.set_graphs(graphs)
    be = eng._backend_impl
    eng.run_steps(warmup)
    torch.cuda.synchronize(dev)
    c0 = be.counters()
    st = torch.cuda.current_stream(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    eng.run_steps(steps)
    e1.record(st)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    agent_steps = be.counters()["agent_steps"] - c0["agent_steps"]
    del eng, be
    torch.cuda.empty_cache()
    eng = W.build_engine(sp, state0)
    be = eng._backend_impl
    eng.run_steps(warmup)
    be.set_profiling(True)
    eng.run_steps(steps)
    prof = be.profile()
    be.set_profiling(False)
    del eng, be
    torch.cuda.empty_cache()
    nvox = int(np.prod(sp.field_dims))
    sub_ms = prof["ms_substeps"] / max(1, prof["substep_launches"])
    peaks = measured_peaks()
    achieved = 4 * nvox / (sub_ms / 1e3) / 1e9
    return {"storage": storage, "steps": steps, "ms_per_step": ms / steps,
            "agent_steps_per_s": agent_steps / (ms / 1e3),
            "voxel_updates_per_s": sp.voxel_updates_per_step() * steps / (ms / 1e3),
            "substep_us": sub_ms * 1e3, "substep_alg_bytes": 4 * nvox, "substep_achieved_gbs": achieved,
            "substep_frac_of_measured_hbm": achieved / peaks["hbm_gbs"],
            "stages_ms_per_step": {k[3:]: prof[k] / max(1, prof["steps"]) for k in
                                   ("ms_sink", "ms_substeps", "ms_grid", "ms_rules", "ms_contact", "ms_collect")}}


def measure_field_error(spec, storages: tuple, steps: int, checkpoints: tuple = (), nthreads: int = 0) -> dict:
    """Field error of 16-bit storage against FP64 on the workload at its own
    size.  Every storage runs its own simulation from the same initial state;
    before each step its O2 sink (the uptake the agents deposited, which the
    step's reaction consumes) is copied to the host, and an FP64 evaluation of
    the field scheme (the oracle's orc_diffuse_f64: implicit sink, then S
    substeps with decay in every substep) advances with it, so the comparison
    isolates the storage's rounding from the agents' trajectory.  The drug
    field takes no sinks, so one FP64 run serves every storage.  Relative L2,
    maximum and mean absolute error of each field after ``steps`` steps (and
    at ``checkpoints``)."""
    import torch

    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle  # the FP64 evaluation (checker only)

    from oncolytica_b200 import workloads as W

    state0 = W.initial_state(spec)
    o2_0, drug_0 = W.initial_fields(spec)
    shp = tuple(spec.field_dims[::-1])
    engines = {st: W.build_engine(replace(spec, storage=st), state0) for st in storages}
    for eng in engines.values():
        # children dropped at capacity change the agents' trajectory, not the
        # comparison: each run's own sinks are replayed into its FP64 field
        eng.on_device_status = "warn"
    ref = {st: np.ascontiguousarray(o2_0, dtype=np.float64) for st in storages}
    tmp = np.zeros(shp, np.float64)
    drug = np.ascontiguousarray(drug_0, dtype=np.float64) if spec.has_drug else None
    enc = {st: {f: eng._backend_impl.field_codec(f)[1] for f in eng._backend_impl.layout.chem_fields}
           for st, eng in engines.items()}
    t_cpu = 0.0
    out = {"steps": steps, "workload": spec.name, "field_dims": list(spec.field_dims),
           "reference": "oracle orc_diffuse_f64 (FP64) with each run's per-step O2 sinks replayed", "by_step": {}}

    def errors(step: int) -> None:
        rec = {}
        for st, eng in engines.items():
            be = eng._backend_impl
            fb = be._current()[1]
            rec[st] = {}
            for name, r in (("o2", ref[st]), ("drug", drug)):
                if r is None:
                    continue
                got = be._field_values(be.layout.chem_fields.index(name), fb).reshape(shp).astype(np.float64)
                d = got - r
                rec[st][name] = {"rel_l2": float(np.linalg.norm(d) / np.linalg.norm(r)),
                                 "max_abs": float(np.abs(d).max()), "mean_abs": float(np.abs(d).mean()),
                                 "encoding": int(enc[st][name])}
        out["by_step"][str(step)] = rec

    for step in range(steps):
        sinks = {}
        for st, eng in engines.items():
            be = eng._backend_impl
            sinks[st] = be.fields_dev[be.layout.chem_fields.index("o2")][2].cpu().numpy().reshape(shp)
            eng.run_step()
        t0 = time.perf_counter()
        for st in storages:
            ref[st] = oracle.diffuse_f64(ref[st], sinks[st], spec.dx, spec.dt, spec.D_o2, 0.0, spec.bnd_o2,
                                         spec.S_o2, nthreads=nthreads, tmp=tmp)
        if drug is not None:
            drug = oracle.diffuse_f64(drug, None, spec.dx, spec.dt, spec.D_drug, spec.decay_drug, spec.bnd_drug,
                                      spec.S_drug, nthreads=nthreads, tmp=tmp)
        t_cpu += time.perf_counter() - t0
        if step + 1 in checkpoints and step + 1 != steps:
            torch.cuda.synchronize()
            errors(step + 1)
    torch.cuda.synchronize()
    errors(steps)
    out["final"] = out["by_step"][str(steps)]
    out["status"] = {st: eng._backend_impl.counters()["status"] for st, eng in engines.items()}
    out["agents_end"] = {st: eng._backend_impl.counters()["n_agents"] for st, eng in engines.items()}
    out["max_agents"] = spec.capacity
    out["fp64_host_seconds"] = t_cpu
    for eng in engines.values():
        eng.close()
    return out


def precision_specs(workload_base: str, steps: int, sims: int = 512, encoding: str = "auto", rank: int = 0) -> list:
    """The workloads of --workload precision: a named configuration, or with
    ``batch:K[,K...]`` members K of the batched sweep (each reproduces its
    batched run bit for bit) with the batched run's capacity for ``steps``
    steps; ``encoding`` other than "auto" overrides the element encoding."""
    from oncolytica_b200 import workloads as W

    if workload_base.startswith("batch:"):
        members = W.batched_specs(sims, steps=steps)
        specs = [members[int(k)] for k in workload_base[len("batch:"):].split(",") if k]
        if not specs:
            raise ValueError("--workload-base batch: names no member")
    else:
        base = W.CONFIGS[workload_base]
        # room for the population of a long run (unchecked growth doubles it
        # about every 140 steps until O2 runs short)
        specs = [replace(base, seed=base.seed + rank, capacity=32 * base.n_agents)]
    if encoding != "auto":
        specs = [replace(sp, encoding=encoding) for sp in specs]
    return specs


def run_precision_workload(args) -> None:
    """Field error of the scale workload with 16-bit fields against FP64
    (``--storages``, ``--steps`` steps; checkpoints every quarter)."""
    import torch

    rank, world, local = env_ranks()
    torch.cuda.set_device(local)
    storages = tuple(s for s in args.storages.split(",") if s)
    cps = tuple(sorted({max(1, args.steps * k // 4) for k in (1, 2, 3)}))
    specs = precision_specs(args.workload_base, args.steps, args.sims, args.encoding, rank)
    runs = [measure_field_error(sp, storages, args.steps, checkpoints=cps) for sp in specs]
    r = runs[0] if len(runs) == 1 else {"members": runs}
    spec = specs[0]
    worst = max(e["rel_l2"] for run in runs for st in run["final"].values() for e in st.values())
    line = {"metric": METRIC, "value": worst, "unit": "relative L2 field error vs FP64 (worst field and storage)",
            "n_gpus": world, "steps": args.steps, "warmup": 0, "ms_per_step": None, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "/".join(storages) + " fields, f32 update",
            "data": "synthetic (numpy default_rng, seed 0 + rank)",
            "config": {"workload": ", ".join(sp.name for sp in specs) + " with 16-bit fields (field error against FP64)",
                       "field_dims": [list(sp.field_dims) for sp in specs] if len(specs) > 1 else list(spec.field_dims),
                       "storages": list(storages), "encoding": args.encoding},
            "precision": r}
    if rank == 0:
        print(json.dumps(line), flush=True)


def measure_batch(n_sims: int, steps: int, warmup: int, graphs: bool = True, solo_sample: int = 0,
                  seed: int = 0, storage: str = "f32", encoding: str = "auto") -> dict:
    """The batched workload: ``n_sims`` sweep members (uneven agent counts,
    grids and diffusion) stepped by one BatchEngine.  Device time with CUDA
    events over ``steps`` steps after ``warmup``; stage times from a second
    batch replaying the same steps eagerly with events between stages.  With
    ``solo_sample`` > 0 the same number of members (spread over the sweep) also
    run one at a time through solo engines, for the batched-vs-solo ratio."""
    import torch

    from oncolytica_b200 import workloads as W

    specs = [replace(sp, storage=storage, encoding=encoding)
             for sp in W.batched_specs(n_sims, seed=seed, steps=warmup + steps)]
    states = [W.initial_state(sp) for sp in specs]
    dev = torch.device("cuda", torch.cuda.current_device())

    def timed(b):
        b.run_steps(warmup)
        torch.cuda.synchronize(dev)
        c0 = b.counters()
        st = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        b.run_steps(steps)
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1), b.counters()["agent_steps"] - c0["agent_steps"], b

    tune = None
    if storage == "f32":  # the batched FP32 substep's tile depth per member grid size
        from oncolytica_b200 import autotune

        tune = autotune.tune_batch(lambda: W.build_batch(specs, states), steps=2)

    def build():
        b = W.build_batch(specs, states)
        if tune is not None:
            autotune.apply_batch(b, tune["depths"])
        return b

    batch = build()
    batch.set_graphs(graphs)
    ms, agent_steps, batch = timed(batch)
    status = batch.counters()["status"]
    del batch
    torch.cuda.empty_cache()
    prof_batch = build()
    prof_batch.run_steps(warmup)
    prof_batch.set_profiling(True)
    prof_batch.run_steps(steps)
    prof = prof_batch.profile()
    prof_batch.set_profiling(False)
    del prof_batch
    torch.cuda.empty_cache()
    vox = sum(int(np.prod(sp.field_dims)) * (sp.S_o2 + sp.S_drug) for sp in specs) * steps
    out = {"n_sims": n_sims, "steps": steps, "warmup": warmup, "ms_per_step": ms / steps,
           "agent_steps_per_s": agent_steps / (ms / 1e3), "voxel_updates_per_s": vox / (ms / 1e3),
           "agents_start": int(sum(sp.n_agents for sp in specs)),
           "voxels_per_field": int(sum(int(np.prod(sp.field_dims)) for sp in specs)),
           "substeps_o2": [min(sp.S_o2 for sp in specs), max(sp.S_o2 for sp in specs)],
           "stages_ms_per_step": {k[3:]: prof[k] / max(1, prof["steps"]) for k in
                                  ("ms_sink", "ms_substeps", "ms_grid", "ms_rules", "ms_contact", "ms_collect")},
           "gpu_launches_per_step": prof["kernel_launches"] / max(1, prof["steps"]),
           "graphs": graphs, "status": status, "storage": storage, "encoding": encoding,
           "tile_depths": tune["depths"] if tune is not None else None}
    if solo_sample:
        idx = np.linspace(0, n_sims - 1, solo_sample).astype(int)
        sub = [specs[i] for i in idx]
        sub_states = [states[i] for i in idx]
        solo_ms, solo_as = 0.0, 0
        for sp, st0 in zip(sub, sub_states):
            # the plain path: the member alone on a solo engine with FP32 fields
            e = W.build_engine(replace(sp, storage="f32"), st0)
            e.set_graphs(graphs)
            m, a, _ = timed(_SoloAsBatch(e))
            solo_ms += m
            solo_as += a
            del e
        bsub = W.build_batch(sub, sub_states)
        if tune is not None:
            autotune.apply_batch(bsub, tune["depths"])
        bsub.set_graphs(graphs)
        bm, ba, _ = timed(bsub)
        del bsub
        out["solo_vs_batch_sample"] = {"members": solo_sample, "solo_agent_steps_per_s": solo_as / (solo_ms / 1e3),
                                      "solo_storage": "f32", "batch_storage": storage,
                                      "batch_agent_steps_per_s": ba / (bm / 1e3),
                                      "speedup": (ba / (bm / 1e3)) / (solo_as / (solo_ms / 1e3))}
    return out


def measure_serving(rate: float, duration: float, seed: int = 0, storage: str = "f32", solo_sample: int = 0,
                    hbm_fraction: float = 0.3, max_slots: int = 2048, depth: int = 6, prefetch: float = 0.5) -> dict:
    """The serving mix: requests drawn like sweep members (steps U{100..1000})
    arrive as a Poisson process at ``rate``/s for ``duration`` s and are served
    by one pool (continuous batching, admission by free HBM: the arenas take
    ``hbm_fraction`` of the free device memory, split as the mix uses them).
    Wall-clock time to completion per request (arrival to result on the host)
    and whole-run throughput (device agent-step counter / wall time from the
    first arrival to the last result).  With ``solo_sample`` > 0 that many
    requests (spread over the mix) also run alone on the plain FP32 path (solo
    engine, CUDA graphs), for the throughput ratio."""
    import torch

    from oncolytica_b200 import workloads as W
    from oncolytica_b200._geometry import voxel_table_size
    from oncolytica_b200.serving import Footprint, PoolDevice, ServingPool, SimRequest, plan_arenas

    sched = W.serving_schedule(rate=rate, duration=duration, seed=seed, storage=storage)
    specs = [sp for _, sp, _ in sched]
    mix = [Footprint(sp.capacity, voxel_table_size(sp.tissue_dims), int(np.prod(sp.field_dims))) for sp in specs]
    tdims = tuple(max(sp.tissue_dims[i] for sp in specs) for i in range(3))
    free, _ = torch.cuda.mem_get_info()
    code = {"f32": 0, "bf16": 1, "f16": 2, "bf16_sr": 3, "f16_sr": 4}[storage]
    plan = plan_arenas(int(hbm_fraction * free), mix, n_cols=8, storages=[code, code], sinks=[True, False])
    proto = W.configure_engine(specs[0])
    dev = PoolDevice(proto, max_slots=max_slots, max_tissue_dims=tdims, **plan)
    # warm-up outside the timed run: one short request loads every kernel
    warm = ServingPool(dev)
    e, s = W.configure_engine(specs[0])
    warm.submit(SimRequest(e, s, 3, return_state=True))
    warm.drain()
    pool = ServingPool(dev, depth=depth)
    dev.time_steps = True

    def factory(sp, n):
        return lambda: SimRequest(*W.configure_engine(sp), n, return_state=True)

    arrivals = [(t, factory(sp, n)) for t, sp, n in sched]
    torch.cuda.synchronize()
    c0 = dev.counters()
    t0 = time.perf_counter()
    results = pool.serve(arrivals, prefetch=prefetch)
    t1 = time.perf_counter()
    c1 = dev.counters()
    busy = dev.device_seconds()
    done = [r for r in results if r.status == "done"]
    ttc = np.array([r.ttc for r in done]) if done else np.zeros(1)
    wait = np.array([r.admitted - r.arrival for r in done]) if done else np.zeros(1)
    wall = t1 - t0
    agent_steps = c1["agent_steps"] - c0["agent_steps"]
    vox = sum(r.voxel_updates for r in done)
    statuses, failed = {}, []
    for r in results:
        statuses[r.status] = statuses.get(r.status, 0) + 1
        if r.status != "done" and len(failed) < 5:
            _, sp, n = sched[r.request_id]
            failed.append({"request": r.request_id, "status": r.status, "error": (r.error or "")[:160],
                           "agents": sp.n_agents, "capacity": sp.capacity, "grid": sp.field_dims[0], "steps": n})
    out = {"rate_per_s": rate, "duration_s": duration, "requests": len(sched), "status": statuses,
           "storage": storage, "wall_s": wall, "steps_run": pool.steps_run, "ms_per_batch_step": 1e3 * wall / max(1, pool.steps_run),
           "ttc_p50_s": float(np.percentile(ttc, 50)), "ttc_p99_s": float(np.percentile(ttc, 99)),
           "ttc_mean_s": float(ttc.mean()), "ttc_max_s": float(ttc.max()),
           "queue_wait_p99_s": float(np.percentile(wait, 99)),
           "agent_steps_per_s": agent_steps / wall, "voxel_updates_per_s": vox / wall,
           "max_resident": pool.max_resident, "device_status": c1["status"], "not_done": failed,
           "device_busy_s": busy, "device_busy_frac": busy / wall, "depth": depth, "prefetch_s": prefetch,
           "arenas": {k: int(v) for k, v in plan.items()},
           "peak_usage": {k: int(v) for k, v in pool.peak_usage.items()},
           "hbm_fraction": hbm_fraction}
    dev.close()
    del dev, pool, warm
    torch.cuda.empty_cache()
    if solo_sample:
        order = np.argsort([int(np.prod(sp.field_dims)) * (sp.S_o2 + sp.S_drug) + sp.n_agents for sp in specs])
        idx = order[np.linspace(0, len(order) - 1, solo_sample).astype(int)]
        solo_ms, solo_as, served_as_est = 0.0, 0, 0
        solo_each = []
        st = torch.cuda.current_stream()
        for i in idx:
            _, sp, n = sched[i]
            sp32 = replace(sp, storage="f32")
            eng = W.build_engine(sp32)
            eng.set_graphs(True)
            be = eng._backend_impl
            a0 = be.counters()["agent_steps"]
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            eng.run_steps(n)
            e1.record(st)
            torch.cuda.synchronize()
            solo_ms += e0.elapsed_time(e1)
            solo_each.append(e0.elapsed_time(e1) / 1e3)
            solo_as += be.counters()["agent_steps"] - a0
            del eng, be
        out["solo_fp32_sample"] = {"requests": int(solo_sample), "agent_steps_per_s": solo_as / (solo_ms / 1e3),
                                   "served_vs_solo": out["agent_steps_per_s"] / (solo_as / (solo_ms / 1e3)),
                                   "sample": "requests spread over the mix by size, each run alone for its own "
                                             "step count on a solo FP32 engine with CUDA graphs"}
        out["solo_largest_s"] = max(solo_each)
        torch.cuda.empty_cache()
    # the stated latency target of the serving mix (requests of up to 1,000
    # steps arriving at 20/s for 120 s): every pool step advances all residents
    # by one step, so a request's time to completion is about its step count
    # times the pool's step time; 8 s bounds a 1,000-step request at 8 ms per
    # pool step, twice the step time of the mix's peak occupancy
    out["p99_target_s"] = P99_TARGET_S
    out["p99_target_met"] = bool(out["ttc_p99_s"] <= P99_TARGET_S)
    return out


class _SoloAsBatch:
    """A solo Engine behind the two calls measure_batch's timer uses."""

    def __init__(self, eng) -> None:
        self.eng = eng

    def run_steps(self, n: int) -> None:
        self.eng.run_steps(n)

    def counters(self) -> dict:
        return self.eng._backend_impl.counters()


def run_batch_workload(args) -> None:
    import torch

    rank, world, local = env_ranks()
    torch.cuda.set_device(local)
    r = measure_batch(args.sims, args.steps, args.warmup, graphs=not args.no_graphs, solo_sample=args.solo_sample,
                      seed=rank, storage=args.storage, encoding=args.encoding)
    peaks = measured_peaks()
    line = {"metric": METRIC, "value": r["agent_steps_per_s"],
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.storage == "f32" else f"{args.storage} fields, f32 update",
            "data": "synthetic (numpy default_rng, seed 0 + rank)",
            "config": {"workload": f"batched sweep, {args.sims} members", "members": args.sims,
                       "agents": r["agents_start"], "voxels_per_field": r["voxels_per_field"], "fields": "o2+drug",
                       "substeps_o2": r["substeps_o2"], "parallelism": f"replicas x{world}"},
            "voxel_updates_per_s": r["voxel_updates_per_s"], "batch": r, "peak_hbm_gbs": peaks["hbm_gbs"]}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_serving_workload(args) -> None:
    import torch

    rank, world, local = env_ranks()
    torch.cuda.set_device(local)
    r = measure_serving(args.rate, args.duration, seed=rank, storage=args.storage, solo_sample=args.solo_sample)
    line = {"metric": METRIC, "value": r["agent_steps_per_s"], "unit": UNIT, "n_gpus": world, "steps": r["steps_run"],
            "warmup": 1, "ms_per_step": r["ms_per_batch_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if args.storage == "f32" else f"{args.storage} fields, f32 update",
            "data": "synthetic (numpy default_rng, seed 0 + rank)",
            "config": {"workload": f"serving mix, Poisson {args.rate}/s for {args.duration} s",
                       "parallelism": f"replicas x{world}"},
            "serving": r}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_stencil_workload(args) -> None:
    """The diffusion kernels alone on one G^3 field (--grid): FP32 one or two
    substeps per pass (--stencil-pair CTA sizes) and the 16-bit storages with
    each element encoding (--encodings), through the tuned stage entries
    (olc_stage_diffuse_tuned, olc_stage_diffuse16).  Device time per substep
    over --steps calls of 40 substeps after --warmup, CUDA events."""
    import ctypes as C

    import torch

    rank, world, local = env_ranks()
    torch.cuda.set_device(local)
    from oncolytica_b200 import _lib
    from oncolytica_b200._fieldcodec import ENCODINGS

    olc = _lib.load()
    n, S, dx, D = args.grid, 40, 4.0, 2000.0
    dt = 0.15 * dx * dx * S / D  # D dt / (S dx^2) = 0.15
    dims = (C.c_int32 * 3)(n, n, n)
    dev = torch.device("cuda", local)
    st = torch.cuda.current_stream(dev)
    gen = torch.Generator(device=dev).manual_seed(rank)
    f32 = torch.rand(n ** 3, device=dev, generator=gen) * 0.8 + 0.1

    def timed(fn) -> float:
        for _ in range(max(1, args.warmup)):
            fn()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(args.steps):
            fn()
        e1.record(st)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) * 1e3 / (args.steps * S)

    out = {}
    spec = _lib.OlcDiffusion(diffusion=D, decay=0.0, boundary=1.0, substeps=S, has_sink=0)
    f, tmp = f32.clone(), torch.empty_like(f32)
    for nt in (int(v) for v in args.stencil_pair.split(",") if v and v != "none"):
        t = _lib.OlcTuning(8, 8, 0, 16, nt, 0, 0)
        out[f"f32_pair{nt}" if nt else "f32_single"] = timed(lambda: _lib.check(olc.olc_stage_diffuse_tuned(
            f.data_ptr(), tmp.data_ptr(), None, C.byref(dims), dx, dt, C.byref(spec), C.byref(t), None)))
    for keep in (int(v) for v in args.l2_keep.split(",") if v and v != "none"):
        t = _lib.OlcTuning(8, 8, 0, 16, 0, 0, keep)
        out[f"f32_single_l2keep{keep}"] = timed(lambda: _lib.check(olc.olc_stage_diffuse_tuned(
            f.data_ptr(), tmp.data_ptr(), None, C.byref(dims), dx, dt, C.byref(spec), C.byref(t), None)))
    for storage in (3, 4):
        for name in (e for e in args.encodings.split(",") if e and e != "none"):
            code = ENCODINGS[name]
            h = f32.to(torch.bfloat16 if storage == 3 else torch.float16).view(torch.int16)
            if code == 2:
                h = h & 0x3FFF  # flag bits 00: the magnitude is the value
            tmp16, comp = torch.empty_like(h), torch.zeros(n ** 3, dtype=torch.float32, device=dev)
            sp = _lib.OlcDiffusion(diffusion=D, decay=0.0, boundary=1.0, substeps=S, has_sink=0, storage=storage,
                                   encoding=code)
            out[f"{'bf16' if storage == 3 else 'f16'}_sr_{name}"] = timed(lambda: _lib.check(olc.olc_stage_diffuse16(
                h.data_ptr(), tmp16.data_ptr(), None, comp.data_ptr(), C.byref(dims), dx, dt, C.byref(sp), 7, 0,
                None)))
    line = {"metric": "us per substep (one field)", "value": out.get("f32_single"), "unit": "us",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "f32 / 16-bit fields", "data": "synthetic (torch uniform, seed = rank)",
            "config": {"workload": f"diffusion kernels on one {n}^3 field, {S} substeps per call"},
            "us_per_substep": out}
    if rank == 0:
        print(json.dumps(line), flush=True)


def main() -> None:
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "stencil":
        run_stencil_workload(args)
    elif args.workload == "batch":
        run_batch_workload(args)
    elif args.workload == "serve":
        run_serving_workload(args)
    elif args.workload == "precision":
        run_precision_workload(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
