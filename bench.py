#!/usr/bin/env python
"""Benchmark of the per-tick simulation loop on B200.

Workload: the large plain network -- 100,000 neurons x 64 segments (6.4M segments),
16 modifiers per segment drawn from 24 channel/receptor/pump types, Cav2.1 on axon
segments, 10M chemical synapses with 8 receptors each, dt = 0.025 ms -- generated
from a seed (synthetic data; no dataset exists for this path).  A step is one tick.

    python bench.py [--gpus N --steps K --warmup W]          # this backend
    python bench.py --impl reference [--steps K --warmup W]  # reference CPU tick

value       segment-ticks/s of the whole job, device-timed with CUDA events on the
            backend's stream around exactly K ticks (max over ranks for N > 1;
            each rank runs its own network, weak scaling, no collective).
e2e         the same metric through bnc_step_io: per tick, an H2D copy of the
            stimulus amplitudes from pinned memory and a D2H copy of every
            segment's V_m into pinned memory, wall clock around K steps.
roofline    the dominant kernel's algorithmic bytes per launch over its average
            CUDA-event duration, against the measured copy bandwidth.
cpu_baseline the reference's own CPU tick (oracle/_ref, built from the reference
            sources) on a bounded sample of the same workload, 1 core.
draw_order  the same network with each segment's modifiers kept in the order the
            seeded draw produced them instead of listed by type ID (the default):
            another slot order, so other physics from the same distribution.
"""
import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DT = 0.025
WORKLOAD = ("large plain network: 100000 neurons x 64 segments (6.4M segments), 16 modifiers/segment "
            "from 24 types, 10M synapses x 8 receptors, dt 0.025 ms")
METRIC = "segment-ticks/s (plain 6.4M-segment network)"
UNIT = "segment-ticks/s"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--neurons", type=int, default=100000)
    ap.add_argument("--seed", type=int, default=20260)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=100)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ens-members", type=int, default=512)
    ap.add_argument("--ens-ticks", type=int, default=4000)
    ap.add_argument("--ens-seq-ticks", type=int, default=64)
    ap.add_argument("--no-trees", action="store_true")
    ap.add_argument("--trees", type=int, default=16384)
    ap.add_argument("--tree-ticks", type=int, default=20)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-dropin", action="store_true")
    ap.add_argument("--no-draw-order", action="store_true")
    ap.add_argument("--draw-ticks", type=int, default=50)
    ap.add_argument("--dropin-neurons", type=int, default=10000)
    ap.add_argument("--dropin-ticks", type=int, default=10)
    ap.add_argument("--sweep-tasks", type=int, default=256)
    ap.add_argument("--sweep-ticks", type=int, default=1000)
    ap.add_argument("--adj-neurons", type=int, default=256)
    ap.add_argument("--adj-sets", type=int, default=64)
    ap.add_argument("--adj-ticks", type=int, default=1024)
    ap.add_argument("--adj-fitting-only", action="store_true", help="skip the whole-small-set adjoint run")
    return ap.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def rank_seed(seed, rank):
    """Each rank simulates its own network (replicas, weak scaling): seed + rank."""
    return seed + rank


def max_over_ranks(value, dist, device):
    """Max of a float over all ranks; every rank must call it (one all-reduce)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([value], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def rank_barrier(dist, device):
    """Barrier as an all-reduce on the backend's device, then a device synchronize."""
    if dist is None:
        return
    import torch
    t = torch.zeros(1, device=device)
    dist.all_reduce(t)
    if device != "cpu":
        torch.cuda.synchronize()


class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="bnc_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.out = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.out, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        sms, maxes, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                p = [x.strip() for x in line.split(",")]
                if len(p) < 9:
                    continue
                try:
                    sms.append(float(p[1]))
                    maxes.append(float(p[2]))
                    power.append(float(p[3]))
                except ValueError:
                    continue
                for n, v in zip(names, p[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": max(maxes) if maxes else None,
                "reasons": sorted(reasons), "samples": len(sms),
                "power_w_max": max(power) if power else None}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_figure(kernel, key):
    """A per-launch figure (`key: value` line) recorded in the committed ncu summary of
    `kernel`, scaled to the full network, if any."""
    path = os.path.join(ROOT, "profiles", "%s_large_network.md" % kernel)
    try:
        with open(path) as f:
            m = re.search(r"%s:\s*([0-9.eE+]+)" % key, f.read())
            return float(m.group(1)) if m else None
    except OSError:
        return None


def ncu_traffic(kernel):
    """DRAM bytes per launch recorded in the committed ncu summary of `kernel`, if any."""
    return ncu_figure(kernel, "dram_bytes_per_launch_full_size")


def issue_roofline(kernels, sm_mhz, n_gpus_neurons_scale=1.0):
    """The bound these kernels hit: instruction issue.  Warp instructions per launch
    (ncu, committed summaries, scaled to the full network) over the CUDA-event time,
    against the issue peak of the GPU at the SM clock sampled in the timed region (one
    warp instruction per cycle per scheduler, four schedulers per SM)."""
    try:
        import torch
        sms = torch.cuda.get_device_properties(0).multi_processor_count
    except Exception:
        return None
    if not sm_mhz:
        return None
    peak = sms * 4 * sm_mhz * 1e6
    out = {"unit": "warp instructions/s", "peak": peak, "sms": sms, "sm_mhz": sm_mhz,
           "peak_source": "4 schedulers x SMs x median SM clock in the timed region", "kernels": {}}
    for k, ms in kernels.items():
        w = ncu_figure(k, "warp_instructions_per_launch_full_size")
        if w is None or not ms:
            continue
        w *= n_gpus_neurons_scale
        out["kernels"][k] = {"warp_instructions": w, "achieved": w / (ms / 1000.0), "frac": w / (ms / 1000.0) / peak}
    return out


def cpu_reference_rate(neurons, ticks, warm, seed):
    """Reference CPU tick (or the oracle port when the reference build is absent) on a
    generated network; returns (segment-ticks/s, kind, segments)."""
    import ctypes as C
    from bioneuroncore_b200 import Network, NetgenParams, NET_LARGE
    from oracle import oracle as orc
    net = Network(NetgenParams(family=NET_LARGE, n_neurons=neurons, seed=seed))
    nseg = net.data.num_segments
    if orc.reference_available():
        runner, kind = orc.Reference(net), "reference"
    else:
        runner, kind = orc.Oracle(net), "port"
    runner.run(warm, DT)
    t0 = time.perf_counter()
    runner.run(ticks, DT)
    dt = time.perf_counter() - t0
    return nseg * ticks / dt, kind, nseg


def cpu_reference_params(params, ticks, warm):
    """The reference CPU tick (oracle port when the reference build is absent) run
    network by network over `params` (NetgenParams); returns (segment-ticks/s, seconds
    of timed ticks, segments, kind).  Networks are built before the clock starts."""
    from bioneuroncore_b200 import Network
    from oracle import oracle as orc
    total_s, seg_ticks, nseg, kind = 0.0, 0.0, 0, "port"
    for p in params:
        net = Network(p)
        if orc.reference_available():
            runner, kind = orc.Reference(net), "reference"
        else:
            runner, kind = orc.Oracle(net), "port"
        runner.run(warm, DT)
        t0 = time.perf_counter()
        runner.run(ticks, DT)
        total_s += time.perf_counter() - t0
        seg_ticks += float(net.data.num_segments) * ticks
        nseg += net.data.num_segments
    return seg_ticks / total_s, total_s, nseg, kind


def _ref_params_worker(args):
    params, ticks, warm = args
    return cpu_reference_params(params, ticks, warm)


def cpu_reference_parallel(params, ticks, warm, procs):
    """cpu_reference_params with the networks dealt round-robin to `procs` processes
    (spawned: the reference tick is single-threaded and not re-entrant); returns the
    aggregate segment-ticks/s over the wall clock of the timed ticks (max over
    processes) and the process count."""
    import multiprocessing as mp
    procs = max(1, min(procs, len(params)))
    chunks = [params[k::procs] for k in range(procs)]
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_ref_params_worker, [(c, ticks, warm) for c in chunks])
    seg_ticks = sum(r[0] * r[1] for r in res)
    return seg_ticks / max(r[1] for r in res), procs


class _RefBionData:
    """The reference's BionData (include/bion_loader.h:16-28) for its own loader, defined
    here so that the reference arm imports nothing of this backend."""
    @staticmethod
    def make():
        import ctypes as C

        class BionData(C.Structure):
            _fields_ = [("header", C.c_uint8 * 100), ("neurons", C.c_void_p), ("segments", C.c_void_p),
                        ("connections", C.c_void_p), ("synapses", C.c_void_p), ("nuclei", C.c_void_p),
                        ("num_neurons", C.c_uint32), ("num_segments", C.c_uint32),
                        ("num_connections", C.c_uint32), ("num_synapses", C.c_uint32), ("num_nuclei", C.c_uint32)]
        return BionData()


def write_reference_samples(out_dir, neurons, seeds):
    """Child process of the reference arm: generates the sample networks with this
    backend's seeded generator and writes each as a .bion with the reference's own
    bion_save, plus its current steps (CurrentStimulus records) beside it."""
    import ctypes as C
    from bioneuroncore_b200 import Network, NetgenParams, NET_LARGE
    from oracle import oracle as orc
    ref = orc.reference_lib()
    save = getattr(ref, "_Z9bion_savePKcPK8BionData")
    save.argtypes = [C.c_char_p, C.c_void_p]
    save.restype = C.c_int
    for sd in seeds:
        net = Network(NetgenParams(family=NET_LARGE, n_neurons=neurons, seed=sd))
        path = os.path.join(out_dir, "sample_%d.bion" % sd)
        if save(path.encode(), C.byref(net.data)) != 0:
            raise RuntimeError("bion_save failed for %s" % path)
        with open(path + ".stim", "wb") as f:
            f.write(net.stimuli.tobytes())
        net.close()


def _ref_bion_worker(args):
    """One reference-arm process: the reference's bion_load_host reads a sample .bion,
    then its core_run_tick runs warm-up and timed ticks on it.  Returns (segment-ticks/s,
    segments, whether this backend's library is mapped in the process)."""
    path, ticks, warm = args
    import ctypes as C
    from oracle import oracle as orc
    ref = orc.reference_lib()
    load = getattr(ref, "_Z14bion_load_hostPKcP8BionData")
    load.argtypes = [C.c_char_p, C.c_void_p]
    load.restype = C.c_int
    d = _RefBionData.make()
    if load(path.encode(), C.byref(d)) != 0:
        raise RuntimeError("bion_load_host failed for %s" % path)
    raw = open(path + ".stim", "rb").read()
    stim = (C.c_uint8 * max(len(raw), 1)).from_buffer_copy(raw or b"\0")
    n_stim = C.c_uint32(len(raw) // 20)
    tick = C.c_uint64(0)

    def run(n):
        for _ in range(n):
            ref.core_run_tick(d.segments, d.num_segments, d.connections, d.num_connections, d.synapses,
                              d.num_synapses, 0, C.byref(tick), C.c_float(DT), C.addressof(stim), C.byref(n_stim),
                              *([None] * 10))
    run(warm)
    t0 = time.perf_counter()
    run(ticks)
    el = time.perf_counter() - t0
    with open("/proc/self/maps") as f:
        mapped = any("libbnc_b200" in line for line in f)
    return d.num_segments * ticks / el, d.num_segments, mapped


def workload_config(neurons):
    """The workload as both arms name it (the large plain network at `neurons`)."""
    return {"workload": WORKLOAD if neurons == 100000 else WORKLOAD.replace("100000 neurons", "%d neurons" % neurons),
            "segments_per_gpu": neurons * 64, "synapses_per_gpu": neurons * 100, "dt_ms": DT}


def run_reference_arm(a):
    """The reference's own CPU tick (oracle/_ref, compiled from the reference's sources)
    on the workload, one process per host core: the tick is single-threaded and not
    re-entrant (function-local statics, diffusion_kernel.h:50,124-128).  Each process
    runs a bounded sample of the workload (128 neurons x 64 segments of the same
    generator, its own seed) read from a .bion by the reference's loader; the samples
    are written beforehand by a separate process, so no process of this arm maps this
    backend's library."""
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    import multiprocessing as mp
    import shutil
    ncores = os.cpu_count() or 1
    neurons = 128   # 8192 segments, 12,800 synapses per process and step
    tmp = tempfile.mkdtemp(prefix="bnc_ref_samples_")
    try:
        seeds = [a.seed + i for i in range(ncores)]
        subprocess.run([sys.executable, os.path.abspath(__file__), "--write-reference-samples", tmp, str(neurons)]
                       + [str(x) for x in seeds], check=True)
        paths = [os.path.join(tmp, "sample_%d.bion" % sd) for sd in seeds]
        t0 = time.perf_counter()
        with mp.get_context("spawn").Pool(ncores) as pool:
            res = pool.map(_ref_bion_worker, [(p, a.steps, a.warmup) for p in paths])
        wall = time.perf_counter() - t0
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    value = sum(r[0] for r in res)
    seg = res[0][1]
    sample = ("%d processes, each the reference's tick on its own %d-neuron x 64-segment sample of the generator "
              "(%d segments, %d synapses x 8 receptors) read by its bion_load_host; %d ticks after %d warm-up"
              % (ncores, neurons, seg, neurons * 100, a.steps, a.warmup))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": 1000.0 * seg * ncores / value if value else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(a.neurons),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "this_backend_mapped_in_reference_processes": any(r[2] for r in res),
        "wall_s": wall,
    }
    print(json.dumps(line), flush=True)
    return 0


def run_draw_order(a, device):
    """The headline network with each segment's 16 large-set modifiers kept in the order
    the seeded categorical draw produced them (BNC_NETGEN_DRAW_ORDER), instead of
    listed by type ID.  The slot order is the order the tick applies them in, so this
    is different physics of the same distribution, and the phase groups' warps see less
    uniform model sequences.  Device-timed with CUDA events over a.draw_ticks ticks."""
    from bioneuroncore_b200 import Backend, NetgenParams, NET_LARGE, NETGEN_DRAW_ORDER
    b = Backend(device)
    try:
        t0 = time.perf_counter()
        b.load_generated(NetgenParams(family=NET_LARGE, n_neurons=a.neurons, seed=a.seed, flags=NETGEN_DRAW_ORDER))
        setup = time.perf_counter() - t0
        info = b.info()
        b.run_ticks(a.warmup, DT)
        n_prof = 5
        ms_mod, ms_diff, ms_syn = b.profile_ticks(n_prof, DT)
        ms = b.time_ticks(a.draw_ticks, DT)
        return {"workload": workload_config(a.neurons)["workload"] + ", modifiers in draw order",
                "metric": UNIT, "ticks": a.draw_ticks, "value": float(info.n_segments) * a.draw_ticks / (ms / 1000.0),
                "ms_per_tick": ms / a.draw_ticks, "phases": info.n_phases,
                "kernels_ms": {"k_modifiers": ms_mod / n_prof, "k_diffusion": ms_diff / n_prof,
                               "k_synapse": ms_syn / n_prof},
                "setup_s": round(setup, 1)}
    finally:
        b.close()


def run_ensemble(a, device, dist=None):
    """Batched ensemble: a.ens_members independent networks of uneven size (segments
    log-uniform in [200, 20000], gNa/gK/gleak/gCa x U[0.5, 2], one seed each) in one
    device structure -- grouping autotuned on a sample, tick loop captured in a CUDA
    graph -- against the same networks run one after another with plain launches.
    The ensemble runs its a.ens_ticks ticks (4,000 by default) as one launch of the
    captured loop; the sequential leg runs a.ens_seq_ticks ticks per network.  Both are
    device-timed with CUDA events after warm-up and compared per tick."""
    from bioneuroncore_b200 import Backend, ensemble_params
    from bioneuroncore_b200.shard import deal_members, member_segments
    ps_all = list(ensemble_params(a.seed, a.ens_members, 200, 20000))
    world = dist.get_world_size() if dist is not None else 1
    rank = dist.get_rank() if dist is not None else 0
    sizes = member_segments(ps_all)
    deal = deal_members(sizes, world)   # whole members per rank, greedy size balance
    ps = [ps_all[m] for m in deal[rank]]
    total_segments = sum(sizes)
    ens = Backend(device)
    t0 = time.perf_counter()
    tune = ens.load_ensemble_tuned(ps, 32, DT)
    setup_s = time.perf_counter() - t0
    info = ens.info()
    ens.run_ticks_graph(max(a.warmup, 3), DT)
    ms_ens = max_over_ranks(ens.time_ticks_graph(a.ens_ticks, DT), dist, "cuda")
    ens.close()
    ms_seq = 0.0
    seq_segments = 0
    for p in ps:
        b = Backend(device)
        b.load_generated(p)
        b.run_ticks(max(a.warmup, 3), DT)
        ms_seq += b.time_ticks(a.ens_seq_ticks, DT)
        seq_segments += b.info().n_segments
        b.close()
    assert seq_segments == info.n_segments
    ms_seq = max_over_ranks(ms_seq, dist, "cuda")
    cpu = None
    if not a.no_cpu_baseline and world == 1:
        try:   # a seeded sample of the members, then all 8 host cores on it
            sample = ps[:: max(1, len(ps) // 32)][:32]
            rate1, secs, nseg_s, kind = cpu_reference_params(sample, 2, 1)
            rate8, procs = cpu_reference_parallel(sample, 2, 1, os.cpu_count() or 1)
            cpu = {"value": rate1, "unit": "segment-ticks/s", "cores": 1, "kind": kind,
                   "parallel_value": rate8, "parallel_processes": procs,
                   "sample": "%d of the %d networks (%d segments), 2 ticks after 1 warm-up each" %
                             (len(sample), len(ps), nseg_s),
                   "sequential_512_ms_per_tick_extrapolated": 1000.0 * info.n_segments / rate1}
        except Exception as exc:
            cpu = {"unavailable": str(exc)[:200]}
    rate_ens = total_segments * a.ens_ticks / (ms_ens / 1000.0)
    rate_seq = total_segments * a.ens_seq_ticks / (ms_seq / 1000.0)
    return {
        "workload": "%d networks, 200-20000 segments each (log-uniform), %d segments in total, conductances "
                    "x U[0.5, 2], own seeds" % (a.ens_members, total_segments),
        "ranks": world, "members_per_rank": [len(x) for x in deal],
        "segments_per_rank": [sum(sizes[m] for m in x) for x in deal],
        "metric": "segment-ticks/s", "ticks": a.ens_ticks, "value": rate_ens, "ms_per_tick": ms_ens / a.ens_ticks,
        "sequential_value": rate_seq, "sequential_ms_per_tick": ms_seq / a.ens_seq_ticks,
        "sequential_ticks": a.ens_seq_ticks,
        "speedup_vs_sequential": rate_ens / rate_seq,
        "launch": "one structure; all ticks of the call as one CUDA graph launch (a conditional while node "
                  "around one captured tick)",
        "sequential_launch": "each network alone, plain launches (gather, one per modifier phase, diffusion, synapse: phases + 3 per tick), device time summed",
        "grouping": {"warp_cap": tune.warp_cap, "tile_segs": tune.tile_segs,
                     "candidates_tried": tune.candidates_tried, "sample_members": tune.sample_members},
        "setup_s": round(setup_s, 1),
        "cpu_reference": cpu,
    }


def run_trees(a, device):
    """Electrodiffusion-heavy workload: a.trees seeded binary dendritic trees of depth 10
    (2,047 segments each; 16,384 trees = 33.5M segments), initial ions perturbed +-5%,
    Nernst-Planck for 7 ions with the reference's fixed 50-sweep Jacobi solves.  Each
    tree spans a 2-CTA cluster.  Device-timed with CUDA events over a.tree_ticks ticks."""
    from bioneuroncore_b200 import Backend, NetgenParams, NET_TREES, NETGEN_PERTURB_IONS
    b = Backend(device)
    t0 = time.perf_counter()
    b.load_generated(NetgenParams(family=NET_TREES, n_neurons=a.trees, tree_depth=10, seed=a.seed,
                                  flags=NETGEN_PERTURB_IONS))
    setup_s = time.perf_counter() - t0
    info = b.info()
    b.run_ticks(max(a.warmup, 3), DT)
    n_prof = 3
    ms_mod, ms_diff, ms_syn = b.profile_ticks(n_prof, DT)
    ms_fixed = b.time_ticks(a.tree_ticks, DT)
    # the workload's own solver: Jacobi to a residual of 1e-6 with FP64 iterates and
    # the per-ion FP64 ledger (bnc_set_diffusion_mode), on the same network
    from bioneuroncore_b200 import DIFFUSION_RESIDUAL, DIFFUSION_LEDGER
    b.set_diffusion_mode(DIFFUSION_RESIDUAL | DIFFUSION_LEDGER, 1e-6, 100000)
    b.run_ticks(1, DT)
    b.diffusion_stats(reset=True)
    ms = b.time_ticks(a.tree_ticks, DT)
    dst = b.diffusion_stats()
    b.close()
    cpu = None
    if not a.no_cpu_baseline:
        try:   # a seeded subset of the trees, per-segment throughput
            n_sub = 16
            rate, secs, nseg_s, kind = cpu_reference_params(
                [NetgenParams(family=NET_TREES, n_neurons=n_sub, tree_depth=10, seed=a.seed, flags=NETGEN_PERTURB_IONS)],
                2, 1)
            cpu = {"value": rate, "unit": "segment-ticks/s", "cores": 1, "kind": kind,
                   "sample": "%d trees (%d segments), 2 ticks after 1 warm-up" % (n_sub, nseg_s)}
        except Exception as exc:
            cpu = {"unavailable": str(exc)[:200]}
    return {
        "workload": "%d binary dendritic trees of depth 10 (%d segments), ions perturbed +-5%%, Jacobi solves to "
                    "a residual of 1e-6 in FP64, FP64 per-ion ledger" % (a.trees, info.n_segments),
        "metric": "segment-ticks/s", "ticks": a.tree_ticks, "value": info.n_segments * a.tree_ticks / (ms / 1000.0),
        "ms_per_tick": ms / a.tree_ticks,
        "solver": {"max_sweeps_v": dst.max_sweeps_v, "max_sweeps_phi": dst.max_sweeps_phi,
                   "capped_group_solves": dst.capped_v + dst.capped_phi,
                   "ledger_rounding_abs_sum": float(sum(abs(x) for x in dst.rounding))},
        "fixed_50_sweeps": {"value": info.n_segments * a.tree_ticks / (ms_fixed / 1000.0),
                            "ms_per_tick": ms_fixed / a.tree_ticks,
                            "note": "the reference's fixed 50 sweeps per solve (parity mode)"},
        "kernels_ms": {"k_modifiers": ms_mod / n_prof, "k_diffusion": ms_diff / n_prof, "k_synapse": ms_syn / n_prof},
        "cluster": "2 CTAs per tree (distributed shared memory)", "setup_s": round(setup_s, 1),
        "cpu_reference": cpu,
    }


def run_adjoint_full_small_set(a, device, rng):
    """The adjoint workload with the whole small set (Cav1.3 and the Na/K pump on every
    segment, the pump's ATP diffusing): its cost ratio, beside the fitting family's."""
    import numpy as np
    from bioneuroncore_b200 import Adjoint, Backend, Network, NetgenParams, NET_ADJOINT, NETGEN_FULL_SMALL_SET
    netf = Network(NetgenParams(family=NET_ADJOINT, n_neurons=a.adj_neurons, seed=a.seed, flags=NETGEN_FULL_SMALL_SET))
    bf = Backend(device)
    bf.load_network(netf)
    adjf = Adjoint(bf, a.adj_sets, a.adj_ticks, DT, checkpoint_every=256)
    adjf.record()
    basef = adjf.get_params(0)
    adjf.set_params(0, *[x * f for x, f in zip(basef, (1.15, 0.85, 1.25, 0.8))])
    _, trf = adjf.forward(trace=True)
    adjf.set_target(trf[0])
    for p in range(a.adj_sets):
        adjf.set_params(p, *[(x * np.exp(0.1 * rng.standard_normal(x.shape))).astype(np.float32) for x in basef])
    adjf.forward()
    adjf.backward()
    ffwd, fbwd = adjf.timings()
    adjf.close()
    bf.close()
    return {"forward_ms": ffwd, "backward_ms": fbwd, "backward_over_forward": fbwd / ffwd,
            "note": "the same workload with Cav1.3 and the Na/K pump on every segment (BNC_NETGEN_FULL_SMALL_SET)"}


def run_adjoint(a, device):
    """Adjoint fitting workload: a.adj_neurons neurons x 64 segments with 2,000 synapses
    per 256 neurons (the fitting family: Nav, Kv_DR, K2P leak, AMPA/GABA-A; also timed
    with Cav1.3 and the Na/K pump added), a.adj_sets
    parameter sets in one launch, checkpoints every 256 ticks.  Targets come from a
    hidden parameter set; the forward and backward passes are device-timed (CUDA events
    inside the library) and their ratio is the adjoint's cost in forward passes."""
    import numpy as np
    from bioneuroncore_b200 import Adjoint, Backend, Network, NetgenParams, NET_ADJOINT
    t0 = time.perf_counter()
    net = Network(NetgenParams(family=NET_ADJOINT, n_neurons=a.adj_neurons, seed=a.seed))
    b = Backend(device)
    b.load_network(net)
    adj = Adjoint(b, a.adj_sets, a.adj_ticks, DT, checkpoint_every=256)
    adj.record()
    i = adj.info
    base = adj.get_params(0)
    hidden = [x * f for x, f in zip(base, (1.15, 0.85, 1.25, 0.8))]
    adj.set_params(0, *hidden)
    _, tr = adj.forward(trace=True)
    adj.set_target(tr[0])
    rng = np.random.default_rng(a.seed)
    for p in range(a.adj_sets):   # parameter sets spread around the network's densities
        adj.set_params(p, *[(x * np.exp(0.1 * rng.standard_normal(x.shape))).astype(np.float32) for x in base])
    setup_s = time.perf_counter() - t0
    loss, _ = adj.forward()       # the kernels are warm from the target pass
    g = adj.backward()
    fwd_ms, bwd_ms = adj.timings()
    seg_ticks = float(i.n_segments) * a.adj_sets * a.adj_ticks
    adj.close()
    b.close()
    spec_ticks = 20000
    full = None
    if not a.adj_fitting_only:
        full = run_adjoint_full_small_set(a, device, rng)
    cpu = None
    if not a.no_cpu_baseline:
        try:   # the reference's CPU tick on the same network: the forward pass of one set
            n_cpu = 20
            rate, secs, nseg_s, kind = cpu_reference_params(
                [NetgenParams(family=NET_ADJOINT, n_neurons=a.adj_neurons, seed=a.seed)], n_cpu, 1)
            per_tick = secs / n_cpu
            cpu = {"forward_s_all_sets": per_tick * a.adj_ticks * a.adj_sets, "cores": 1, "kind": kind,
                   "forward_over_gpu_forward": per_tick * a.adj_ticks * a.adj_sets / (fwd_ms / 1000.0),
                   "sample": "%d ticks of one set (%d segments), scaled to %d ticks x %d sets" %
                             (n_cpu, nseg_s, a.adj_ticks, a.adj_sets)}
        except Exception as exc:
            cpu = {"unavailable": str(exc)[:200]}
    return {
        "workload": "%d neurons x 64 segments (%d segments), %d synapses, %d parameter sets, %d ticks, "
                    "checkpoints every 256 ticks; loss = MSE of somatic V_m against a hidden parameter set"
                    % (a.adj_neurons, i.n_segments, i.n_synapses, a.adj_sets, a.adj_ticks),
        "forward_ms": fwd_ms, "backward_ms": bwd_ms, "backward_over_forward": bwd_ms / fwd_ms,
        "forward_segment_ticks_per_s": seg_ticks / (fwd_ms / 1000.0),
        "gradient_segment_ticks_per_s": seg_ticks / ((fwd_ms + bwd_ms) / 1000.0),
        "loss_mean": float(np.mean(loss)), "grad_abs_sum_gleak": float(np.abs(g[2]).sum()),
        "extrapolated_20000_ticks_s": {"forward": fwd_ms / 1000.0 * spec_ticks / a.adj_ticks,
                                       "backward": bwd_ms / 1000.0 * spec_ticks / a.adj_ticks,
                                       "note": "linear in ticks; the timed run is %d ticks" % a.adj_ticks},
        "memory_bytes": {"checkpoints": i.checkpoint_bytes, "window": i.window_bytes, "scratch": i.scratch_bytes},
        "launch": "one CTA per (neuron, parameter set); forward %d threads, %d B shared; backward %d B shared"
                  % (i.threads, i.smem_forward, i.smem_backward),
        "setup_s": round(setup_s, 1),
        "full_small_set": full,
        "cpu_reference": cpu,
    }


def run_dropin(a, device):
    """The reference-facing drop-in call: gpu_backend_run_tick on a network loaded from
    host Segment/Synapse records (bnc_load_aos).  After every tick the call leaves those
    records coherent with the device state: as in the reference's backend, the records
    live in managed memory and a device kernel writes the tick's changing words into
    them, so a host read migrates only what it touches.  Timed two ways by the host
    wall clock: the calls alone, and each call followed by a host read of every
    record's V_m (every record's page comes to the host and goes back to the device
    at the next tick).  Then the same two with the records in plain host memory
    (bnc_set_records_residency(1)): the changing state is copied to the host and
    scattered into them after each tick, so reads cost nothing more.  Beside them the
    device-only tick of the same network."""
    import numpy as np
    from bioneuroncore_b200 import Backend, Network, NetgenParams, NET_LARGE
    from bioneuroncore_b200.abi import view, SEGMENT_DTYPE
    net = Network(NetgenParams(family=NET_LARGE, n_neurons=a.dropin_neurons, seed=a.seed))
    b = Backend(device)
    b.load_network(net)
    b.run_tick(DT)
    d = b.bion_data()
    seg = view(d.segments, SEGMENT_DTYPE, d.num_segments)
    t0 = time.perf_counter()
    for _ in range(a.dropin_ticks):
        b.run_tick(DT)
    el = time.perf_counter() - t0
    acc = 0.0
    t0 = time.perf_counter()
    for _ in range(a.dropin_ticks):
        b.run_tick(DT)
        acc += float(seg["V_m"].sum())
    el_read = time.perf_counter() - t0
    coherent = bool(np.array_equal(seg["V_m"].astype(np.float32), np.asarray(b.segment_field("V"), np.float32)))
    managed = bool(b.lib.bnc_records_managed(b.h))
    host_res = None
    if managed and b.lib.bnc_set_records_residency(b.h, 1) == 0:
        d = b.bion_data()                       # the records moved: a new view
        seg = view(d.segments, SEGMENT_DTYPE, d.num_segments)
        b.run_tick(DT)
        t0 = time.perf_counter()
        for _ in range(a.dropin_ticks):
            b.run_tick(DT)
        el_h = time.perf_counter() - t0
        t0 = time.perf_counter()
        for _ in range(a.dropin_ticks):
            b.run_tick(DT)
            acc += float(seg["V_m"].sum())
        el_hr = time.perf_counter() - t0
        host_res = {"ms_per_tick": 1000.0 * el_h / a.dropin_ticks,
                    "ms_per_tick_reading_every_V_m": 1000.0 * el_hr / a.dropin_ticks,
                    "host_view_coherent": bool(np.array_equal(seg["V_m"].astype(np.float32),
                                                              np.asarray(b.segment_field("V"), np.float32)))}
    dev_ms = b.time_ticks(a.dropin_ticks, DT) / a.dropin_ticks
    nseg = net.data.num_segments
    b.close()
    return {"call": "gpu_backend_run_tick (Segment/Synapse records coherent after every tick)",
            "workload": "large plain network at %d neurons (%d segments, %d synapses x 8 receptors)"
                        % (a.dropin_neurons, nseg, net.data.num_synapses),
            "value": nseg * a.dropin_ticks / el, "unit": UNIT, "ms_per_tick": 1000.0 * el / a.dropin_ticks,
            "ms_per_tick_reading_every_V_m": 1000.0 * el_read / a.dropin_ticks,
            "device_ms_per_tick": dev_ms, "ticks": a.dropin_ticks, "host_view_coherent": coherent,
            "records_in_managed_memory": managed, "records_on_host": host_res,
            "timing": "host wall clock around the calls"}


def run_sweep(a, device):
    """Parameter sweep: a.sweep_tasks parameterised runs of one 64-neuron network (2,048
    segments, 400 synapses) as one ensemble (bnc_sweep_run), each task with its own K2P
    conductance and Kv gate overrides and release seed, a.sweep_ticks ticks of 0.1 ms
    with the reference batch mode's tick counter.  Timed end to end by wall clock: host
    network in, per-task metrics out.  The reference runs such tasks one process each;
    its CPU tick is timed on a bounded sample of one task."""
    import numpy as np
    from bioneuroncore_b200 import Backend, Network, NetgenParams, NET_SMALL, sweep_run
    spec = dict(family=NET_SMALL, n_neurons=64, seed=a.seed, stim_pA=3000.0, stim_duration_ms=10.0)
    base = Network(NetgenParams(**spec))
    rng = np.random.default_rng(a.seed)
    tasks = [([(107, float(rng.uniform(50.0, 150.0))), (123, float(rng.uniform(0.0, 0.3)))], int(q + 1))
             for q in range(a.sweep_tasks)]
    b = Backend(device)
    sweep_run(b, base, tasks[:2], 10, 0.1)                    # warm-up: module load, constant tables
    t0 = time.perf_counter()
    res = sweep_run(b, base, tasks, a.sweep_ticks, 0.1)
    wall = time.perf_counter() - t0
    b.close()
    seg_ticks = float(base.data.num_segments) * a.sweep_tasks * a.sweep_ticks
    cpu = None
    try:
        from oracle.oracle import Reference, reference_available
        if reference_available():
            net = Network(NetgenParams(**spec))
            ref = Reference(net)
            n_cpu = 20
            c0 = time.perf_counter()
            ref.run(n_cpu, 0.1, tick_stride=2)
            per_tick = (time.perf_counter() - c0) / n_cpu
            cpu = {"seconds_per_task": per_tick * a.sweep_ticks, "cores": 1,
                   "sweep_seconds_one_process_per_task": per_tick * a.sweep_ticks * a.sweep_tasks,
                   "sample": "%d ticks of one task (reference core_run_tick, FP64 state)" % n_cpu}
    except Exception as exc:
        cpu = {"unavailable": str(exc)[:200]}
    return {
        "workload": "%d tasks x 64 neurons (%d segments each), %d ticks of 0.1 ms, batch-mode tick counter"
                    % (a.sweep_tasks, base.data.num_segments, a.sweep_ticks),
        "seconds": wall, "tasks_per_s": a.sweep_tasks / wall, "segment_ticks_per_s": seg_ticks / wall,
        "timing": "wall clock of bnc_sweep_run: copies, build, tick loop, metrics",
        "spike_count_mean": float(np.mean([r.spike_count for r in res])),
        "spike_count_note": "the reference's metric (core_compute_metrics, simulation_host.cpp:825-880): "
                            "segments above -20 mV at the last tick, a snapshot, not the spikes of the run",
        "cpu_reference": cpu,
    }


def main():
    if len(sys.argv) > 1 and sys.argv[1] == "--write-reference-samples":
        write_reference_samples(sys.argv[2], int(sys.argv[3]), [int(x) for x in sys.argv[4:]])
        return 0
    a = parse_args()
    if a.impl == "reference":
        return run_reference_arm(a)
    rank, local_rank, world = dist_env()
    dist = None
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    from bioneuroncore_b200 import Backend, NetgenParams, NET_LARGE
    b = Backend(local_rank if world > 1 else 0)
    t0 = time.perf_counter()
    b.load_generated(NetgenParams(family=NET_LARGE, n_neurons=a.neurons, seed=rank_seed(a.seed, rank)))
    setup_s = time.perf_counter() - t0
    info = b.info()
    b.run_ticks(a.warmup, DT)
    n_prof = max(3, min(10, a.steps))
    ms_mod, ms_diff, ms_syn = b.profile_ticks(n_prof, DT)

    def barrier():
        rank_barrier(dist, "cuda")

    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ms = b.time_ticks(a.steps, DT)
    clk = clocks.stop()
    barrier()
    ms_max = max_over_ranks(ms, dist, "cuda")
    seg_ticks = float(info.n_segments) * a.steps * world
    value = seg_ticks / (ms_max / 1000.0)

    # end-to-end through the public step call with pinned host buffers
    e2e = None
    if not a.no_e2e:
        import torch
        n_stim = int(info.n_segments // 64 * 0.1 + 0.5)
        amp = torch.full((n_stim,), 200.0, dtype=torch.float32).pin_memory()
        vout = torch.empty(info.n_segments, dtype=torch.float32).pin_memory()
        b.step_io(DT, amp.data_ptr(), n_stim, vout.data_ptr(), info.n_segments)
        barrier()
        t1 = time.perf_counter()
        for _ in range(a.e2e_steps):
            b.step_io(DT, amp.data_ptr(), n_stim, vout.data_ptr(), info.n_segments)
        el = max_over_ranks(time.perf_counter() - t1, dist, "cuda")
        e2e = {"value": float(info.n_segments) * a.e2e_steps * world / el, "unit": UNIT,
               "h2d_bytes_per_step": 4 * n_stim, "d2h_bytes_per_step": 4 * info.n_segments,
               "steps": a.e2e_steps, "timing": "host wall clock around the steps, max over ranks"}

    dropin = None
    if not a.no_dropin and rank == 0 and world == 1:
        dropin = run_dropin(a, local_rank if world > 1 else 0)

    # roofline of the dominant kernel
    peak, peak_kind = measured_peak()
    kernels = {"k_modifiers": (ms_mod / n_prof, info.modifier_kernel_bytes),
               "k_diffusion": (ms_diff / n_prof, info.diffusion_kernel_bytes),
               "k_synapse": (ms_syn / n_prof, info.synapse_kernel_bytes_per_tick)}
    kname = max(kernels, key=lambda k: kernels[k][0])
    kms, kbytes = kernels[kname]
    achieved = kbytes / (kms / 1000.0) / 1e9
    roofline = {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_source": peak_kind, "traffic": ncu_traffic(kname),
                "algo_bytes_per_launch": kbytes, "avg_launch_ms": kms,
                "kernels_ms": {k: v[0] for k, v in kernels.items()},
                "kernels_frac": {k: v[1] / (v[0] / 1000.0) / 1e9 / peak for k, v in kernels.items()},
                "tick_bytes": info.algo_bytes_per_tick,
                "tick_frac": info.algo_bytes_per_tick / (ms_max / a.steps / 1000.0) / 1e9 / peak}
    # the summaries' instruction counts are per launch of the 6.4M-segment network
    roofline["issue"] = issue_roofline({k: v[0] for k, v in kernels.items()}, clk.get("sm_mhz"),
                                       info.n_segments / 6.4e6)

    draw_order = None
    if not a.no_draw_order and rank == 0 and world == 1:
        b.close()   # free the large network's device memory first
        draw_order = run_draw_order(a, 0)

    ensemble = None
    if not a.no_ensemble:
        b.close()
        ensemble = run_ensemble(a, local_rank if world > 1 else 0, dist)

    trees = None
    if not a.no_trees:
        b.close()
        trees = run_trees(a, local_rank if world > 1 else 0)

    sweep = None
    if not a.no_sweep:
        b.close()
        sweep = run_sweep(a, local_rank if world > 1 else 0)

    adjoint = None
    if not a.no_adjoint:
        b.close()
        adjoint = run_adjoint(a, local_rank if world > 1 else 0)

    cpu = None
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        try:
            rate, kind, nseg = cpu_reference_rate(1000, 5, 1, a.seed)
            cpu = {"value": rate, "unit": UNIT, "cores": 1, "kind": kind,
                   "sample": "1000 neurons x 64 segments (%d segments, 100,000 synapses) of the same generator, "
                             "5 ticks after 1 warm-up tick" % nseg}
        except Exception as exc:  # the baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": 1, "kind": "unavailable", "sample": str(exc)[:200]}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 state, f64 GHK/accumulators", "data": "synthetic (seeded generator)",
            "config": workload_config(a.neurons),
            "build": {"parallelism": "replicas" if world > 1 else "single",
                      "l2": "inputs larger than L2 (device state ~8 GB per GPU)", "tiles": info.n_tiles,
                      "phases": info.n_phases, "diffusion_barrier_group": info.group_tiles_64 and 64 or
                      (info.group_tiles_32 and 32 or 0), "setup_s": round(setup_s, 1)},
            "e2e": e2e, "e2e_dropin": dropin, "roofline": roofline, "cpu_baseline": cpu, "clocks": clk,
            "gpu_launches": (info.modifier_launches + 1 + info.synapse_launches) * a.steps, "ensemble": ensemble, "trees": trees,
            "adjoint": adjoint, "sweep": sweep, "draw_order": draw_order,
        }
        print(json.dumps(line), flush=True)
    b.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
