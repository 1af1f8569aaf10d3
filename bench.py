"""Throughput of the DTB per-timestep hot path on B200: synaptic events/s and
simulated-ms per wall-second on the 5M-neuron regional network (200 populations,
in-degree 1000, FP32 weights, OU background, 10,000 steps of 0.1 ms).

Contract (one JSON line on rank 0):
* a bench step = one window of 500 simulation steps (50 ms simulated) of the whole
  network, with per-step population spike counts recorded (RunRequest output_freq);
  --steps 20 is the configuration's full 10,000-step run;
* value = synaptic events delivered / device time, events summed over ranks and
  time = max over ranks of CUDA-event time on the engine's own stream;
* e2e = the same metric through the public C-ABI call (dtb_set_ou + dtb_run) with
  host buffers: each window uploads new per-population OU parameters and reads
  back every step's spike counts and mean potentials;
* roofline = the push kernel (the dominant kernel) against the measured HBM copy
  bandwidth; cpu_baseline = the C port of the reference CPU model on the bounded
  CPU sample (20 x 90 simulated steps of a 50,000-neuron network of the same
  construction);
* batched / served (single GPU, default configuration) = the metric's second half on
  reduced configurations: a 16-member BF16 ensemble batched vs the same members run
  one by one on the plain FP32 path, and a 60-request Poisson stream at 40/s over 32
  resident networks served with continuous batching (BF16) vs one request at a time
  (plain FP32), p50/p99 latency at the same offered rate; each with its own clocks.
N > 1 GPUs run independent replicas (no data-path collective: "scaling": "weak").
--impl reference: the reference arm, the C port of the reference CPU model on the
host cores, W warm-up and K timed bench steps of the CPU sample.

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "synaptic events/s and sim-ms per wall-s; batched/served vs plain p50/p99 at equal rate"
UNIT = "synaptic events/s"
WINDOW = 500
N_NEURONS, N_POPS, IN_DEGREE, SPEC_SEED = 5_000_000, 200, 1000, 1
# the bounded CPU sample: the regional construction at 50,000 neurons (the 5M network needs
# 200-280 GB of host memory as block_new's sparse tensors); one bench step = 75 simulated steps
CPU_SAMPLE = dict(n=50_000, pops=20, in_degree=1000, seed=7, burn_in=400, per_step=90)
CPU_WORKLOAD = ("50,000-neuron regional LIF network, 20 populations, in-degree 1000, f32 weights, OU background "
                "(the 5M-neuron network's construction at a size the host runs)")
BYTES_STATE = 56          # V, J x4, i_ou, t_last read + written per neuron per step
CSR_COL_BYTES = 4
ACC_BYTES = 8             # one logical accumulator update (a float pair) per event
ROW_BYTES = 12            # rowptr pair + spike-list entry per spiking row
PUSH_KINDS = ["reg", "tma", "local"]
# DRAM bytes per delivered synaptic event of the population-local push (measured on local:2008)
# with FP32 weights on the 5M-neuron network: ncu's dram__bytes_read + dram__bytes_write of both
# push kernels over 50 consecutive steps (one burst cycle, 5.0e9 events), caches flushed before
# each launch (profiles/push_traffic_5m_50steps.md)
LOCAL_PUSH_DRAM_BYTES_PER_EVENT_F32 = 14.94
PUSH_KERNELS = ["push_kernel", "push_tma_kernel", "push_kernel (cross-population) + push_local_kernel (windows)"]


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--weights", default="f32", choices=["f32", "bf16"])
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-forms", action="store_true",
                   help="skip the reduced batched and served comparisons of the default line")
    p.add_argument("--neurons", type=int, default=N_NEURONS, help="network size (profiling runs use a small one)")
    p.add_argument("--pops", type=int, default=N_POPS)
    p.add_argument("--degree", type=int, default=IN_DEGREE)
    p.add_argument("--push", default="auto", help="push kernel: auto (autotuned), reg:4|8|16|1016|1008, tma:256|512, local:8|1016")
    p.add_argument("--form", default="plain", choices=["plain", "ensemble", "serve", "precision"],
                   help="plain: the 5M-neuron network; ensemble: 64 DA members batched (BF16) vs sequential (FP32); "
                        "serve: Poisson request stream, continuous batching (BF16) vs one at a time (FP32); "
                        "precision: bf16 + pull vs the FP64 oracle on a 200k-neuron network")
    p.add_argument("--requests", type=int, default=200, help="requests in the served trace (serve form)")
    p.add_argument("--rate", type=float, default=40.0, help="request arrival rate, 1/s (serve form)")
    p.add_argument("--slice", type=int, default=100, help="steps per continuous-batching slice (serve form)")
    p.add_argument("--hbm-cap-gb", type=float, default=150.0, help="HBM cap of the resident networks (serve form)")
    p.add_argument("--members", type=int, default=None, help="ensemble members (64) or served networks (128)")
    p.add_argument("--net", default="regional", choices=["regional", "uniform"],
                   help="regional: the structured regional network; uniform: the plain one-population block")
    p.add_argument("--syn", default="push", choices=["push", "exact", "pull", "fixed"],
                   help="synaptic mode: float push, exact (64-bit fixed-point) push, deterministic pull, or the "
                        "deterministic 32-bit fixed-point push")
    p.add_argument("--window", type=int, default=800, help="steps per assimilation window (ensemble form)")
    p.add_argument("--graph", default="on", choices=["on", "off"], help="replay repeated windows from CUDA graphs")
    p.add_argument("--batched-syn", default="fixed", choices=["fixed", "push"],
                   help="synaptic mode of the batched / served side of the ensemble and serve forms: the "
                        "deterministic fixed-point push (a member equals its solo run) or the float push")
    p.add_argument("--profile-steps", type=int, default=0,
                   help="profiling run: after the warm-up windows, K single-step runs; prints their events and "
                        "spikes per step (no bench line), so an ncu capture of those steps' push launches "
                        "(launches 2 x warm-up steps + 1 .. of a forced local push) can be normalised per event")
    return p.parse_args()


# ---------------------------------------------------------------------------
# CPU: the C port of the reference model on a bounded sample
# ---------------------------------------------------------------------------
def cpu_port_run(timed, warm):
    """The C port of models/block_new.py on the CPU sample (CPU_WORKLOAD): an untimed burn-in
    past the network's quiet start, `warm` untimed bench steps, then `timed` bench steps of
    CPU_SAMPLE["per_step"] simulated steps each, on every host thread."""
    import __graft_entry__
    __graft_entry__.load_package()        # registers the package (network specs only; no CUDA library)
    from dtb_b200 import network as nw
    from oracle import c_oracle as cc
    s = CPU_SAMPLE
    spec = nw.structured_spec(s["n"], s["pops"], s["in_degree"], s["seed"])
    orc = cc.COracle(cc.structured_edges(spec))
    rng = np.random.default_rng(0)
    orc.run(rng.standard_normal((s["burn_in"], spec.n), dtype=np.float32), record=False)
    for _ in range(warm):
        orc.run(rng.standard_normal((s["per_step"], spec.n), dtype=np.float32), record=False)
    events = spikes = 0
    wall = 0.0
    for _ in range(timed):
        z = rng.standard_normal((s["per_step"], spec.n), dtype=np.float32)
        t0 = time.perf_counter()
        _, counts, ev = orc.run(z, record=False)
        wall += time.perf_counter() - t0
        events += ev
        spikes += int(counts.sum())
    threads = cc.lib().oracle_threads()
    sim_steps = timed * s["per_step"]
    sample = (f"C port of models/block_new.py (W.s over all synapses each step, float32), {threads} threads, on "
              f"the {CPU_WORKLOAD}: {sim_steps} simulated steps timed ({timed} x {s['per_step']}) after "
              f"{s['burn_in'] + warm * s['per_step']} untimed; {spikes} spikes, {events} events in {wall:.2f} s. "
              f"models/block_new.py itself (torch.sparse_coo weights) steps this network 1,400x slower than the "
              f"port on the same threads (profiles/cpu_port_vs_block_new_50k.md)")
    return dict(value=events / wall, unit=UNIT, cores=threads, kind="port", sample=sample, wall_s=wall,
                sim_ms_per_wall_s=sim_steps * 0.1 / wall, ms_per_step=1e3 * wall / max(timed, 1), steps=timed)


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 8 and (not self.uuid or parts[0].endswith(self.uuid) or self.uuid.endswith(parts[0])):
                self.rows.append(parts)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        for r in self.rows:
            for name, val in zip(self.NAMES, r[4:8]):
                if val.strip().lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ---------------------------------------------------------------------------
def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_per_launch(events_per_launch, push_kind, f32):
    """DRAM bytes of one push launch: the ncu-measured bytes per event (local push, FP32
    weights, 5M neurons; profiles/push_traffic_5m_50steps.md) times the launch's events; None
    for variants without such a measurement."""
    if push_kind == 2 and f32:
        return LOCAL_PUSH_DRAM_BYTES_PER_EVENT_F32 * events_per_launch
    return None


def aggregate_replicas(counts, times_ms, dist=None, device=None):
    """Whole-job totals of independent replicas: counts summed over ranks, device
    times maxed over ranks (each rank timed its own stream with CUDA events)."""
    import torch
    c = np.asarray(counts, np.float64)
    t = np.asarray(times_ms, np.float64)
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        tc = torch.tensor(c, device=device)
        dist.all_reduce(tc, op=dist.ReduceOp.SUM)
        tt = torch.tensor(t, device=device)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        c, t = tc.cpu().numpy(), tt.cpu().numpy()
    return c, t


def run_ours(args):
    import torch
    import __graft_entry__
    __graft_entry__.load_package()
    from dtb_b200 import engine as E
    from dtb_b200 import network as nw

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.profile_steps and world > 1:
        raise SystemExit("--profile-steps profiles one GPU; run it without torchrun")
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    wt = E.W_BF16 if args.weights == "bf16" else E.W_F32
    syn = {"push": E.SYN_PUSH, "exact": E.SYN_PUSH_EXACT, "pull": E.SYN_PULL, "fixed": E.SYN_PUSH_FIXED}[args.syn]
    t0 = time.perf_counter()
    if args.net == "uniform":
        # the plain block: one population, fixed in-degree, uniform sources (host-built CSR)
        net = nw.make_uniform_block(args.neurons, args.degree, seed=0)
        if wt == E.W_BF16:
            net["weight"] = net["weight"].astype(np.float32)
        eng = E.Engine.from_arrays(net, weight_type=wt, seed=1000 + rank, push=syn != E.SYN_PULL, pull=syn == E.SYN_PULL)
        del net
    else:
        spec = nw.structured_spec(args.neurons, args.pops, args.degree, SPEC_SEED)
        eng = E.Engine.structured(spec, weight_type=wt, seed=1000 + rank, push=syn != E.SYN_PULL, pull=syn == E.SYN_PULL)
    build_s = time.perf_counter() - t0
    if args.push != "auto":
        kind, param = args.push.split(":")
        eng.set_push_variant(PUSH_KINDS.index(kind), int(param))
    eng.set_graph(args.graph == "on")
    info = eng.info()
    stream = torch.cuda.ExternalStream(eng.stream(), device=dev)
    P = eng.n_pops
    fr = np.zeros((WINDOW, P), np.int32)

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        eng.run(WINDOW, freq=True, out=(fr, None), syn_mode=syn)

    if args.profile_steps:
        steps = []
        for _ in range(args.profile_steps):
            r = eng.run(1, freq=True, out=(fr[:1], None), syn_mode=syn)
            steps.append({"events": int(r.events), "spikes": int(fr[0].sum()), "launches": int(r.launches)})
        torch.cuda.synchronize()
        info = eng.info()
        print(json.dumps({"profile_steps": steps, "warm_steps": args.warmup * WINDOW, "neurons": info.n_neurons,
                          "push_variant": f"{PUSH_KINDS[info.push_kind]}:{info.push_param}",
                          "local_windows": info.local_windows, "weights": args.weights}), flush=True)
        eng.close()
        return None

    uuid = str(getattr(torch.cuda.get_device_properties(dev), "uuid", ""))
    sampler = ClockSampler(uuid)
    barrier()
    sampler.start()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    events = 0
    spikes = 0
    launches = 0
    with torch.cuda.stream(stream):
        start.record(stream)
        for _ in range(args.steps):
            r = eng.run(WINDOW, freq=True, out=(fr, None), syn_mode=syn)
            events += r.events
            spikes += int(fr.sum())
            launches += r.launches
        end.record(stream)
    end.synchronize()
    barrier()
    clocks = sampler.stop()
    ms = start.elapsed_time(end)

    info = eng.info()
    tuning = [{"kernel": PUSH_KINDS[k], "param": p, "ms": m} for k, p, m in eng.tuning_report()]
    # per-kernel timing window (after the timed region)
    rk = eng.run(WINDOW, freq=True, out=(fr, None), time_kernels=True, syn_mode=syn)
    lif_ms, push_ms = rk.kernel_ms[0] / WINDOW, rk.kernel_ms[1] / WINDOW
    ev_launch = rk.events / WINDOW
    spk_launch = fr.sum() / WINDOW
    wbytes = 4 if wt == E.W_BF16 else 8
    push_bytes = spk_launch * ROW_BYTES + ev_launch * (CSR_COL_BYTES + wbytes + ACC_BYTES)
    lif_bytes = info.n_neurons * BYTES_STATE + info.n_neurons / 8
    roof_kernel = PUSH_KERNELS[info.push_kind]
    if syn == E.SYN_PULL:
        # algorithmic bytes of the pull: every in-edge (4 + B_w bytes), the bitmap and the neuron
        # state (the kernel itself reads a weight pair only for an edge whose source spiked)
        lif_ms, push_ms = 0.0, rk.kernel_ms[2] / WINDOW
        push_bytes = info.n_edges * (CSR_COL_BYTES + wbytes) + info.n_neurons / 8 + lif_bytes
        lif_bytes = 0.0
        roof_kernel = "lif_pull_kernel (in-degree gather fused with the LIF step)"

    # e2e through the C-ABI with host buffers (H2D of OU parameters, D2H of every step's outputs)
    rng = np.random.default_rng(rank)
    pop_ids = eng.pop_ids
    vm = np.zeros((WINDOW, P), np.float32)
    e2e_events = 0
    barrier()
    e_start, e_end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e_start.record(stream)
        for _ in range(args.steps):
            mean = rng.uniform(0.55, 0.65, P).astype(np.float32)
            sigma = rng.uniform(0.18, 0.22, P).astype(np.float32)
            eng.set_ou(pop_ids, mean, sigma, np.full(P, 10.0, np.float32))
            r = eng.run(WINDOW, freq=True, vmean=True, out=(fr, vm), syn_mode=syn)
            e2e_events += r.events
        e_end.record(stream)
    e_end.synchronize()
    barrier()
    e2e_ms = e_start.elapsed_time(e_end)

    (events, e2e_events, spikes), (ms, e2e_ms) = aggregate_replicas(
        [events, e2e_events, spikes], [ms, e2e_ms], dist, dev)
    value = events / (ms / 1e3)
    out = None
    if rank == 0:
        peak, peak_kind = peaks()
        achieved = push_bytes / (push_ms * 1e-3) / 1e9
        traffic = traffic_per_launch(ev_launch, info.push_kind, wt == E.W_F32) if syn == E.SYN_PUSH else None
        step_bytes = push_bytes + lif_bytes
        cpu = None
        if world == 1 and not args.no_cpu:
            cpu = cpu_port_run(20, 0)
            cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")}
        h2d = P * 96 + P * 3 * 4
        d2h = WINDOW * P * (4 + 8)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if wt == E.W_F32 else "bf16-weights/f32-state",
            "data": ("synthetic (seeded uniform block built on the host)" if args.net == "uniform"
                     else "synthetic (seeded regional network generated on the device)"),
            "sim_ms_per_wall_s": args.steps * WINDOW * 0.1 / (ms / 1e3),
            "config": {"workload": f"{info.n_neurons}-neuron {args.net} LIF network, {P} populations, "
                                   f"in-degree {args.degree}, {args.weights} weights, OU background, "
                                   f"{ {'push': 'push', 'exact': 'exact fixed-point push', 'pull': 'deterministic pull', 'fixed': 'fixed-point push'}[args.syn] } propagation",
                       "neurons": info.n_neurons, "synapses": int(info.n_edges), "populations": P,
                       "dt_ms": 0.1, "steps_per_bench_step": WINDOW,
                       "timed_sim_steps": args.steps * WINDOW, "warmup_sim_steps": args.warmup * WINDOW,
                       "mean_rate_hz": spikes / (world * args.steps * WINDOW) / info.n_neurons * 1e4,
                       "events_per_sim_step": events / (world * args.steps * WINDOW),
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": f"inputs larger than L2 ({info.n_edges * (4 + wbytes) / 1e9:.1f} GB CSR, "
                             f"{info.n_neurons * 56 / 1e6:.0f} MB neuron state)",
                       "device_bytes": int(info.device_bytes), "build_s": build_s,
                       "lif_ms_per_step": lif_ms, "push_ms_per_step": push_ms,
                       "push_variant": PUSH_KINDS[info.push_kind] + f":{info.push_param}",
                       "local_windows": int(info.local_windows),
                       "push_autotune": tuning,
                       "step_roofline_frac": step_bytes / ((lif_ms + push_ms) * 1e-3) / 1e9 / peak},
            "roofline": {"bound": "hbm", "kernel": roof_kernel, "achieved": achieved, "peak": peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "algorithmic_bytes_per_launch": push_bytes},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_events / (e2e_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "clocks": clocks,
            "gpu_launches": int(launches),
        }
        if cpu:
            out["config"]["gpu_over_cpu_port"] = value / cpu["value"]
    eng.close()
    del stream
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if out is not None and world == 1 and not args.no_forms and args.net == "regional" and \
            args.neurons == N_NEURONS:
        # the metric's second half, batched/served vs plain at equal rate, on reduced configurations
        out["batched"] = measure_ensemble(16, 4, 800, 3, args.batched_syn)
        out["served"] = measure_serve(32, 60, 40.0, 800, 100, 150.0, args.batched_syn)
    return out


def isi_cv(spikes):
    """Pooled ISI coefficient of variation of a [steps, neurons] boolean raster."""
    isis = []
    for j in range(spikes.shape[1]):
        t = np.nonzero(spikes[:, j])[0]
        if t.size > 2:
            isis.append(np.diff(t))
    if not isis:
        return float("nan")
    x = np.concatenate(isis).astype(np.float64)
    return float(x.std() / x.mean())


def _clock_sampler(torch):
    return ClockSampler(str(getattr(torch.cuda.get_device_properties(torch.cuda.current_device()), "uuid", "")))


def measure_ensemble(n_members, windows, W, warmup, batched_syn, seed=3):
    """Batched BF16 data-assimilation ensemble vs the same members run one by one through
    the plain FP32 path, same windows and property updates.  Returns the comparison."""
    import torch
    import __graft_entry__
    __graft_entry__.load_package()
    from dtb_b200 import engine as E
    from dtb_b200 import network as nw

    specs = nw.ensemble_specs(n_members=n_members, seed=seed)
    rng_hp = np.random.default_rng(11)
    # per-window DA hyper-parameter factors (mul_property_by_subblk of g_AMPA per population)
    factors = [[rng_hp.uniform(0.97, 1.03, s.n_pops).astype(np.float32) for s in specs] for _ in range(windows)]
    samples = [np.linspace(0, s.n - 1, 200).astype(np.uint32) for s in specs]
    g_ampa = E.PROP_IDS["CONDUCT_G_AMPA"]

    def build(wt, seed_base=100, members=None):
        t0 = time.perf_counter()
        engs = [E.Engine.structured(s, weight_type=wt, seed=seed_base + i) for i, s in enumerate(specs[:members])]
        for e, smp in zip(engs, samples):
            e.set_samples(smp)
        torch.cuda.synchronize()
        return engs, time.perf_counter() - t0

    def summarise(results):
        rates, cvs = [], []
        for i, (fr, ss) in enumerate(results):
            rates.append(fr.sum(0) / (fr.shape[0] * specs[i].pop_sizes) * 1e4)
            cvs.append(isi_cv(ss.astype(bool)))
        return rates, np.array(cvs)

    # ---- batched BF16 (one graph-replayed launch sequence per window for all members)
    bsyn = E.SYN_PUSH_FIXED if batched_syn == "fixed" else E.SYN_PUSH
    engs, build_b = build(E.W_BF16)
    batch = E.Batch(engs)
    for _ in range(warmup):
        batch.run(W, syn_mode=bsyn)
    acc = [[np.zeros((0, s.n_pops), np.int32), np.zeros((0, 200), np.uint8)] for s in specs]
    ev_b = 0
    dev_b = 0.0
    sampler = _clock_sampler(torch)
    sampler.start()
    t0 = time.perf_counter()
    for w in range(windows):
        for e, s, f in zip(engs, specs, factors[w]):
            e.update_prop_cols([g_ampa] * s.n_pops, np.arange(s.n_pops), f)
        res = batch.run(W, sample_spike=True, syn_mode=bsyn)
        dev_b += res[0].device_ms
        for i, r in enumerate(res):
            ev_b += r.events
            acc[i][0] = np.concatenate([acc[i][0], r.freqs])
            acc[i][1] = np.concatenate([acc[i][1], r.sample_spike])
    wall_b = time.perf_counter() - t0
    clocks = sampler.stop()
    rates_b, cv_b = summarise(acc)
    binfo = batch.info()
    batch.close()
    for e in engs:
        e.close()
    del engs
    # ---- sequential plain FP32 (each member through its own dtb_run)
    engs, build_s = build(E.W_F32)
    for e in engs:
        for _ in range(warmup):
            e.run(W)
    acc = [[np.zeros((0, s.n_pops), np.int32), np.zeros((0, 200), np.uint8)] for s in specs]
    ev_s = 0
    dev_s = 0.0
    t0 = time.perf_counter()
    for w in range(windows):
        for i, (e, s, f) in enumerate(zip(engs, specs, factors[w])):
            e.update_prop_cols([g_ampa] * s.n_pops, np.arange(s.n_pops), f)
            r = e.run(W, sample_spike=True)
            dev_s += r.device_ms
            ev_s += r.events
            acc[i][0] = np.concatenate([acc[i][0], r.freqs])
            acc[i][1] = np.concatenate([acc[i][1], r.sample_spike])
    wall_s = time.perf_counter() - t0
    rates_s, cv_s = summarise(acc)
    for e in engs:
        e.close()
    # noise floor of the comparison: the first members again on the same FP32 path with other
    # seeds (another realisation of the same network, untimed)
    n_sp = min(8, len(specs))
    engs, _ = build(E.W_F32, seed_base=5000, members=n_sp)
    acc2 = [[np.zeros((0, s.n_pops), np.int32), np.zeros((0, 200), np.uint8)] for s in specs[:n_sp]]
    for e in engs:
        for _ in range(warmup):
            e.run(W)
    for w in range(windows):
        for i, (e, s, f) in enumerate(zip(engs, specs, factors[w])):
            e.update_prop_cols([g_ampa] * s.n_pops, np.arange(s.n_pops), f)
            r = e.run(W, sample_spike=True)
            acc2[i][0] = np.concatenate([acc2[i][0], r.freqs])
            acc2[i][1] = np.concatenate([acc2[i][1], r.sample_spike])
    for e in engs:
        e.close()
    rates_2, cv_2 = summarise(acc2)
    rate_rel = np.concatenate([np.abs(a - b) / np.maximum(b, 1e-9) for a, b in zip(rates_b, rates_s)])
    rate_seed = np.concatenate([np.abs(a - b) / np.maximum(b, 1e-9) for a, b in zip(rates_2, rates_s)])
    member_steps = len(specs) * windows * W
    return {
        "workload": f"{len(specs)} ensemble members (N in [20k, 400k], in-degree in {{100, 200, 500}}, 10-50 "
                    f"populations), {windows} windows of {W} steps, g_AMPA multiplied per population between "
                    f"windows, {warmup} warm-up window(s)",
        "neurons": int(sum(s.n for s in specs)), "synapses": int(sum(s.n_edges for s in specs)),
        "batched_synaptic_mode": batched_syn, "sequential_synaptic_mode": "push",
        "batched_graph_launches": binfo["graph_launches"],
        "batched_push_variant": binfo["push_kind"] * 10000 + binfo["push_param"],
        "batched_bf16": {"events_per_s_wall": ev_b / wall_b, "events_per_s_device": ev_b / (dev_b / 1e3),
                         "member_steps_per_s": member_steps / wall_b, "wall_s": wall_b, "device_s": dev_b / 1e3,
                         "build_s": build_b},
        "sequential_f32": {"events_per_s_wall": ev_s / wall_s, "events_per_s_device": ev_s / (dev_s / 1e3),
                           "member_steps_per_s": member_steps / wall_s, "wall_s": wall_s, "device_s": dev_s / 1e3,
                           "build_s": build_s},
        "speedup_wall": (ev_b / wall_b) / (ev_s / wall_s),
        "speedup_device": (ev_b / dev_b) / (ev_s / dev_s),
        "accuracy_bf16_batched_vs_f32_sequential": {
            "mean_rate_hz": float(np.mean(np.concatenate(rates_b))),
            "population_rate_rel_diff_median": float(np.median(rate_rel)),
            "population_rate_rel_diff_p95": float(np.percentile(rate_rel, 95)),
            "isi_cv_batched_mean": float(np.nanmean(cv_b)), "isi_cv_sequential_mean": float(np.nanmean(cv_s)),
            "isi_cv_rel_diff_median": float(np.nanmedian(np.abs(cv_b - cv_s) / cv_s)),
            # the same statistics between two seeds of the sequential FP32 path (first members):
            # what two realisations of one network differ by
            "seed_spread_members": n_sp,
            "population_rate_rel_diff_median_fp32_two_seeds": float(np.median(rate_seed)),
            "isi_cv_rel_diff_median_fp32_two_seeds": float(np.nanmedian(np.abs(cv_2 - cv_s[:n_sp]) / cv_s[:n_sp])),
        },
        "clocks": clocks,
    }


def run_ensemble(args):
    m = measure_ensemble(args.members or 64, args.steps, args.window, args.warmup, args.batched_syn)
    wall_b = m["batched_bf16"]["wall_s"]
    return {
        "metric": METRIC, "form": "ensemble", "value": m["batched_bf16"]["events_per_s_wall"],
        "unit": UNIT + " (ensemble, wall)", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * wall_b / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16-weights/f32-state", "data": "synthetic (seeded DA members generated on the device)",
        "config": {k: m[k] for k in ("workload", "neurons", "synapses", "batched_graph_launches",
                                     "batched_synaptic_mode", "sequential_synaptic_mode", "batched_push_variant")},
        **{k: m[k] for k in ("batched_bf16", "sequential_f32", "speedup_wall", "speedup_device",
                             "accuracy_bf16_batched_vs_f32_sequential", "clocks")},
    }


def measure_serve(n_nets, n_requests, rate, window, slice_steps, cap_gb, batched_syn, seed=4):
    """Served form: a Poisson stream of simulate-window requests over resident networks,
    continuous batching (BF16) vs the plain single-network path one request at a time (FP32),
    at the same offered rate."""
    import torch
    import __graft_entry__
    __graft_entry__.load_package()
    from dtb_b200 import engine as E
    from dtb_b200 import network as nw

    specs = nw.ensemble_specs(n_members=n_nets, seed=seed)
    rng = np.random.default_rng(12)
    t, reqs = 0.0, []
    for _ in range(n_requests):
        t += float(rng.exponential(1.0 / rate))
        net = int(rng.integers(len(specs)))
        P = specs[net].n_pops
        ou = (rng.uniform(0.55, 0.65, P).astype(np.float32), rng.uniform(0.18, 0.22, P).astype(np.float32),
              np.full(P, 10.0, np.float32))
        reqs.append(dict(net=net, iters=window, arrival_s=t, ou=ou))
    # warm-up past step 300 plus the tuner's samples (every 47 steps) on every network, so each
    # engine (plain path) and the batch (batched path) has autotuned its push before the timed trace
    warm = [dict(net=i, iters=600, arrival_s=0.0, ou=None) for i in range(len(specs))]

    def serve(wt, policy, syn):
        t0 = time.perf_counter()
        srv = E.Server(hbm_cap_bytes=cap_gb * 1e9, slice_steps=slice_steps, max_batch=64, syn_mode=syn,
                       autotune=True)
        for i, sp in enumerate(specs):
            srv.add_structured(sp, weight_type=wt, seed=200 + i)
        build_s = time.perf_counter() - t0
        srv.play(warm, policy)
        torch.cuda.synchronize()
        sampler = _clock_sampler(torch)
        sampler.start()
        got = srv.play(reqs, policy)
        clocks = sampler.stop()
        info = srv.info()
        srv.close()
        lat = np.array([g["latency_s"] for g in got]) * 1e3
        svc = np.array([g["finish_s"] - g["start_s"] for g in got]) * 1e3
        span = max(g["finish_s"] for g in got) - reqs[0]["arrival_s"]
        ev = sum(g["events"] for g in got)
        rates = np.concatenate([g["freqs"].sum(0) / (window * specs[r["net"]].pop_sizes) * 1e4
                                for g, r in zip(got, reqs)])
        return {"latency_ms": {"p50": float(np.percentile(lat, 50)), "p90": float(np.percentile(lat, 90)),
                               "p99": float(np.percentile(lat, 99)), "mean": float(lat.mean()), "max": float(lat.max())},
                "in_service_ms_mean": float(svc.mean()), "events_per_s": ev / span, "span_s": span,
                "requests_per_s": len(got) / span, "build_s": build_s,
                "mean_requests_per_slice": info["batch_members_sum"] / max(1, info["slices"]),
                "evictions": info["evictions"], "resident_gb": info["resident_bytes"] / 1e9,
                "clocks": clocks}, rates

    batched, rates_b = serve(E.W_BF16, E.SERVE_BATCHED, E.SYN_PUSH_FIXED if batched_syn == "fixed" else E.SYN_PUSH)
    plain, rates_s = serve(E.W_F32, E.SERVE_SEQUENTIAL, E.SYN_PUSH)
    rel = np.abs(rates_b - rates_s) / np.maximum(rates_s, 1e-9)
    return {
        "workload": f"Poisson arrivals {rate}/s, {n_requests} requests of {window} steps with new per-population "
                    f"OU parameters, {len(specs)} resident networks of the ensemble distribution, HBM cap "
                    f"{cap_gb} GB, slices of {slice_steps} steps",
        "neurons": int(sum(s.n for s in specs)), "synapses": int(sum(s.n_edges for s in specs)),
        "batched_synaptic_mode": batched_syn, "sequential_synaptic_mode": "push",
        "batched_bf16": batched, "plain_sequential_f32": plain,
        "p50_ratio_plain_over_batched": plain["latency_ms"]["p50"] / batched["latency_ms"]["p50"],
        "p99_ratio_plain_over_batched": plain["latency_ms"]["p99"] / batched["latency_ms"]["p99"],
        "population_rate_rel_diff_median": float(np.median(rel)),
    }


def run_serve(args):
    m = measure_serve(args.members or 128, args.requests, args.rate, args.window, args.slice, args.hbm_cap_gb,
                      args.batched_syn)
    return {
        "metric": METRIC, "form": "serve", "value": m["batched_bf16"]["latency_ms"]["p99"],
        "unit": "ms p99 request latency", "n_gpus": 1, "steps": args.requests, "warmup": 1,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "bf16-weights/f32-state (batched), f32 (plain)",
        "data": "synthetic (seeded networks of the ensemble distribution generated on the device)",
        "config": {k: m[k] for k in ("workload", "neurons", "synapses", "batched_synaptic_mode",
                                     "sequential_synaptic_mode")},
        **{k: m[k] for k in ("batched_bf16", "plain_sequential_f32", "p50_ratio_plain_over_batched",
                             "p99_ratio_plain_over_batched", "population_rate_rel_diff_median")},
    }


def spike_agreement(a, b):
    """First step where two rasters differ, and |A and B| / |A or B| over all steps."""
    bad = np.nonzero((a != b).any(axis=1))[0]
    inter = np.logical_and(a, b).sum()
    union = np.logical_or(a, b).sum()
    return (int(bad[0]) if bad.size else None), float(inter / max(union, 1))


def run_precision(args):
    """Precision form: bf16 weights + the deterministic pull kernel (and the float32 /
    float-push variants) against the FP64 restatement of block_new on a 200k-neuron
    network of the regional construction, with the float32 CPU model beside them."""
    import __graft_entry__
    __graft_entry__.load_package()
    from dtb_b200 import engine as E
    from dtb_b200 import network as nw
    from oracle import c_oracle as cc

    n = args.neurons if args.neurons != N_NEURONS else 200_000
    pops = max(1, round(n / 25_000)) if args.pops == N_POPS else args.pops
    steps, n_v = args.window, 64
    warm = 200
    spec = nw.structured_spec(n, pops, args.degree, SPEC_SEED)
    net = cc.structured_edges(spec)
    z = np.random.default_rng(7).standard_normal((steps, n), dtype=np.float32)
    t0 = time.perf_counter()
    sp64, cnt64, ev64, v64 = cc.COracle64(net).run(z, n_v=n_v)
    t64 = time.perf_counter() - t0
    t0 = time.perf_counter()
    sp32, _, _ = cc.COracle(net).run(z)
    t32 = time.perf_counter() - t0
    sp64c, _, _, _ = cc.COracle64(net).run(z, clock32=True)
    del net
    pop_of = np.repeat(np.arange(pops), spec.pop_sizes)

    def pop_rates(sp):
        return np.bincount(pop_of, weights=sp[warm:].sum(0), minlength=pops) / (spec.pop_sizes * (steps - warm)) * 1e4

    r64 = pop_rates(sp64)

    r32 = pop_rates(sp32)

    def compare(sp, vt=None):
        first, jac = spike_agreement(sp, sp64)
        r = pop_rates(sp)
        rel = np.abs(r - r64) / np.maximum(r64, 1e-9)
        rel32 = np.abs(r - r32) / np.maximum(r32, 1e-9)
        first32, jac32 = spike_agreement(sp, sp32)
        out = {"first_divergence_step": first, "spike_jaccard": jac,
               "rate_hz": float(sp[warm:].mean() * 1e4), "pop_rate_rel_err_median": float(np.median(rel)),
               "pop_rate_rel_err_max": float(rel.max()),
               "vs_f32_block_new": {"first_divergence_step": first32, "spike_jaccard": jac32,
                                    "pop_rate_rel_diff_max": float(rel32.max())}}
        if vt is not None:
            upto = first if first is not None else steps
            if upto > 0:
                d = np.abs(vt[:upto] - v64[:upto]) / np.abs(v64[:upto])
                out["v_rel_err_max_before_divergence"] = float(d.max())
        return out

    res = {"cpu_f32_block_new": compare(sp32), "cpu_fp64_with_float32_clock": compare(sp64c)}
    idx = np.arange(n_v, dtype=np.uint32)
    for name, wt, syn in (("gpu_bf16_pull", E.W_BF16, E.SYN_PULL), ("gpu_f32_pull", E.W_F32, E.SYN_PULL),
                          ("gpu_bf16_push", E.W_BF16, E.SYN_PUSH), ("gpu_f32_push", E.W_F32, E.SYN_PUSH)):
        with E.Engine.structured(spec, weight_type=wt, push=syn != E.SYN_PULL, pull=syn == E.SYN_PULL) as eng:
            eng.set_noise_injected(z)
            eng.set_samples(idx)
            r = eng.run(steps, record_spikes=True, sample_v=True, syn_mode=syn)
            res[name] = compare(r.spikes, r.sample_v)
            res[name]["device_ms_per_step"] = r.device_ms / steps
    return {
        "metric": METRIC, "form": "precision", "value": res["gpu_bf16_pull"]["pop_rate_rel_err_median"],
        "unit": "median relative error of population rates vs FP64", "n_gpus": 1, "steps": steps, "warmup": 0,
        "higher_is_better": False, "dtype": "bf16-weights/f32-state",
        "data": "synthetic (seeded regional network, replayed on the host for the oracles)",
        "config": {"workload": f"{n}-neuron regional network, {pops} populations, in-degree {args.degree}, "
                               f"{steps} steps, injected float32 normal draws shared by every run, "
                               f"rates over steps {warm}-{steps}",
                   "neurons": n, "synapses": int(spec.n_edges), "fp64_oracle_s": t64, "f32_oracle_s": t32,
                   "fp64_rate_hz": float(sp64[warm:].mean() * 1e4), "fp64_events": ev64},
        "vs_fp64": res,
    }


def run_reference(args):
    """The reference arm: the C port of the reference CPU model (models/block_new.py) on the
    box's host cores -- W warm-up and K timed bench steps of the CPU sample; rank 0 only."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    cpu = cpu_port_run(args.steps, args.warmup)
    v = cpu["value"]
    return {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": cpu["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded regional network, generated on the host)",
        "sim_ms_per_wall_s": cpu["sim_ms_per_wall_s"],
        "config": {"workload": CPU_WORKLOAD, "neurons": CPU_SAMPLE["n"], "populations": CPU_SAMPLE["pops"],
                   "in_degree": CPU_SAMPLE["in_degree"], "sim_steps_per_bench_step": CPU_SAMPLE["per_step"],
                   "timed_sim_steps": args.steps * CPU_SAMPLE["per_step"], "timed_s": cpu["wall_s"]},
        "cpu_baseline": {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample")},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    args = parse()
    if args.impl == "reference":
        out = run_reference(args)
    elif args.form == "ensemble":
        out = run_ensemble(args)
    elif args.form == "serve":
        out = run_serve(args)
    elif args.form == "precision":
        out = run_precision(args)
    else:
        out = run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
