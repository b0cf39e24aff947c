#!/usr/bin/env python
"""UMAP fit benchmark on B200: the 70,000 x 784 full pipeline.

Workload (one step = one complete fit): seeded prototype mixture 70,000 x 784
(10 classes of 7,000; stands in for Fashion-MNIST, which is not available
offline), NNDescent k=15 with the reference's defaults (n_iters 20, delta
0.015), fuzzy simplicial set, spectral init, 500 layout epochs, 2 components.

  value   positive-edge updates of the whole fit per second, summed over ranks
          (edges/s of the whole fit_transform, inputs resident on the device)
  fit_s   seconds per fit (the other half of the metric)
  e2e     the same metric through UMAP.fit_transform on a pinned host tensor,
          host->device input and device->host embedding copies inside the timing
  roofline  the layout epoch (sgd_epoch_kernel + apply_kernel), the largest
          kernel share of a fit: 112 algorithmic bytes per active edge over the
          layout stage's CUDA-event time divided by the epochs
          (+ random_access: 8-byte random reads and atomic adds per second against
          a probe of that access rate on the same table)
  roofline_nndescent  one NNDescent iteration (join + row kernel), CUDA events
          around each launch in the timed fits, against two byte counts: every
          reference candidate row read once, and the rows the blocked join reads
          (+ row_gather: the rows' bytes at a probe's rate for random rows)
  knn_brute  the 20000 x 784 exact-kNN workload (untimed record): its three
          launches timed with CUDA events, tile kernel against the BF16 peak
  learned_init  layout epochs the learned warm start needs to reach the
          500-epoch spectral trustworthiness (untimed record)
  cpu_baseline  the NumPy port of the reference algorithm on the host cores, the
          70,000-row workload at full size with each stage's work units sampled
          (oracle.pipeline.FitSampler)

N > 1 (torchrun): every rank fits its own replica (weak scaling, no
collective on the data path); time = max over ranks.
`--impl reference` times the reference algorithm's CPU port: each step one
sampled full-size fit of FitSampler, rank 0 only.
"""

from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "UMAP fit s & edges/s @70K×784"
N_FULL, D, K_NN, N_EPOCHS = 70000, 784, 15, 500


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--n", type=int, default=N_FULL, help="rows (default: the 70K workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the untimed brute-kNN and learned-init records of the fit line")
    ap.add_argument("--case", choices=["fit", "learned_init", "scale", "nndescent", "nndescent_1m", "knn_brute",
                                       "layout", "encoder"], default="fit",
                    help="fit: the benchmark line; learned_init: epochs-to-trustworthiness of the learned warm start; "
                         "scale: the 1,000,000 x 128 configuration (plain fit, learned vs plain init); "
                         "nndescent / knn_brute / layout: one untimed run of that stage (profiler captures); "
                         "nndescent_1m: one untimed NNDescent build on the 1,000,000 x 128 configuration")
    return ap.parse_args()


def make_data(n):
    from mlx_vis_b200.datasets import prototype_mixture

    return prototype_mixture(n, D, seed=0)


def config(n):
    return {"workload": f"UMAP fit_transform of a {n}x{D} seeded prototype mixture (10 classes); NNDescent k={K_NN} "
                        f"(n_iters 20, delta 0.015), fuzzy set, spectral init, {N_EPOCHS} epochs, 2 components",
            "n": n, "d": D, "n_neighbors": K_NN, "n_epochs": N_EPOCHS, "min_dist": 0.1, "knn_method": "nndescent",
            "init": "spectral", "parallelism": "replicas (one independent fit per GPU)",
            "l2": f"inputs larger than L2: every step streams X ({n * D * 4 / 1e6:.1f} MB fp32, above the 126 MB L2) "
                  "to build its FP16 copy, which evicts the previous step's data"}


# --------------------------------------------------------------------------
def schedule_edge_updates(vals: np.ndarray, n_epochs: int) -> int:
    """Positive-edge updates of a fit: the float32 schedule of umap.py:398-414."""
    w = vals.astype(np.float32)
    n_samples = n_epochs * (w / float(w.max()))
    eps = np.where(n_samples > 0, n_epochs / n_samples, -1.0).astype(np.float32)
    nxt = eps.copy()
    total = 0
    for e in range(n_epochs):
        act = nxt <= e
        c = int(act.sum())
        if c:
            nxt[act] += eps[act]
            total += c
    return total


class Clocks:
    """SM clock and clock-event reasons sampled every 10 ms through NVML while the
    timed region runs (the device is matched to the CUDA device by PCI bus id);
    nvidia-smi at 200 ms when NVML is unavailable."""

    NAMES = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4,
             "hw_power_brake_slowdown": 0x80}

    def __init__(self, index):
        import threading

        self.sm, self.smax, self.reasons, self.power = [], [], set(), []
        self.stop_evt = threading.Event()
        self.thread = None
        self.smi = None
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            pr = torch.cuda.get_device_properties(index)
            try:
                bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
                h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            except Exception:
                h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.smax.append(float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)))

            def poll():
                while not self.stop_evt.is_set():
                    try:
                        self.sm.append(float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)))
                        bits = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                        for nm, b in self.NAMES.items():
                            if bits & b:
                                self.reasons.add(nm)
                        self.power.append(pynvml.nvmlDeviceGetPowerUsage(h) / 1000.0)
                    except Exception:
                        pass
                    self.stop_evt.wait(0.01)

            self.thread = threading.Thread(target=poll, daemon=True)
            self.thread.start()
        except Exception:
            self._start_smi(index)

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def _start_smi(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.smi = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}",
                                         "--format=csv,noheader", "-lms", "200"], stdout=self.f,
                                        stderr=subprocess.DEVNULL)
        except Exception:
            self.smi = None

    def stop(self):
        if self.thread is not None:
            self.stop_evt.set()
            self.thread.join(timeout=5)
            return {"sm_mhz": statistics.median(self.sm) if self.sm else None,
                    "sm_max_mhz": max(self.smax) if self.smax else None, "reasons": sorted(self.reasons),
                    "samples": len(self.sm), "power_w_max": max(self.power) if self.power else None,
                    "source": "nvml, 10 ms"}
        if self.smi is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.smi.terminate()
        self.smi.wait(timeout=10)
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1].split()[0]))
                smax.append(float(parts[2].split()[0]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def measured_peaks():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def measured_bf16_peak():
    """Dense BF16 TFLOP/s (burst: kernels timed alone)."""
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


def committed_traffic(name: str = "nnd_iteration_70k.md"):
    """Per-launch DRAM bytes of a roofline kernel from its committed ncu summary, if any."""
    path = os.path.join(HERE, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return float(line.split(":", 1)[1])
    except OSError:
        pass
    return None


# --------------------------------------------------------------------------
def _row_bytes(info) -> int:
    """Bytes of one distance-space row of an NNDescent iteration (FP16 rows padded to
    multiples of 8 elements)."""
    if info["elem"] == 2:
        return (info["space"] + 7) // 8 * 8 * 2
    return info["space"] * 4


def access_probes(torch, n, row_sizes):
    """Measured ceilings of the two gather-bound steps (untimed, after the timed fits):
    random 8-byte reads and atomic adds on an n x 2 table at 4 and at 3 reads per add
    (the layout's Y; an epoch makes 7 reads and 2 adds per active edge), and one warp per
    random row of each distance-space row size (the NNDescent join's row reads,
    31 n rows)."""
    from mlx_vis_b200 import _lib

    dev = torch.device("cuda")
    s = _lib.stream_handle()

    def best(fn, reps=5):
        fn()
        fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            fn()
            b.record()
            torch.cuda.synchronize()
            ts.append(a.elapsed_time(b) * 1e-3)
        return min(ts)

    table = torch.zeros((n, 2), device=dev)  # the values do not matter, the addresses do
    dtab = torch.zeros((n, 2), device=dev)
    sink = torch.zeros(16, device=dev)
    threads = torch.cuda.get_device_properties(dev).multi_processor_count * 2048
    per = 128
    mix = {}
    for red in (4, 3):  # an atomic add after every `red` reads
        t = best(lambda: _lib.call("umapb_probe_random_access", _lib.ptr(table), _lib.ptr(dtab), n, 2, threads, per,
                                   red, _lib.ptr(sink), s))
        mix[red] = (per, (per + red - 1) // red, t)
    # time = threads (reads c_r + adds c_a): the two mixes give c_r and c_a, and with
    # them the rate at the epoch's mix of 7 reads and 2 adds
    (r4, a4, t4), (r3, a3, t3) = mix[4], mix[3]
    c_a = (t3 - t4) / threads / (a3 - a4)
    c_r = (t4 / threads - a4 * c_a) / r4
    rate4 = threads * (r4 + a4) / t4
    random_rate = {"4:1": rate4, "3:1": threads * (r3 + a3) / t3,
                   "7:2": 9.0 / (7 * c_r + 2 * c_a) if c_r > 0 and c_a > 0 else rate4}
    ids = torch.from_numpy(np.random.default_rng(0).integers(0, n, 31 * n, dtype=np.int32)).to(dev)
    rates = {}
    for rb in sorted(set(row_sizes)):
        tab = torch.zeros(n * rb, dtype=torch.uint8, device=dev)
        t = best(lambda: _lib.call("umapb_probe_row_gather", _lib.ptr(tab), n, rb, _lib.ptr(ids), ids.numel(),
                                   _lib.ptr(sink), s))
        rates[rb] = ids.numel() * rb / t
        del tab
    return random_rate, rates


def max_over_ranks(value: float, dist, device) -> float:
    """The largest per-rank value (a time): every rank calls this at the same point."""
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(units_per_rank: float, world: int, ms_max: float) -> float:
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    return units_per_rank * world / (ms_max * 1e-3)


def run_ours(args, rank, world, local_rank):
    import torch

    from mlx_vis_b200 import UMAP, _lib

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=torch.device("cuda", local_rank))
    n = args.n
    X = make_data(n)
    Xd = torch.from_numpy(X).cuda()
    X_pinned = torch.from_numpy(X).pin_memory()

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def make():
        return UMAP(n_components=2, n_neighbors=K_NN, min_dist=0.1, n_epochs=N_EPOCHS, knn_method="nndescent",
                    random_state=0)

    for _ in range(max(args.warmup, 3)):
        make().fit_transform_device(Xd)
    u = make()
    u.fit_transform(X_pinned)  # warm the host path too

    # positive-edge updates per fit: deterministic given the graph, counted untimed
    # from the same graph stage (NNDescent seed 0, fuzzy set) on the host
    from mlx_vis_b200._nndescent.nndescent import NNDescent

    idx, dd = NNDescent(k=K_NN, random_state=0).build_device(Xd)
    rows, cols, vals, ne = _lib.fuzzy(idx, dd, N_EPOCHS, fp64=True)
    E = int(ne.item())
    edges_per_fit = schedule_edge_updates(vals[:E].cpu().numpy(), N_EPOCHS)

    # ---- device-resident timing ----
    launches0 = _lib.kernel_launches()
    models = [make() for _ in range(args.steps)]
    for m in models:
        m.profile_kernels = True
    barrier()
    gc_pauses = []  # Python garbage-collector pauses inside the timed fits (ms)
    gc_t = [0.0]

    def gc_cb(phase, info):
        if phase == "start":
            gc_t[0] = time.perf_counter()
        else:
            gc_pauses.append((time.perf_counter() - gc_t[0]) * 1e3)

    import gc

    gc.callbacks.append(gc_cb)
    clk = Clocks(local_rank)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record()
    for m in models:
        m.fit_transform_device(Xd)
    t1.record()
    barrier()
    clocks = clk.stop()
    gc.callbacks.remove(gc_cb)
    launches = _lib.kernel_launches() - launches0
    ms = max_over_ranks(t0.elapsed_time(t1) / args.steps, dist, "cuda")

    gc_ms = [round(x, 2) for x in gc_pauses]
    fit_ms_each = [round(m.timings_["total_device"], 2) for m in models]
    stage_ms_each = [{k: round(v, 2) for k, v in m.timings_.items()} for m in models]
    peak, peak_kind = measured_peaks()
    # primary roofline: the layout epoch, the largest kernel share of a fit.  112 B per
    # active edge (edge ids, two Y gathers and two atomic adds of the pair, and per
    # negative sample one gather and one add, at 2 components and rate 5); one epoch =
    # sgd_epoch_kernel + apply_kernel, timed as the layout stage's events / epochs
    lay_ms = sorted(m.timings_["layout"] for m in models)[len(models) // 2]
    t_epoch = lay_ms * 1e-3 / N_EPOCHS
    b_epoch = 112.0 * edges_per_fit / N_EPOCHS
    achieved = b_epoch / t_epoch / 1e9
    roofline = {"kernel": "layout sgd_epoch_kernel<2, 5> + apply_kernel (one epoch)", "bound": "hbm",
                "achieved": round(achieved, 1), "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                "frac": round(achieved / peak, 3), "traffic": committed_traffic("layout_epoch_70k.md"),
                "algorithmic_bytes_per_launch": int(b_epoch), "avg_launch_ms": round(t_epoch * 1e3, 4),
                "launches_per_fit": N_EPOCHS,
                "note": "Y (560 KB) and the edge arrays are L2-resident, so DRAM traffic is far below the "
                        "algorithmic bytes; the epoch is bound by the latency of its random 8-byte Y gathers"}
    # NNDescent iterations from the events around each launch of the timed fits
    durs, bytes_ref, bytes_blk = [], [], []
    for m in models:
        for e0, e1, info in m.nndescent_.kernel_log_:
            durs.append(e0.elapsed_time(e1) * 1e-3)
            s, dsp, kk, nn = info["elem"], info["space"], info["k"], info["n"]
            t_new = info["candidates"] - kk  # mc_new * j_nn (+ k reverse): the reference's candidate count
            ids = nn * (kk + t_new) * 8
            # every reference candidate row read once, plus the query row
            bytes_ref.append(nn * (t_new + 1) * dsp * s + ids)
            if info.get("join"):
                # blocked join: each row once per source that lists it (mc_new), each source
                # and its first j_nn neighbours once, the join's distances written and read
                mc, jn = info["mc_new"], info["j_nn"]
                bytes_blk.append(nn * (mc + 1 + jn) * dsp * s + ids + nn * (mc * jn + kk) * 4 * 2)
            else:
                bytes_blk.append(bytes_ref[-1])
    per_iter = [round(e0.elapsed_time(e1), 3) for e0, e1, _ in models[-1].nndescent_.kernel_log_]
    avg_t = sum(durs) / len(durs)
    avg_ref = sum(bytes_ref) / len(bytes_ref)
    avg_blk = sum(bytes_blk) / len(bytes_blk)
    roofline_nnd = {"kernel": "nndescent join kernel + row kernel (one iteration)", "bound": "hbm", "unit": "GB/s",
                    "peak": peak, "peak_source": peak_kind,
                    "achieved_reference_bytes": round(avg_ref / avg_t / 1e9, 1),
                    "frac_reference_bytes": round(avg_ref / avg_t / 1e9 / peak, 3),
                    "achieved_blocked_bytes": round(avg_blk / avg_t / 1e9, 1),
                    "frac_blocked_bytes": round(avg_blk / avg_t / 1e9 / peak, 3),
                    "traffic": committed_traffic(), "reference_bytes_per_launch": int(avg_ref),
                    "blocked_bytes_per_launch": int(avg_blk), "avg_launch_ms": round(avg_t * 1e3, 3),
                    "launches_per_fit": len(durs) // args.steps, "launch_ms_last_fit": per_iter,
                    "note": "reference bytes count every row of the reference's candidate list as read once "
                            "(above the HBM rate because the join reuses rows); blocked bytes are the rows the "
                            "join and the row kernel must read"}

    # measured ceilings of the two gather-bound steps (rank 0, untimed)
    if rank == 0:
        last = models[-1].nndescent_.kernel_log_
        sizes = [_row_bytes(info) for _, _, info in last]
        random_rate, row_rates = access_probes(torch, n, sizes)
        acc_epoch = 9.0 * edges_per_fit / N_EPOCHS  # 7 reads + 2 atomic adds per active edge (rate 5, 2-D)
        roofline["random_access"] = {
            "achieved_g_per_s": round(acc_epoch / t_epoch / 1e9, 1),
            "probe_g_per_s": round(random_rate["7:2"] / 1e9, 1),
            "frac": round(acc_epoch / t_epoch / random_rate["7:2"], 3),
            "probe_g_per_s_4to1": round(random_rate["4:1"] / 1e9, 1),
            "probe_g_per_s_3to1": round(random_rate["3:1"] / 1e9, 1),
            "frac_4to1": round(acc_epoch / t_epoch / random_rate["4:1"], 3),
            "note": "8-byte random reads and float2 atomic adds per second on the same n x 2 table; the probe "
                    "(umapb_probe_random_access) runs with 4 and with 3 reads per add, which give the cost of "
                    "a read and of an add, and probe_g_per_s is the rate at the epoch's mix of 7 reads and 2 "
                    "adds per active edge"}
        bound = 0.0
        for (e0, e1, info), rb in zip(last, sizes):
            rows = info["n"] * (info["mc_new"] + 1 + info["j_nn"] if info.get("join") else
                                info["candidates"] - info["k"] + 1)
            bound += rows * rb / row_rates[rb]
        meas = sum(e0.elapsed_time(e1) for e0, e1, _ in last) * 1e-3
        roofline_nnd["row_gather"] = {
            "probe_gb_per_s": {str(rb): round(r / 1e9, 1) for rb, r in row_rates.items()},
            "bound_ms_per_fit": round(bound * 1e3, 3), "measured_ms_per_fit": round(meas * 1e3, 3),
            "frac": round(bound / meas, 3),
            "note": "bound: each iteration's candidate-row bytes (the join's rows, or the reference's candidate "
                    "rows when the row kernel computes every distance) at the probe's rate for random rows of that "
                    "size (umapb_probe_row_gather, one warp per row)"}

    # ---- end to end through the public API (pinned host input, host output) ----
    barrier()
    h0 = time.perf_counter()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        Y = make().fit_transform(X_pinned)
    e1.record()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, dist, "cuda")
    e2e_wall = (time.perf_counter() - h0) * 1e3 / args.steps
    iters = len(models[-1].nndescent_.history_)
    h2d = n * D * 4 + n * K_NN * 4 + D * 100 * 4 + D * 300 * 4 + n * 2 * 4
    d2h = n * 2 * 4 + iters * 16

    out = None
    if rank == 0:
        stages = models[-1].timings_
        out = {"metric": METRIC, "value": job_rate(edges_per_fit, world, ms), "unit": "edges/s",
               "n_gpus": world, "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": round(ms, 3),
               "fit_s": round(ms * 1e-3, 4), "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "fp32 (fp16 NNDescent iterations 1-4 and bf16 brute-force tiles as in the design; fp64 sigma)",
               "data": "synthetic (seeded prototype mixture standing in for Fashion-MNIST)",
               "config": config(n),
               "edges_per_fit": edges_per_fit, "n_edges_graph": E,
               "stage_ms": {k: round(v, 2) for k, v in stages.items()}, "fit_ms_each": fit_ms_each,
               "stage_ms_each": stage_ms_each, "gc_pause_ms": gc_ms,
               "layout_edges_per_s": edges_per_fit / (stages["layout"] * 1e-3),
               "roofline": roofline, "roofline_nndescent": roofline_nnd,
               "e2e": {"value": job_rate(edges_per_fit, world, e2e_ms), "unit": "edges/s", "fit_s": round(e2e_ms * 1e-3, 4),
                       "wall_ms_per_step": round(e2e_wall, 2), "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
               "gpu_launches": launches, "gpu_launches_per_step": launches // args.steps,
               "clocks": clocks}
        if not args.no_extras and world == 1:
            # untimed records after the timed region: the brute-force kNN workload
            # (20000 x 784) and the learned warm start against plain init
            out["knn_brute"] = knn_brute_record(torch)
            out["learned_init"] = learned_init_record(torch, X)
        if not args.no_cpu_baseline and world == 1 and n == N_FULL:
            out["cpu_baseline"] = cpu_baseline()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out


def knn_brute_record(torch):
    """umapb_knn_brute on the 20000 x 784 exact-kNN workload (k = 15, 31 candidates
    reranked), the three launches timed with CUDA events (median of 5 calls after 2
    warm-up calls): roofline of the tensor-core tile kernel on 2 n^2 d FLOPs."""
    from mlx_vis_b200 import _lib
    from mlx_vis_b200.datasets import prototype_mixture

    n = 20000
    Xd = torch.from_numpy(prototype_mixture(n, D, seed=0)).cuda()
    runs = [_lib.knn_brute_timed(Xd, K_NN, extra=16)[2] for _ in range(7)][2:]
    med = [statistics.median(r[i] for r in runs) for i in range(3)]
    peak, src = measured_bf16_peak()
    flops = 2.0 * n * n * D
    call_ms = sum(med)
    return {"workload": f"{n}x{D} prototype mixture, k={K_NN}, BF16 tcgen05 tiles + FP32 rerank of {K_NN + 16}",
            "stage_ms": {"prep": round(med[0], 4), "tiles": round(med[1], 4), "rerank": round(med[2], 4)},
            "call_ms": round(call_ms, 4), "bound": "tensor", "unit": "TFLOP/s", "peak": peak, "peak_source": src,
            "achieved_tiles": round(flops / (med[1] * 1e-3) / 1e12, 1),
            "frac_tiles": round(flops / (med[1] * 1e-3) / 1e12 / peak, 3),
            "achieved_call": round(flops / (call_ms * 1e-3) / 1e12, 1),
            "frac_call": round(flops / (call_ms * 1e-3) / 1e12 / peak, 3)}


LI_TRAIN_SETS, LI_EPOCHS = 8, (25, 50, 100, 200, 500)


def learned_init_record(torch, X):
    """The metric's second half on the benchmark's own 70K input: an encoder
    784 -> 512 -> 512 -> 2 trained (by the library's kernels) on 8 seeded 20000 x 784
    draws sharing the benchmark's prototypes (seeds 1..8), then layout epochs needed
    by the learned start to reach, within 0.005, the trustworthiness@15 of 500
    epochs from the spectral start (10,000-row sample)."""
    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.datasets import prototype_mixture
    from mlx_vis_b200.encoder import Encoder
    from mlx_vis_b200.metrics import trustworthiness

    t0 = time.perf_counter()
    Xs = [prototype_mixture(20000, D, seed=j, proto_seed=0) for j in range(1, LI_TRAIN_SETS + 1)]
    enc = Encoder.train_on_umap_runs(Xs, n_epochs=200, encoder_epochs=30, seed=0)
    train_s = time.perf_counter() - t0
    Xd = torch.from_numpy(X).cuda()
    sub = np.random.default_rng(0).choice(X.shape[0], 10000, replace=False)
    curves = {}
    for init in ("spectral", "learned"):
        curves[init] = {}
        for ne in LI_EPOCHS:
            u = UMAP(n_epochs=ne, random_state=0, knn_method="nndescent", init=init, encoder=enc)
            Y = u.fit_transform_device(Xd).cpu().numpy()
            curves[init][ne] = {"trust": round(trustworthiness(X[sub], Y[sub], 15), 5),
                                "fit_ms": round(u.timings_["total_device"], 2)}
    ref = curves["spectral"][500]["trust"]
    first = {tol: {init: next((ne for ne in LI_EPOCHS if curves[init][ne]["trust"] >= ref - tol), None)
                   for init in ("spectral", "learned")} for tol in (0.005, 0.001)}
    return {"workload": f"the benchmark's {X.shape[0]}x{D} input; encoder trained on {LI_TRAIN_SETS} x 20000x{D} "
                        "draws with the same prototypes (200-epoch UMAP targets); trustworthiness@15 on 10,000 rows",
            "train_s": round(train_s, 2), "spectral_500_trust": ref, "curves": curves,
            "epochs_to_within_0.005": first[0.005], "epochs_to_within_0.001": first[0.001],
            "learned_epoch_fraction_within_0.005": (None if first[0.005]["learned"] is None
                                                    else first[0.005]["learned"] / 500)}


_SAMPLER = None


def fit_sampler():
    """The reference algorithm's CPU port on the 70K workload (oracle.pipeline.FitSampler),
    fed with the reference's own NNDescent graph and update log of this input
    (tests/golden/c3_70k.npz)."""
    global _SAMPLER
    if _SAMPLER is None:
        from mlx_vis_b200._curve import find_ab_params
        from oracle.pipeline import FitSampler

        g = np.load(os.path.join(HERE, "tests", "golden", "c3_70k.npz"))
        a, b = find_ab_params(1.0, 0.1)
        _SAMPLER = FitSampler(make_data(N_FULL), g["idx"], g["updates"], n_epochs=N_EPOCHS, a=a, b=b)
    return _SAMPLER


def cpu_baseline():
    fs = fit_sampler()
    t = time.perf_counter()
    r = fs.step()
    wall = time.perf_counter() - t
    return {"value": fs.updates_total / r["fit"], "unit": "edges/s", "fit_s": round(r["fit"], 2),
            "cores": fs.threads, "kind": "port", "sample": fs.describe(),
            "stage_s": {k: round(v, 2) for k, v in r.items() if k != "fit"}, "cpu_s": round(wall, 2),
            "reference_measured_here": "the reference's own modules on the NumPy mlx shim, the complete 70K fit, "
                                       "measured once when the fixture was made: 508 s on 8 cores"}


# --------------------------------------------------------------------------
LEARNED_TRAIN_SETS, LEARNED_TRAIN_N, LEARNED_EPOCHS = 32, 20000, (25, 50, 100, 200, 300, 500)


def run_learned_init(args):
    """Learned warm start vs spectral init: trustworthiness@15 against layout epochs.

    Encoder trained on 32 seeded 20000x784 prototype mixtures that share their 10
    prototypes (seeds 1..32, like draws from one image distribution), each embedded
    with 200 epochs; evaluated on a fresh 70000x784 draw (seed 1000) and on a
    20000x784 mixture with unseen prototypes.  Trustworthiness on a fixed 10K
    (5K) row sample, on the GPU.
    """
    import torch

    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.datasets import prototype_mixture
    from mlx_vis_b200.encoder import Encoder
    from mlx_vis_b200.metrics import trustworthiness

    t0 = time.perf_counter()
    Xs = [prototype_mixture(LEARNED_TRAIN_N, D, seed=j, proto_seed=0) for j in range(1, LEARNED_TRAIN_SETS + 1)]
    enc = Encoder.train_on_umap_runs(Xs, n_epochs=200, encoder_epochs=30, seed=0)
    train_s = time.perf_counter() - t0
    # encoder training throughput: Encoder.fit on a device-resident 80000 x 784 set
    # (19 batches of 4096 per epoch, the captured step replayed), 10 epochs after a
    # 2-epoch warm-up fit; FLOPs = 6 B (d h + h h + h c) per step
    probe = Encoder(D, seed=1)
    Xp = torch.from_numpy(np.concatenate(Xs[:4])).cuda()
    Tp = torch.from_numpy(np.concatenate(enc.train_embeddings_[:4])).cuda()
    probe.fit([Xp], [Tp], epochs=2)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s0 = probe.step_count
    e0.record()
    probe.fit([Xp], [Tp], epochs=10)
    e1.record()
    torch.cuda.synchronize()
    step_ms = e0.elapsed_time(e1) / (probe.step_count - s0)
    flops = 6.0 * 4096 * (D * enc.h + enc.h * enc.h + enc.h * enc.c)

    def trust_curve(X, init, epochs, sub):
        Xd = torch.from_numpy(X).cuda()
        out = {}
        for ne in epochs:
            u = UMAP(n_epochs=ne, random_state=0, knn_method="nndescent", init=init, encoder=enc)
            Y = u.fit_transform(Xd)
            out[ne] = {"trust": round(trustworthiness(X[sub], Y[sub], 15), 5),
                       "fit_ms": round(u.timings_["total_device"], 2)}
        return out

    Xt = prototype_mixture(N_FULL, D, seed=1000, proto_seed=0)
    sub = np.random.default_rng(0).choice(N_FULL, 10000, replace=False)
    curves = {init: trust_curve(Xt, init, LEARNED_EPOCHS, sub) for init in ("spectral", "learned")}
    Ytr = enc.transform(Xt)
    ref = curves["spectral"][500]["trust"]
    first = {tol: next((ne for ne in LEARNED_EPOCHS if curves["learned"][ne]["trust"] >= ref - tol), None)
             for tol in (0.005, 0.001)}
    Xf = prototype_mixture(20000, D, seed=2000, proto_seed=7)
    subf = np.random.default_rng(1).choice(20000, 5000, replace=False)
    fresh = {init: trust_curve(Xf, init, (100, 500), subf) for init in ("spectral", "learned")}
    return {"case": "learned_init", "metric": "trustworthiness@15 vs layout epochs", "unit": "trustworthiness",
            "config": {"workload": f"encoder {D}->512->512->2 trained on {LEARNED_TRAIN_SETS} x {LEARNED_TRAIN_N}x{D} "
                                   "prototype mixtures (shared prototypes, 200-epoch UMAP targets); evaluated on a "
                                   f"fresh {N_FULL}x{D} draw, 10K-row trustworthiness sample"},
            "train_s": round(train_s, 2), "encoder_step_ms": round(step_ms, 4),
            "encoder_step_note": "per training step of Encoder.fit on a device-resident 80000 x 784 set (batch "
                                 "gather, forward, backward, AdamW; per-epoch shuffle and loss read included)",
            "encoder_tflops": round(flops / (step_ms * 1e-3) / 1e12, 1),
            "curves": curves, "transform_only_trust": round(trustworthiness(Xt[sub], Ytr[sub], 15), 5),
            "spectral_500": ref,
            "learned_epochs_to_within": {str(k): v for k, v in first.items()},
            "epoch_fraction_within_0.005": None if first[0.005] is None else first[0.005] / 500,
            "unseen_prototypes": fresh}


def run_scale(args):
    """1,000,000 x 128 mixture of 100 anisotropic Gaussians (shared cluster parameters,
    param_seed 0): plain UMAP (NNDescent k=15, 200 epochs) timed per stage, then an
    encoder 128 -> 512 -> 512 -> 2 trained on 4 draws of 250,000 rows of the same
    distribution, learned against spectral init; trustworthiness@15 on a fixed
    20,000-row sample."""
    import torch

    from mlx_vis_b200 import UMAP
    from mlx_vis_b200.datasets import anisotropic_mixture
    from mlx_vis_b200.encoder import Encoder
    from mlx_vis_b200.metrics import trustworthiness

    n, d = 1_000_000, 128
    X = anisotropic_mixture(n, d, 100, seed=0, param_seed=0)
    Xd = torch.from_numpy(X).cuda()
    sub = np.random.default_rng(0).choice(n, 20000, replace=False)

    def fit(init, ne, enc=None):
        u = UMAP(n_epochs=ne, random_state=0, knn_method="nndescent", init=init, encoder=enc)
        Y = u.fit_transform_device(Xd)
        return u, Y.cpu().numpy()

    fit("spectral", 200)  # warm-up
    fits = [fit("spectral", 200) for _ in range(3)]
    u, Y = fits[-1]
    plain = {"fit_s": [round(f[0].timings_["total_device"] * 1e-3, 4) for f in fits],
             "stage_ms": {k: round(v, 2) for k, v in u.timings_.items() if not k.startswith("host_")},
             "n_edges": u.graph_info_["n_edges"], "trust": round(trustworthiness(X[sub], Y[sub], 15), 5)}
    t0 = time.perf_counter()
    Xs = [anisotropic_mixture(250_000, d, 100, seed=j, param_seed=0) for j in range(1, 5)]
    enc = Encoder.train_on_umap_runs(Xs, n_epochs=200, encoder_epochs=20, seed=0)
    train_s = time.perf_counter() - t0
    curves = {}
    for init in ("spectral", "learned"):
        curves[init] = {}
        for ne in (25, 50, 100, 200):
            uu, YY = fit(init, ne, enc)
            curves[init][ne] = {"trust": round(trustworthiness(X[sub], YY[sub], 15), 5),
                                "fit_ms": round(uu.timings_["total_device"], 1)}
    ref = curves["spectral"][200]["trust"]
    first = {str(tol): next((ne for ne in (25, 50, 100, 200) if curves["learned"][ne]["trust"] >= ref - tol), None)
             for tol in (0.005, 0.001)}
    return {"case": "scale", "config": {"workload": "UMAP fit_transform of a 1000000x128 mixture of 100 anisotropic "
                                                    "Gaussians (Dirichlet(2) sizes); NNDescent k=15, 200 epochs",
                                        "trust_sample": 20000},
            "plain": plain, "encoder_train_s": round(train_s, 2), "curves": curves,
            "learned_epochs_to_within": first, "transform_only_trust":
                round(trustworthiness(X[sub], enc.transform(X[sub]), 15), 5)}


def run_stage(args):
    """One untimed run of a single stage on its benchmark size, for profiler captures."""
    import torch

    from mlx_vis_b200 import _lib
    from mlx_vis_b200._nndescent.nndescent import NNDescent

    if args.case == "encoder":
        from mlx_vis_b200.datasets import prototype_mixture
        from mlx_vis_b200.encoder import Encoder

        Xe = torch.from_numpy(prototype_mixture(16384, D, seed=0)).cuda()
        Te = torch.randn((16384, 2), device="cuda")
        enc = Encoder(D, seed=0).fit([Xe], [Te], epochs=2)
        torch.cuda.synchronize()
        return {"case": "encoder", "steps": enc.step_count, "launches": _lib.kernel_launches()}
    if args.case == "knn_brute":
        from mlx_vis_b200.datasets import prototype_mixture

        Xd = torch.from_numpy(prototype_mixture(20000, D, seed=0)).cuda()
        idx, d2 = _lib.knn_brute(Xd, K_NN, extra=16)
        torch.cuda.synchronize()
        return {"case": "knn_brute", "n": 20000, "d": D, "k": K_NN, "launches": _lib.kernel_launches()}
    if args.case == "nndescent_1m":
        from mlx_vis_b200.datasets import anisotropic_mixture

        Xs = torch.from_numpy(anisotropic_mixture(1_000_000, 128, 100, seed=0, param_seed=0)).cuda()
        nn = NNDescent(k=K_NN, random_state=0)
        nn.build_device(Xs)
        torch.cuda.synchronize()
        return {"case": "nndescent_1m", "n": 1_000_000, "d": 128, "iterations": len(nn.history_),
                "launches": _lib.kernel_launches()}
    Xd = torch.from_numpy(make_data(args.n)).cuda()
    if args.case == "nndescent":
        nn = NNDescent(k=K_NN, random_state=0)
        nn.build_device(Xd)
        torch.cuda.synchronize()
        return {"case": "nndescent", "n": args.n, "iterations": len(nn.history_), "launches": _lib.kernel_launches()}
    from mlx_vis_b200 import UMAP

    UMAP(n_components=2, n_neighbors=K_NN, n_epochs=N_EPOCHS, knn_method="nndescent", random_state=0,
         use_graph=False).fit_transform_device(Xd)
    torch.cuda.synchronize()
    return {"case": "layout", "n": args.n, "launches": _lib.kernel_launches()}


def run_reference(args, rank):
    if rank != 0:
        return None
    for _ in range(max(args.warmup, 3)):
        cpu_baseline()
    vals, fits, stages = [], [], []
    t = time.perf_counter()
    for _ in range(args.steps):
        cb = cpu_baseline()
        vals.append(cb["value"])
        fits.append(cb["fit_s"])
        stages.append(cb["stage_s"])
    wall_ms = (time.perf_counter() - t) * 1e3 / args.steps
    fit_s = statistics.mean(fits)
    v = fit_sampler().updates_total / fit_s
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "edges/s", "n_gpus": 1, "steps": args.steps,
            "warmup": max(args.warmup, 3), "ms_per_step": round(fit_s * 1e3, 1), "fit_s": round(fit_s, 2),
            "sample_wall_ms_per_step": round(wall_ms, 1),
            "stage_s": {k: round(statistics.mean(s[k] for s in stages), 2) for k in stages[0]},
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "fp32",
            "data": "synthetic (seeded prototype mixture standing in for Fashion-MNIST)", "config": config(N_FULL),
            "cpu_baseline": {"value": v, "unit": "edges/s", "kind": "port", "cores": cb["cores"],
                             "sample": cb["sample"]},
            "e2e": {"value": v, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        out = run_reference(args, rank)
    elif args.case == "learned_init":
        out = run_learned_init(args) if rank == 0 else None
    elif args.case == "scale":
        out = run_scale(args) if rank == 0 else None
    elif args.case != "fit":
        out = run_stage(args) if rank == 0 else None
    else:
        out = run_ours(args, rank, world, local_rank)
    if out is not None and rank == 0:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
