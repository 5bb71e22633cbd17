#!/usr/bin/env python
"""Throughput of the Coulomb-integral path on one node: integrals/s of the FP32 form
(FP32 transforms, FP64 kernel/twiddles/reductions/round sum), every integral checked against
the all-FP64 plain path within max(1e-6 |I|, 1e-9 eV).

A step is one full request over one synthetic zinc-blende structure: pair densities, the
8-round convolution of every prepared density and the real-space reductions of every
requested integral (split-precision tensor-core Gram with FP64 accumulation).  `value` is the
device time (CUDA events) of one CUDA-graph replay of the prepared request per step, with the
inputs resident in HBM; `e2e` runs the public C ABI from pinned host buffers (coefficient and
cell upload, compute, result download) every step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2|c3|c1] [--impl ours|reference]

With N > 1 (torchrun) each rank computes an independent structure of the same size (seeded
by rank; structures are independent objects), so the work per GPU is fixed: weak scaling.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "c1": "zinc-blende 8x8x8 cells, 32^3 grid, 4096 atoms, 10 orbitals, 2e+2h, eeee,hhhh,ehhe,eheh",
    "c2": "zinc-blende 24x24x24 cells (lens-dot states), 96^3 grid, 110592 atoms, 20 orbitals, 6e+6h, "
          "eeee,hhhh,ehhe,eheh",
    "c3": "zinc-blende 64x64x64 cells, 256^3 grid, 2097152 atoms, 20 orbitals, 4e+4h, eeee,hhhh,ehhe,eheh",
    "c4": "zinc-blende 32x32x32 cells (lens-dot Hermite-Gaussian states), 128^3 grid, 262144 atoms, 20 orbitals, "
          "20e+20h, ijkl (all 2,560,000 integrals, 820 pair densities)",
    "c5": "16 independent zinc-blende structures, grids 48^3 ... 96x128x160 (13,824 ... 245,760 atoms), 20 "
          "orbitals, 4e+4h each, eeee,hhhh,ehhe,eheh (16 x 1024 integrals), one CUDA-graph launch per batch",
}
DIELECTRIC = 10.89


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c2", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cells", default=None,
                    help="Lx,Ly,Lz conventional cells instead of the workload's own box (a smaller case of the "
                         "same states and integral list, for profiler captures); the JSON line then names it")
    return ap.parse_args()


def cells_arg(args):
    return tuple(int(v) for v in args.cells.split(",")) if args.cells else None


def workload_name(args):
    if not args.cells:
        return WORKLOADS[args.config]
    L = cells_arg(args)
    return "%s states and integrals on a zinc-blende %dx%dx%d-cell box (%dx%dx%d grid, %d atoms)" % (
        args.config, L[0], L[1], L[2], 4 * L[0], 4 * L[1], 4 * L[2], 8 * L[0] * L[1] * L[2])


def dist_env():
    return (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
            int(os.environ.get("LOCAL_RANK", "0")))


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def peak_tflops_bf16():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            return float(json.load(fh)["bf16_tflops"])
    return 1590.0


def profiled_traffic(config, kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as fh:
        d = json.load(fh)
    return d.get(config, {}).get(kernel)


# ----------------------------------------------------------------------------------------
# clocks during the timed region
# ----------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_uuid=None):
        self.samples = []
        self.proc = None
        cmd = ["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits", "-lms", "50"]
        if device_uuid:
            cmd += ["-i", device_uuid]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) == 7:
                self.samples.append(parts)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for s in self.samples for k in range(4) if s[3 + k] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ----------------------------------------------------------------------------------------
# workload
# ----------------------------------------------------------------------------------------
def build_workload(config, seed_index=None, cells=None):
    from coulombo_lattice_b200 import synth
    import coulombo_lattice_b200 as cl
    d = synth.build(config, cells=cells, seed_index=seed_index)
    n = d["states"].shape[0]
    d["specs"] = np.ascontiguousarray(cl.enumerate_integrals(d["integrals"], n, d["holes"]))
    d["step"] = (synth.A_ZB / 4,) * 3
    return d


def gpu_local_cpus(device):
    """Host CPUs of the GPU's own NUMA node (sysfs local_cpulist of its PCI device), or None."""
    try:
        import torch
        pr = torch.cuda.get_device_properties(device)
        path = "/sys/bus/pci/devices/%04x:%02x:%02x.0/local_cpulist" % (pr.pci_domain_id, pr.pci_bus_id,
                                                                       pr.pci_device_id)
        with open(path) as fh:
            text = fh.read().strip()
        cpus = set()
        for part in text.split(","):
            lo, _, hi = part.partition("-")
            cpus.update(range(int(lo), int(hi or lo) + 1))
        cpus &= os.sched_getaffinity(0)
        return cpus or None
    except Exception:
        return None


def cpu_sample(d, n_left, threads):
    """The oracle's FP64 reference-structured loop (Planner order, 8-round prepare per left
    density, real-space calculate per right density) over the first n_left prepared
    densities; returns (seconds, integrals covered, integrals/s extrapolated to the request)."""
    from oracle import coulomb as C
    from oracle import host as H
    specs = [tuple(int(v) for v in s) for s in d["specs"]]
    n = d["states"].shape[0]
    plan = H.compute_plan(specs, n * (n + 1) // 2)
    lefts = sorted({s[1][0] for s in plan})
    chosen = set(lefts[:n_left])
    t0 = time.perf_counter()
    ghat = C.kernel_spectrum(C.kernel_octant(d["dims"], d["step"], DIELECTRIC), d["dims"])
    t_init = time.perf_counter() - t0

    def density(prod, conj):
        fl, fr = H.product_states(prod)
        rho = C.pair_density_atoms(d["states"][fl - 1], d["states"][fr - 1], conj)
        return C.scatter_density(rho, d["cells_idx"], d["dims"])

    t0 = time.perf_counter()
    covered = 0
    last_left, last_right, last_rc = -1, -1, None
    V = None
    for (sid, left, right) in plan:
        if left[0] not in chosen:
            continue
        if left[0] != last_left:
            V = C.prepare(density(left[0], False), ghat)
            last_left, last_right = left[0], -1
        rc = left[1] != right[1]
        if right[0] != last_right or rc != last_rc:
            C.calculate(V, density(right[0], rc))
            last_right, last_rc = right[0], rc
        covered += 1
    t_loop = time.perf_counter() - t0
    frac = len(chosen) / len(lefts)
    est_total = t_init + t_loop / frac
    return t_loop + t_init, covered, len(specs) / est_total, len(chosen), len(lefts)


def cpu_baseline_entry(d, budget_lefts, threads, kind="port"):
    secs, covered, ips, k, P = cpu_sample(d, budget_lefts, threads)
    return {"value": ips, "unit": "integrals/s", "cores": threads, "kind": kind,
            "sample": "CPU restatement (NumPy/SciPy pocketfft FP64, workers=%d), not the reference binary: "
                      "%d of %d prepared densities with their calculate() calls (%d integrals) in %.1f s, "
                      "extrapolated x%d/%d to the full request" % (threads, k, P, covered, secs, P, k)}


# ----------------------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------------------
def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    d = build_workload(args.config, cells=cells_arg(args))
    threads = os.cpu_count() or 1
    # one step's sample shrinks with the step count, so that --steps K --warmup W ends within a
    # few minutes (C2: about 0.9 s a step with one prepared density)
    n_left = {"c1": 2, "c2": 2, "c3": 1, "c4": 1}[args.config] if args.steps <= 20 else 1
    for _ in range(args.warmup):
        cpu_sample(d, n_left, threads)
    vals, secs = [], []
    for _ in range(args.steps):
        s, covered, ips, k, P = cpu_sample(d, n_left, threads)
        vals.append(ips)
        secs.append(s)
    value = float(np.median(vals))
    line = {
        "impl": "reference", "metric": "integrals/s", "value": value, "unit": "integrals/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * len(d["specs"]) / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_name(args), "integrals_per_step": int(len(d["specs"]))},
        "cpu_baseline": {"value": value, "unit": "integrals/s", "cores": threads, "kind": "port",
                         "sample": "each step: %d of %d prepared densities of the oracle's reference-structured "
                                   "FP64 loop, extrapolated to the full request; median of %d steps"
                                   % (n_left, P, args.steps)},
        "e2e": {"value": value, "unit": "integrals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_batch(args):
    """c5: 16 structures of uneven size as one graph-captured batch (cl_batch)."""
    import torch
    import coulombo_lattice_b200 as cl
    from coulombo_lattice_b200 import synth

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    step = (synth.A_ZB / 4,) * 3
    structs, calcs, reqs = [], [], []
    accuracy_worst = 0.0
    n_int_total = 0
    for i in range(len(synth.C5_CELLS)):
        d = synth.build_c5(i)
        n = d["states"].shape[0]
        specs = np.ascontiguousarray(cl.enumerate_integrals(d["integrals"], n, d["holes"]))
        plain = cl.CoulombCalculator(d["dims"], step, cl.MODE_FP64_PLAIN)
        plain.initialize(dielectric=DIELECTRIC)
        plain.set_states(d["states"], d["cells_idx"], d["holes"])
        v64 = plain.compute(specs)
        plain.close()
        cc = cl.CoulombCalculator(d["dims"], step, cl.MODE_FP32_FOURIER)
        cc.initialize(dielectric=DIELECTRIC)
        cc.set_states(d["states"], d["cells_idx"], d["holes"])
        r = cc.request(specs)
        v32 = r.run()
        err = np.abs(v32 - v64)
        accuracy_worst = max(accuracy_worst, float((err / np.maximum(1e-6 * np.abs(v64), 1e-9)).max()))
        structs.append((d, specs))
        calcs.append(cc)
        reqs.append(r)
        n_int_total += specs.shape[0]
    batch = cl.Batch(reqs)
    for _ in range(max(3, args.warmup)):
        batch.run()
    if world > 1:
        torch.distributed.barrier()
    ms = []
    for _ in range(args.steps):
        batch.run()
        ms.append(batch.last_ms())
    dev_ms = sum(ms)
    if world > 1:
        t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        dev_ms = float(t.item())
    ms_per_step = dev_ms / args.steps
    value = world * n_int_total / (ms_per_step / 1e3)
    # one eager pass per structure with per-kernel profiling for the roofline
    peak, peak_kind = measured_peaks()
    prof_tot = {}
    for cc, r in zip(calcs, reqs):
        cc.set_profiling(True)
        r.run()
        for k, v in cc.kernel_profile().items():
            a = prof_tot.setdefault(k, [0.0, 0, 0.0])
            a[0] += v[0]
            a[1] += v[1]
            a[2] += v[2]
        cc.set_profiling(False)
    fft = {k: v for k, v in prof_tot.items() if k in ("x_forward", "y_pass", "z_pass", "x_inverse")}
    dom = max(fft, key=lambda k: fft[k][0])
    line = {
        "metric": "integrals/s", "value": value, "unit": "integrals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOADS["c5"], "integrals_per_step": int(n_int_total),
                   "grids": [list(map(int, d["dims"])) for d, _ in structs]},
        "accuracy": {"worst_err_over_gate": accuracy_worst, "pass": accuracy_worst <= 1.0,
                     "gate": "max(1e-6|I|, 1e-9 eV) vs the all-FP64 plain path"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": fft[dom][2] / (fft[dom][0] / 1e3) / 1e9,
                     "peak": peak, "unit": "GB/s",
                     "frac": fft[dom][2] / (fft[dom][0] / 1e3) / 1e9 / peak, "peak_source": peak_kind,
                     "traffic": None, "note": "from one eager pass per structure"},
        "gpu_launches": int(sum(v[1] for v in prof_tot.values())),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    batch.close()
    for r in reqs:
        r.close()
    for cc in calcs:
        cc.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def run_ours(args):
    import torch
    import coulombo_lattice_b200 as cl

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    d = build_workload(args.config, seed_index=(int(args.config[1:]) + 1000 * rank) if rank else None,
                       cells=cells_arg(args))
    n = d["states"].shape[0]
    specs = d["specs"]
    n_int = specs.shape[0]

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        return float(t.item())

    # all-FP64 plain path: accuracy reference and the 1x point of the FP32/FP64 ratio
    plain = cl.CoulombCalculator(d["dims"], d["step"], cl.MODE_FP64_PLAIN)
    plain.initialize(dielectric=DIELECTRIC)
    plain.set_states(d["states"], d["cells_idx"], d["holes"])
    v64 = plain.compute(specs)
    # timed like the FP32 form: graph replays of the prepared request (best of 3)
    preq = plain.request(specs)
    pgraph64 = cl.Batch([preq])
    pgraph64.run()
    plain_ms = []
    for _ in range(3):
        pgraph64.run()
        plain_ms.append(pgraph64.last_ms())
    pgraph64.close()
    preq.close()
    plain.close()
    plain_ms = max_over_ranks(min(plain_ms))

    calc = cl.CoulombCalculator(d["dims"], d["step"], cl.MODE_FP32_FOURIER)
    t0 = time.perf_counter()
    calc.initialize(dielectric=DIELECTRIC)
    init_ms = 1e3 * (time.perf_counter() - t0)
    calc.set_states(d["states"], d["cells_idx"], d["holes"])
    for _ in range(max(3, args.warmup)):
        v32 = calc.compute(specs)

    err = np.abs(v32 - v64)
    lim = np.maximum(1e-6 * np.abs(v64), 1e-9)
    accuracy = {"max_rel_err": float(np.max(err / np.maximum(np.abs(v64), 1e-300))),
                "max_abs_err_eV": float(err.max()), "worst_err_over_gate": float((err / lim).max()),
                "gate": "max(1e-6|I|, 1e-9 eV) vs the all-FP64 plain path", "pass": bool(np.all(err <= lim))}

    # ---- timed region: resident inputs, one CUDA-graph replay of the prepared request per
    # step (pair densities, 8 rounds, reductions, results to pinned host), device time ---------
    req = calc.request(specs)
    v_req = req.run()
    if not np.allclose(v_req, v32, rtol=1e-9, atol=1e-15):
        raise RuntimeError("prepared-request results differ from cl_compute")
    graph = cl.Batch([req])
    for _ in range(max(3, args.warmup)):
        graph.run()
    uuid = None
    try:
        uuid = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        pass
    clocks = ClockSampler(uuid)
    barrier()
    wall0 = time.perf_counter()
    dev_ms = 0.0
    for _ in range(args.steps):
        graph.run()
        dev_ms += graph.last_ms()
    barrier()
    wall_ms = 1e3 * (time.perf_counter() - wall0)
    # per-kernel device times: the same request captured with a CUDA-event pair around every
    # launch, replayed for the same number of steps
    calc.set_profiling(True)
    pgraph = cl.Batch([req])
    pgraph.run()
    calc.set_profiling(False)
    calc.set_profiling(True)
    prof_dev_ms = 0.0
    for _ in range(args.steps):
        pgraph.run()
        prof_dev_ms += pgraph.last_ms()
    prof = calc.kernel_profile()
    calc.set_profiling(False)
    clock_info = clocks.stop()
    pgraph.close()
    graph.close()
    req.close()
    dev_ms = max_over_ranks(dev_ms)
    ms_per_step = dev_ms / args.steps
    value = world * n_int / (ms_per_step / 1e3)

    # ---- e2e: pinned host inputs through the C ABI ---------------------------------------
    # The host buffers are allocated and the calls made from the GPU's own NUMA node, so the
    # uploads do not cross the inter-socket link; the affinity is restored afterwards.
    saved_affinity = os.sched_getaffinity(0)
    local_cpus = gpu_local_cpus(local)
    if local_cpus:
        os.sched_setaffinity(0, local_cpus)
    coeff_h = torch.from_numpy(np.ascontiguousarray(d["states"]).view(np.float64).reshape(-1)).pin_memory()
    cells_h = torch.from_numpy(np.ascontiguousarray(d["cells_idx"], dtype=np.int64)).pin_memory()
    spec_h = torch.from_numpy(np.ascontiguousarray(specs, dtype=np.int16).reshape(-1)).pin_memory()
    out_h = torch.zeros(2 * n_int, dtype=torch.float64).pin_memory()
    h2d = coeff_h.numel() * 8 + cells_h.numel() * 8 + spec_h.numel() * 2
    d2h = out_h.numel() * 8
    def e2e_step():
        # one C-ABI call: coefficients and cells in (pinned host memory), integrals out; the
        # coefficient upload overlaps the transforms (cl_compute_states)
        calc.compute_states_raw(n, d["holes"], d["states"].shape[1], d["states"].shape[2], coeff_h.data_ptr(),
                                cells_h.data_ptr(), n_int, spec_h.data_ptr(), out_h.data_ptr())

    for _ in range(2):
        e2e_step()
    barrier()
    e0 = time.perf_counter()
    call_ms, call_dev_ms = [], []
    for _ in range(args.steps):
        c0 = time.perf_counter()
        e2e_step()
        call_ms.append(1e3 * (time.perf_counter() - c0))
        call_dev_ms.append(calc.timings()["total_ms"])  # first upload to last result, on the device
    barrier()
    e2e_ms = max_over_ranks(1e3 * (time.perf_counter() - e0) / args.steps)
    e2e_device_ms = call_dev_ms[-1]
    os.sched_setaffinity(0, saved_affinity)
    e2e_vals = out_h.numpy()[0::2] + 1j * out_h.numpy()[1::2]
    if not np.allclose(e2e_vals, v32, rtol=1e-9, atol=1e-15):
        raise RuntimeError("e2e results differ from the resident-input results")

    # ---- roofline of the dominant kernel --------------------------------------------------
    peak, peak_kind = measured_peaks()
    fft_classes = {k: v for k, v in prof.items() if k in ("x_forward", "y_pass", "z_pass", "x_inverse")}
    dom = max(fft_classes, key=lambda k: fft_classes[k][0])
    ms_k, launches_k, bytes_k = fft_classes[dom]
    achieved = bytes_k / (ms_k / 1e3) / 1e9
    traffic = profiled_traffic(args.config, dom)
    fft_ms = sum(v[0] for v in fft_classes.values())
    # FFT HBM-roofline %: sum of 2*M*s bytes over every 3D transform (8 forward + 8 inverse
    # per prepared density) / time of all transform passes / peak.
    M = int(np.prod(d["dims"]))
    plan_steps = cl.plan(n, specs)
    n_prepared = len({int(s[1]) for s in plan_steps})
    n_right = len({int(s[3]) for s in plan_steps})
    n_cells = int(np.unique(d["cells_idx"]).size)
    gram_tc = None
    if "gram" in prof and "gram_split" in prof:
        # split-precision Gram: 3 TF32 products of a (2 n_left) x (2 n_right) x atoms real GEMM;
        # the TF32 tensor rate is half the measured BF16 rate
        g_ms, g_launches, _ = prof["gram"]
        flops = 3 * 2.0 * (2 * n_prepared) * (2 * n_right) * n_cells * args.steps
        tf32_peak = peak_tflops_bf16() / 2
        gram_tc = {"bound": "tensor", "kernel": "gram", "achieved": flops / (g_ms / 1e3) / 1e12,
                   "peak": tf32_peak, "unit": "TFLOP/s", "frac": flops / (g_ms / 1e3) / 1e12 / tf32_peak,
                   "peak_source": "measured BF16 burst / 2 (TF32 rate)",
                   "flops_per_launch": flops / g_launches, "avg_launch_ms": g_ms / g_launches}
    fft_bytes = args.steps * 16 * n_prepared * 2.0 * M * 8
    buf_mb = n_prepared * M * 8 / 1e6
    total_launches = sum(v[1] for v in prof.values())

    line = {
        "metric": "integrals/s", "value": value, "unit": "integrals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": workload_name(args), "integrals_per_step": int(n_int),
                   "form": "FP32 transforms; FP64 kernel, twiddles, V accumulation and round sum; split-precision "
                           "(3xTF32) tensor-core reductions accumulated in FP64",
                   "l2": "inputs larger than L2 (126 MB): %.0f MB of transformed grids per request, "
                         "streamed in chunks" % buf_mb, "prepared_densities": n_prepared,
                   "init_ms_kernel_build": init_ms, "wall_ms_per_step": wall_ms / args.steps,
                   "timing": "device time (CUDA events) of one CUDA-graph replay of the prepared request per "
                             "step; per-kernel times from the same graph captured with an event pair around "
                             "every launch (%.3f ms per step)" % (prof_dev_ms / args.steps)},
        "accuracy": accuracy,
        "plain_fp64": {"value": world * n_int / (plain_ms / 1e3), "ms_per_step": plain_ms,
                       "timing": "device time of a CUDA-graph replay of the prepared request, best of 3",
                       "speedup_of_fp32_form": plain_ms / ms_per_step},
        "e2e": {"value": world * n_int / (e2e_ms / 1e3), "unit": "integrals/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms,
                "call": "cl_compute_states from pinned host buffers (coefficient upload overlapped with the "
                        "transforms), wall clock per call",
                "host_numa": ("calls and pinned buffers on the GPU's NUMA node (%d CPUs)" % len(local_cpus)
                              if local_cpus else "GPU NUMA node unknown: default affinity"),
                "device_ms_last_call": e2e_device_ms,
                "call_ms": {"min": min(call_ms), "median": statistics.median(call_ms), "max": max(call_ms)},
                "call_device_ms": {"min": min(call_dev_ms), "median": statistics.median(call_dev_ms),
                                   "max": max(call_dev_ms)}},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_kind,
                     "traffic": traffic, "algorithmic_bytes_per_launch": bytes_k / launches_k,
                     "avg_launch_ms": ms_k / launches_k},
        "kernels": {k: {"ms": v[0] / args.steps, "launches": v[1] // args.steps,
                        "GBps": (v[2] / (v[0] / 1e3) / 1e9) if v[0] > 0 else None} for k, v in prof.items()},
        "fft_share_of_step": fft_ms / (dev_ms if world == 1 else fft_ms + 1e-30),
        "fft_hbm_roofline": {"frac": fft_bytes / (fft_ms / 1e3) / 1e9 / peak,
                             "transforms_per_density": 16, "bytes_per_transform": "2*M*8 (FP32 complex)"},
        "gram_tensor_roofline": gram_tc,
        "autotune": [ln for ln in cl.autotune_report().splitlines()
                     if "fp32 %dx%dx%d:" % tuple(d["dims"]) in ln],
        "gpu_launches": int(total_launches),
        "clocks": clock_info,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        n_left = {"c1": 2, "c2": 4, "c3": 1, "c4": 1}[args.config]
        line["cpu_baseline"] = cpu_baseline_entry(d, n_left, threads)
    if rank == 0:
        print(json.dumps(line), flush=True)
    calc.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.config == "c5":
        run_batch(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
