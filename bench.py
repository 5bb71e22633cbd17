#!/usr/bin/env python
"""Throughput of the Coulomb-integral path on one node: integrals/s of the FP32 form, every
integral checked against the all-FP64 plain path within max(1e-6 |I|, 1e-9 eV), and a bounded
sample of integrals against the FP64 oracle.

A step is one full request over one synthetic zinc-blende structure: pair densities, the
convolution of every prepared density and the real-space reductions of every requested
integral (split-precision tensor-core Gram with FP64 accumulation).  `value` is the device
time (CUDA events) of one CUDA-graph replay of the prepared request per step, with the inputs
resident in HBM; `e2e` runs the public C ABI from pinned host buffers (coefficient and cell
upload, compute, result download) every step.  The default workload is the 2.1M-atom box
(64^3 zinc-blende cells, 256^3 grid, 20 orbitals, 4 e + 4 h, 1,024 integrals).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--config c1|c2|c3|c4|c5] [--impl ours|reference]

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
HEADLINE_MODE = 3  # coulombo_lattice_b200.MODE_FP32_SUBLATTICE
FORM_TEXT = {
    0: "all-FP64: 8 rounds of N-point FFTs (the reference's method), FP64 Gram",
    1: "FP32 transforms in 8 rounds; FP64 kernel, twiddles, V accumulation and round sum; split-precision "
       "(3xTF32) tensor-core reductions accumulated in FP64 (FP64 reductions under 65,536 atoms)",
    2: "all-FP64 sub-lattice decomposition (exact): per residue class of the atoms' grid points, zero-padded "
       "(2n/m)^3 transforms and one class-mixing step per frequency; FP64 Gram",
    3: "sub-lattice decomposition with FP32 transforms; FP64 kernel spectrum, class kernels and phases built in "
       "FP64 and rounded once; split-precision (3xTF32) tensor-core reductions accumulated in FP64 (FP64 "
       "tensor-core reductions under 65,536 atoms)",
}
FORM_KEYS = {0: "fp64_rounds", 1: "fp32_rounds", 2: "fp64_sublattice", 3: "fp32_sublattice"}
# kernel classes bound by HBM (the tensor-core Gram is reported against the tensor rate)
HBM_CLASSES = ("pair_density", "x_forward", "y_pass", "z_pass", "x_inverse", "gram_split", "round_sum")
TRANSFORM_CLASSES = ("x_forward", "y_pass", "z_pass", "x_inverse")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--split", default="densities", choices=["densities", "structures"],
                    help="N > 1: one request split by left densities over the ranks with one all-reduce of the "
                         "integrals (strong scaling), or one independent structure per rank (weak scaling)")
    ap.add_argument("--profile", action="store_true",
                    help="profiler runs: only the headline form's timed replays (inside an NVTX range 'timed'); "
                         "no other forms, no e2e, no CPU baseline -- the line is not a bench result")
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
def build_workload(config, seed_index=None, cells=None, with_library=True):
    """Synthetic structure, states and integral list.  The reference arm enumerates the
    integrals with the oracle's restatement of Pattern (with_library=False), so that its
    process never loads this repository's library."""
    from coulombo_lattice_b200 import synth
    d = synth.build(config, cells=cells, seed_index=seed_index)
    n = d["states"].shape[0]
    if with_library:
        import coulombo_lattice_b200 as cl
        d["specs"] = np.ascontiguousarray(cl.enumerate_integrals(d["integrals"], n, d["holes"]))
    else:
        from oracle import host as H
        d["specs"] = np.array(H.enumerate_integrals(H.Pattern(d["integrals"], d["holes"]), n),
                              dtype=np.int16).reshape(-1, 4)
    d["step"] = (synth.A_ZB / 4,) * 3
    return d


def config_of(args, n_int):
    """The `config` object of both arms' JSON lines (identical by construction)."""
    return {"workload": workload_name(args), "integrals_per_step": int(n_int)}


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


class OracleLoop:
    """The oracle's FP64 restatement of the reference's integral loop, structured like the
    reference (coulombo.cpp:186-209): in plan order, a dense zeroed pair-density grid per
    product (Product.cpp:16-30), 8 rounds of N-point FFTs per new left density
    (CoulombCalculator.cpp:105-163) and a dense sum over the grid per right density
    (CoulombCalculator.cpp:165-172).  SciPy's pocketfft runs on every host thread.

    Large integral lists (more than 50,000) are planned over the integrals of their first two
    left products only, which is all a bounded sample reaches."""

    def __init__(self, d):
        from oracle import coulomb as C
        from oracle import host as H
        self.C, self.H, self.d = C, H, d
        specs = d["specs"]
        n = d["states"].shape[0]
        ids = np.arange(len(specs))
        if len(specs) > 50000:
            lp = np.array([H.product_of(int(a), int(b))[0] for a, b in zip(specs[:, 0], specs[:, 3])])
            keep = np.isin(lp, np.unique(lp)[:2])
            ids = ids[keep]
        sub = [tuple(int(v) for v in specs[i]) for i in ids]
        plan = H.compute_plan(sub, n * (n + 1) // 2)
        self.groups = []  # [(left, [(spec id, left, right), ...])] in plan order
        for (sid, left, right) in plan:
            if not self.groups or self.groups[-1][0] != left[0]:
                self.groups.append((left[0], []))
            self.groups[-1][1].append((int(ids[sid]), left, right))
        t0 = time.perf_counter()
        self.ghat = C.kernel_spectrum(C.kernel_octant(d["dims"], d["step"], DIELECTRIC), d["dims"])
        self.init_s = time.perf_counter() - t0
        self.next_group = 0

    def _density(self, prod, conj):
        fl, fr = self.H.product_states(prod)
        rho = self.C.pair_density_atoms(self.d["states"][fl - 1], self.d["states"][fr - 1], conj)
        return self.C.scatter_density(rho, self.d["cells_idx"], self.d["dims"])

    def run(self, budget_s=None, groups=1):
        """Runs the next `groups` left densities (cycling) with all their steps, or stops after
        the step that crosses budget_s.  Returns (seconds, {spec id: value})."""
        C = self.C
        values = {}
        t0 = time.perf_counter()
        for _ in range(groups):
            left, steps = self.groups[self.next_group % len(self.groups)]
            self.next_group += 1
            V = C.prepare(self._density(left, False), self.ghat)
            last_right, last_rc, val = -1, None, 0j
            for (sid, lf, right) in steps:
                rc = lf[1] != right[1]
                if right[0] != last_right or rc != last_rc:
                    val = C.calculate(V, self._density(right[0], rc))
                    last_right, last_rc = right[0], rc
                values[sid] = np.conj(val) if lf[1] else val
                if budget_s is not None and time.perf_counter() - t0 > budget_s:
                    return time.perf_counter() - t0, values
        return time.perf_counter() - t0, values


def accuracy_vs_oracle(values, got, fp64):
    """Worst error over the gate of `got` (full integral vector) on the oracle's sample."""
    ids = np.array(sorted(values), dtype=np.int64)
    want = np.array([values[i] for i in ids])
    err = np.abs(got[ids] - want)
    lim = (1e-10 * np.abs(want) + 1e-16) if fp64 else np.maximum(1e-6 * np.abs(want), 1e-9)
    return {"integrals": int(len(ids)), "worst_err_over_gate": float((err / lim).max()),
            "max_abs_err_eV": float(err.max()),
            "max_rel_err": float((err / np.maximum(np.abs(want), 1e-300)).max()), "pass": bool(np.all(err <= lim)),
            "gate": "1e-10 relative" if fp64 else "max(1e-6 |I|, 1e-9 eV)"}


# ----------------------------------------------------------------------------------------
# arms
# ----------------------------------------------------------------------------------------
def run_reference(args):
    """The reference's CPU path on the host cores: the oracle's reference-structured FP64 loop
    (no repository library is loaded).  One step = the next prepared left density with all of
    its calculate() calls; value = integrals computed / seconds over the timed steps."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    threads = len(os.sched_getaffinity(0))
    if args.config == "c5":
        # the sixteen structures in turn, one left density of the next structure per step
        from coulombo_lattice_b200 import synth
        loops, n_req = [], 0
        for i in range(len(synth.C5_CELLS)):
            dd = synth.build_c5(i)
            from oracle import host as H
            dd["specs"] = np.array(H.enumerate_integrals(H.Pattern(dd["integrals"], dd["holes"]),
                                                         dd["states"].shape[0]), dtype=np.int16).reshape(-1, 4)
            dd["step"] = (synth.A_ZB / 4,) * 3
            n_req += len(dd["specs"])
            loops.append(OracleLoop(dd))
        budget = None
    else:
        d = build_workload(args.config, cells=cells_arg(args), with_library=False)
        n_req = len(d["specs"])
        loops = [OracleLoop(d)]
        budget = {"c4": 8.0}.get(args.config)  # a C4 left density has ~3,200 dense steps
    k = 0
    for _ in range(args.warmup):
        loops[k % len(loops)].run(budget)
        k += 1
    secs, covered = [], 0
    for _ in range(args.steps):
        s, vals = loops[k % len(loops)].run(budget)
        k += 1
        secs.append(s)
        covered += len(vals)
    loop = loops[0]
    value = covered / sum(secs)
    line = {
        "impl": "reference", "metric": "integrals/s", "value": value, "unit": "integrals/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_of(args, n_req),
        "cpu_baseline": {"value": value, "unit": "integrals/s", "cores": threads, "kind": "port",
                         "sample": "the oracle's FP64 restatement of the reference's loop (dense pair-density grids, "
                                   "8 rounds of SciPy pocketfft FFTs on %d threads per left density, dense calculate "
                                   "per step), not the reference binary (MPI/FFTW/Armadillo are not installed): each "
                                   "step is the next of %d left densities%s, %d integrals in %.1f s over %d steps; the "
                                   "one-time kernel spectrum (%.2f s) is excluded like the GPU arm's"
                                   % (threads, sum(len(lp.groups) for lp in loops),
                                      " (cut at %.0f s)" % budget if budget else "", covered, sum(secs), args.steps,
                                      sum(lp.init_s for lp in loops))},
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
        cc = cl.CoulombCalculator(d["dims"], step, HEADLINE_MODE)
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
        "config": config_of(args, n_int_total),
        "details": {"grids": [list(map(int, d["dims"])) for d, _ in structs], "form": FORM_TEXT[HEADLINE_MODE]},
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


def run_sharded(args):
    """N > 1 GPUs on one request: rank r runs shard r of the plan's left densities (a prepared
    request of cl_request_create_shard, replayed as a CUDA graph), then one NCCL all-reduce (sum,
    FP64) of the integral vector.  A step is both; its time is the max over ranks of the device
    time of the replay plus the all-reduce (CUDA events).  The total work is fixed: strong scaling.
    e2e: every rank uploads the coefficients from pinned host memory (cl_set_states) and computes
    its shard (cl_compute_shard); the all-reduced integrals come back to the host."""
    import datetime
    import torch
    import torch.distributed as dist
    import coulombo_lattice_b200 as cl

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    d = build_workload(args.config, cells=cells_arg(args))  # the same structure on every rank
    n = d["states"].shape[0]
    specs = d["specs"]
    n_int = specs.shape[0]
    calc = cl.CoulombCalculator(d["dims"], d["step"], HEADLINE_MODE)
    calc.initialize(dielectric=DIELECTRIC)
    calc.set_states(d["states"], d["cells_idx"], d["holes"])
    full = calc.compute(specs)
    req = calc.request(specs, rank, world)
    calc.set_profiling(True)
    req.run()
    launches_per_step = sum(v[1] for v in calc.kernel_profile().values())
    calc.set_profiling(False)
    graph = cl.Batch([req])
    vec = torch.zeros(2 * n_int, dtype=torch.float64, device="cuda")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def step():
        part = graph.run()[0]
        dev = graph.last_ms()
        vec.copy_(torch.from_numpy(np.ascontiguousarray(part).view(np.float64)), non_blocking=False)
        ev0.record()
        dist.all_reduce(vec, op=dist.ReduceOp.SUM)
        ev1.record()
        ev1.synchronize()
        return dev + ev0.elapsed_time(ev1)

    for _ in range(max(3, args.warmup)):
        step()
    got = vec.cpu().numpy().view(np.complex128)
    if not np.allclose(got, full, rtol=1e-9, atol=1e-15):
        raise RuntimeError("sharded integrals differ from the single-GPU request")
    torch.cuda.synchronize()
    dist.barrier()
    dev_ms = sum(step() for _ in range(args.steps))
    t = torch.tensor([dev_ms], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_per_step = float(t.item()) / args.steps
    graph.close()
    req.close()
    # e2e through the C ABI from pinned host buffers
    coeff_h = torch.from_numpy(np.ascontiguousarray(d["states"]).view(np.float64).reshape(-1)).pin_memory()
    cells_h = torch.from_numpy(np.ascontiguousarray(d["cells_idx"], dtype=np.int64)).pin_memory()
    spec_h = torch.from_numpy(np.ascontiguousarray(specs, dtype=np.int16).reshape(-1)).pin_memory()
    out_h = torch.zeros(2 * n_int, dtype=torch.float64).pin_memory()

    def e2e_step():
        calc.set_states_raw(n, d["holes"], d["states"].shape[1], d["states"].shape[2], coeff_h.data_ptr(),
                            cells_h.data_ptr())
        calc.compute_raw_shard(n_int, spec_h.data_ptr(), rank, world, out_h.data_ptr())
        vec.copy_(out_h, non_blocking=False)
        dist.all_reduce(vec, op=dist.ReduceOp.SUM)
        out_h.copy_(vec, non_blocking=False)

    e2e_step()
    torch.cuda.synchronize()
    dist.barrier()
    e0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    torch.cuda.synchronize()
    dist.barrier()
    e2e_ms = 1e3 * (time.perf_counter() - e0) / args.steps
    t = torch.tensor([e2e_ms], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
    line = {
        "metric": "integrals/s", "value": n_int / (ms_per_step / 1e3), "unit": "integrals/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_of(args, n_int),
        "details": {"form": FORM_TEXT[HEADLINE_MODE], "split": "left densities dealt round-robin over the ranks "
                    "(cl_request_create_shard), one NCCL all-reduce (sum, FP64) of the integral vector per step",
                    "timing": "max over ranks of the device time of the shard's graph replay plus the all-reduce "
                              "(CUDA events)"},
        "e2e": {"value": n_int / (e2e_ms / 1e3), "unit": "integrals/s",
                "h2d_bytes_per_step": int(coeff_h.numel() * 8 + cells_h.numel() * 8 + spec_h.numel() * 2),
                "d2h_bytes_per_step": int(out_h.numel() * 8), "ms_per_step": e2e_ms,
                "call": "per rank: cl_set_states + cl_compute_shard from pinned host buffers, all-reduce, "
                        "integrals back to the host; wall clock, max over ranks"},
        "gpu_launches": int(launches_per_step * args.steps),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    calc.close()
    dist.barrier()
    dist.destroy_process_group()



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

    def time_form(mode):
        """Values and device ms per request (graph replay of the prepared request, best of 3)."""
        cc = cl.CoulombCalculator(d["dims"], d["step"], mode)
        cc.initialize(dielectric=DIELECTRIC)
        cc.set_states(d["states"], d["cells_idx"], d["holes"])
        vals = cc.compute(specs)
        r = cc.request(specs)
        g = cl.Batch([r])
        g.run()
        ms = []
        for _ in range(3):
            g.run()
            ms.append(g.last_ms())
        info = cc.form_info()
        g.close()
        r.close()
        cc.close()
        return vals, max_over_ranks(min(ms)), info

    # the all-FP64 8-round path: accuracy reference and the 1x point of the FP32/FP64 ratio; the
    # other forms timed alike, to separate what the decomposition and the precision each give
    v64, plain_ms, _ = time_form(cl.MODE_FP64_PLAIN) if not args.profile else (None, float("nan"), None)
    other_forms = {}
    for mode in ([] if args.profile else cl.ALL_MODES):
        if mode in (cl.MODE_FP64_PLAIN, HEADLINE_MODE):
            continue
        vals, ms, info = time_form(mode)
        err = np.abs(vals - v64)
        if cl.mode_is_fp64(mode):
            lim = 1e-10 * np.abs(v64) + 1e-16
        else:
            lim = np.maximum(1e-6 * np.abs(v64), 1e-9)
        other_forms[FORM_KEYS[mode]] = {"ms_per_step": ms, "value": world * n_int / (ms / 1e3),
                                        "speedup_vs_fp64_rounds": plain_ms / ms,
                                        "worst_err_over_gate_vs_fp64_rounds": float((err / lim).max()),
                                        "sublattice": info["sublattice"], "form": FORM_TEXT[mode]}

    calc = cl.CoulombCalculator(d["dims"], d["step"], HEADLINE_MODE)
    t0 = time.perf_counter()
    calc.initialize(dielectric=DIELECTRIC)
    init_ms = 1e3 * (time.perf_counter() - t0)
    calc.set_states(d["states"], d["cells_idx"], d["holes"])
    form_info = calc.form_info()
    for _ in range(max(3, args.warmup)):
        v32 = calc.compute(specs)

    if v64 is None:
        v64 = v32
    err = np.abs(v32 - v64)
    lim = np.maximum(1e-6 * np.abs(v64), 1e-9)
    accuracy = {"vs_plain_fp64": {
        "integrals": int(n_int), "max_rel_err": float(np.max(err / np.maximum(np.abs(v64), 1e-300))),
        "max_abs_err_eV": float(err.max()), "worst_err_over_gate": float((err / lim).max()),
        "gate": "max(1e-6|I|, 1e-9 eV) vs the all-FP64 plain path on every integral",
        "pass": bool(np.all(err <= lim))}}

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
    torch.cuda.nvtx.range_push("timed")
    wall0 = time.perf_counter()
    dev_ms = 0.0
    for _ in range(args.steps):
        graph.run()
        dev_ms += graph.last_ms()
    barrier()
    torch.cuda.nvtx.range_pop()
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
    if not args.profile:
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
    else:
        local_cpus, h2d, d2h = None, 0, 0
        e2e_ms = e2e_device_ms = float("nan")
        call_ms = call_dev_ms = [float("nan")]

    # ---- the integral files (coulombo.cpp:213-262), written on the host threads -----------
    import tempfile
    with tempfile.TemporaryDirectory() as td:
        t0 = time.perf_counter()
        cl.write_integrals(os.path.join(td, ""), d["holes"], n - d["holes"], specs, v32)
        export_ms = 1e3 * (time.perf_counter() - t0)

    # ---- roofline of the dominant kernel --------------------------------------------------
    peak, peak_kind = measured_peaks()
    fft_classes = {k: v for k, v in prof.items() if k in TRANSFORM_CLASSES}
    hbm_classes = {k: v for k, v in prof.items() if k in HBM_CLASSES}
    dom = max(hbm_classes, key=lambda k: hbm_classes[k][0])
    ms_k, launches_k, bytes_k = hbm_classes[dom]
    achieved = bytes_k / (ms_k / 1e3) / 1e9
    traffic = profiled_traffic(args.config, dom)
    fft_ms = sum(v[0] for v in fft_classes.values())
    fft_alg_bytes = sum(v[2] for v in fft_classes.values())
    # FFT HBM-roofline %: sum of 2*M*s bytes over every 3D transform (8 forward + 8 inverse
    # per prepared density) / time of all transform passes / peak.
    M = int(np.prod(d["dims"]))
    plan_steps = cl.plan(n, specs)
    n_prepared = len({int(s[1]) for s in plan_steps})
    n_right = len({int(s[3]) for s in plan_steps})
    n_cells = int(np.unique(d["cells_idx"]).size)
    gram_tc = None
    if "gram" in prof and n_cells >= 65536:
        # split-precision Gram (fused, or after the split pass): 3 TF32 products of a
        # (2 n_left) x (2 n_right) x atoms real GEMM; the TF32 tensor rate is half the measured
        # BF16 rate
        g_ms, g_launches, _ = prof["gram"]
        flops = 3 * 2.0 * (2 * n_prepared) * (2 * n_right) * n_cells * args.steps
        tf32_peak = peak_tflops_bf16() / 2
        gram_tc = {"bound": "tensor", "kernel": "gram", "achieved": flops / (g_ms / 1e3) / 1e12,
                   "peak": tf32_peak, "unit": "TFLOP/s", "frac": flops / (g_ms / 1e3) / 1e12 / tf32_peak,
                   "peak_source": "measured BF16 burst / 2 (TF32 rate)",
                   "flops_per_launch": flops / g_launches, "avg_launch_ms": g_ms / g_launches}
    if form_info["sublattice"]:
        pts = form_info["classes"] * form_info["lengths"][0] * form_info["lengths"][1] * (
            form_info["lengths"][2] // 2)
        buf_mb = n_prepared * pts * 8 / 1e6
    else:
        buf_mb = n_prepared * M * 8 / 1e6
    total_launches = sum(v[1] for v in prof.values())

    line = {
        "metric": "integrals/s", "value": value, "unit": "integrals/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": config_of(args, n_int),
        "details": {"form": FORM_TEXT[HEADLINE_MODE], "form_info": form_info,
                    "export_ms": export_ms,
                    "export": "cl_write_integrals of the request's %d integrals (the XXXX.txt files), wall clock, "
                              "outside value and e2e" % n_int,
                    "l2": "inputs larger than L2 (126 MB): %.0f MB of transformed grids per request, "
                          "streamed in chunks" % buf_mb, "prepared_densities": n_prepared,
                    "init_ms_kernel_build": init_ms, "wall_ms_per_step": wall_ms / args.steps,
                    "timing": "device time (CUDA events) of one CUDA-graph replay of the prepared request per "
                              "step; per-kernel times from the same graph captured with an event pair around "
                              "every launch (%.3f ms per step)" % (prof_dev_ms / args.steps)},
        "accuracy": accuracy,
        "plain_fp64": {"value": world * n_int / (plain_ms / 1e3), "ms_per_step": plain_ms,
                       "form": FORM_TEXT[cl.MODE_FP64_PLAIN],
                       "timing": "device time of a CUDA-graph replay of the prepared request, best of 3",
                       "speedup_of_fp32_form": plain_ms / ms_per_step},
        "other_forms": other_forms,
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
        "fft_hbm_roofline": {"frac": fft_alg_bytes / (fft_ms / 1e3) / 1e9 / peak,
                             "achieved_GBps": fft_alg_bytes / (fft_ms / 1e3) / 1e9,
                             "definition": "algorithmic bytes of every transform-pass launch (x, y, z passes) / "
                                           "their summed device time / measured HBM peak"},
        "gram_tensor_roofline": gram_tc,
        "autotune": [ln for ln in cl.autotune_report().splitlines()
                     if ln.split(":")[0].split(" ", 1)[1].startswith("fp32")],
        "gpu_launches": int(total_launches),
        "clocks": clock_info,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not args.profile:
        # the oracle's reference-structured FP64 loop on a bounded sample (about 20 s) of this
        # workload's left densities: the CPU baseline, and the per-integral check of both forms
        loop = OracleLoop(d)
        budget = {"c1": 5.0}.get(args.config, 20.0)
        secs, vals = 0.0, {}
        while secs < budget and loop.next_group < len(loop.groups):
            s_, v_ = loop.run(budget - secs)
            secs += s_
            vals.update(v_)
        threads = len(os.sched_getaffinity(0))
        line["cpu_baseline"] = {
            "value": len(vals) / secs, "unit": "integrals/s", "cores": threads, "kind": "port",
            "sample": "the oracle's FP64 restatement of the reference's loop (dense pair-density grids, 8 rounds of "
                      "SciPy pocketfft FFTs on %d threads, dense calculate per step), not the reference binary: "
                      "%d of the request's %d integrals (%d left densities) in %.1f s, not extrapolated"
                      % (threads, len(vals), n_int, loop.next_group, secs)}
        line["accuracy"]["vs_oracle"] = {"fp32_form": accuracy_vs_oracle(vals, v32, False),
                                         "plain_fp64": accuracy_vs_oracle(vals, v64, True)}
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
    elif dist_env()[1] > 1 and args.split == "densities":
        run_sharded(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
