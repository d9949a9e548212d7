#!/usr/bin/env python
"""Throughput benchmark of the batched GFN2-xTB energy+forces path.

Workload: the 4096-system ragged batch of hetero-alkane chains (C3..C40,
10 % of interior CH2 replaced by O or NH, seed 1), GFN2-xTB energy + analytic
forces + Mulliken charges to SCC convergence (charge 1e-6, energy 1e-8, 300 K,
Broyden 8/0.4).  One step = one ``xtbloom_compute`` call over the whole batch.

Two execution forms are timed on the same batch: FP64 throughout (the
headline ``value``) and split precision (3xTF32 tensor-core GEMMs until a
system's residual is below 1e-5, then FP64), with the largest difference of
every output between them.

  python bench.py [--gpus N --steps K --warmup W]        # this library (CUDA)
  python bench.py --impl reference [...]                 # reference CPU library

``value`` is measured with positions and outputs resident in HBM; ``e2e`` is
the same call with host positions and host outputs (the library's own
host<->device copies inside the timed region).  Multi-GPU runs shard the
independent systems (each rank its own 4096-system batch, no collective in
the data path) and report the whole-job throughput from the slowest rank.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

from xtbloom_b200 import abi  # noqa: E402
from xtbloom_b200 import workloads as W  # noqa: E402

METRIC = ("GFN2 E+F systems/s on 1 B200: mixed vs FP64 path at |ΔE|≤1e-6 Eh; roofline %")
STAGES = ["setup_integrals", "lowdin", "potential", "fock", "gemm_transform", "tridiag", "eigvals",
          "inverse_iteration", "backtransform", "gemm_density", "mulliken", "energy_mixer",
          "compact", "force_pairs", "classical", "cn_chain", "publish", "refine"]
# DRAM bytes per algorithmic byte of the Householder tridiagonalisation,
# measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum of
# k_tridiag_smem on 512 systems of this workload: 6.38 MB read, 0 written,
# for 6.38 MB of matrices read once): the kernel reads each matrix once.
TRIDIAG_DRAM_PER_ALG_BYTE = 1.0
REF_LIB = ROOT / "oracle" / "_ref" / "libxtbloom_ref.so"
WORKLOAD = ("GFN2-xTB E+F+q, ragged batch of 4096 hetero-alkane chains C_nH_(2n+2), n uniform "
            "in 3..40, 10% interior CH2 -> O/NH, seed 1; SCC 1e-6/1e-8, 300 K, Broyden 8/0.4")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--systems", type=int, default=4096)
    p.add_argument("--cpu-sample", type=int, default=192)
    p.add_argument("--cpu-sample-1t", type=int, default=24,
                   help="systems of the single-thread CPU baseline sample")
    p.add_argument("--no-gfn1", action="store_true", help="skip the GFN1 radical-batch line")
    p.add_argument("--no-autograd", action="store_true", help="skip the point-charge autograd line")
    p.add_argument("--no-water", action="store_true", help="skip the water-cluster line")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--form", default="both", choices=["both", "mixed", "fp64"])
    p.add_argument("--graphs", type=int, default=1)
    p.add_argument("--once", action="store_true",
                   help="one device-resident call of the chosen form and exit (profiler runs)")
    p.add_argument("--indices", default="",
                   help="with --once: comma-separated systems of the 4096-system batch to run "
                        "(e.g. the slowly converging ones, for profiles of the few-system regime)")
    p.add_argument("--workload", default="hetero", choices=["hetero", "water", "radicals"],
                   help="with --once: the batch to run (hetero: --systems hetero-alkanes; water: "
                        "--systems water clusters of 600-1200 AOs; radicals: --systems GFN1 radicals)")
    return p.parse_args()


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x: float, world: int) -> float:
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def fetch(lib, name, cap=256):
    f = lib.lib.xtbloom_b200_debug_fetch
    f.restype = C.c_int32
    f.argtypes = [C.c_void_p, C.c_char_p, C.c_int64, C.POINTER(C.c_double), C.c_size_t,
                  C.POINTER(C.c_size_t)]
    out = np.zeros(cap)
    cnt = C.c_size_t()
    f(lib.ctx, name.encode(), 0, out.ctypes.data_as(C.POINTER(C.c_double)), cap, C.byref(cnt))
    return out[:cnt.value].copy()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    def __init__(self, device: int):
        self.path = Path(tempfile.gettempdir()) / f"xtb_clocks_{os.getpid()}.csv"
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={device}", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        rows = []
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                rows.append(parts)
        self.path.unlink(missing_ok=True)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        sm = [float(r[0]) for r in rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def stage_work(n: np.ndarray, iters: np.ndarray, nocc: np.ndarray) -> dict:
    """Algorithmic FP64 flops and HBM bytes per stage over one step (all systems)."""
    n = n.astype(float)
    it = iters.astype(float)
    m = nocc.astype(float)
    d8 = 8.0
    return {
        "gemm_transform": {"flops": float(np.sum(it * 4 * n ** 3)), "bytes": float(np.sum(it * 6 * n * n * d8))},
        "tridiag": {"flops": float(np.sum((it + 1) * 4 / 3 * n ** 3)), "bytes": float(np.sum((it + 1) * 2 * n * n * d8))},
        "backtransform": {"flops": float(np.sum(it * 2 * n * n * m)), "bytes": float(np.sum(it * 3 * n * m * d8))},
        "gemm_density": {"flops": float(np.sum(it * 4 * n * n * m)), "bytes": float(np.sum(it * (3 * n * n + 2 * n * m) * d8))},
        "fock": {"flops": float(np.sum(it * 22 * n * n)), "bytes": float(np.sum(it * 12 * n * n * d8))},
        "mulliken": {"flops": float(np.sum(it * 22 * n * n)), "bytes": float(np.sum(it * 11 * n * n * d8))},
    }


def load_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def reference_sample(batch, count: int):
    idx = np.linspace(0, batch.batch_size - 1, count).round().astype(int)
    return W.subset(batch, idx), idx


def cpu_run(sample, threads: int = 0, repeats: int = 3) -> tuple[float, dict]:
    """Median wall time of `repeats` calls on the sample, after one equal
    warm-up call (the reference arm's protocol)."""
    lib = abi.Library(str(REF_LIB), backend=abi.BACKEND_CPU, cpu_threads=threads)
    out = lib.compute(sample)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        out = lib.compute(sample)
        times.append(time.perf_counter() - t0)
    lib.close()
    return statistics.median(times), out


def host_cores() -> int:
    try:
        return min(len(os.sched_getaffinity(0)), 64)
    except AttributeError:
        return min(os.cpu_count() or 1, 64)


def run_reference(args, world, rank):
    if rank != 0:
        return
    if not REF_LIB.exists():
        print(json.dumps({"impl": "reference",
                          "unavailable": "oracle/_ref/libxtbloom_ref.so was not built (build() builds it from the reference sources)"}))
        return
    batch = W.config1(args.systems, seed=1)
    sample, _ = reference_sample(batch, args.cpu_sample)
    lib = abi.Library(str(REF_LIB), backend=abi.BACKEND_CPU, cpu_threads=0)
    for _ in range(args.warmup):
        lib.compute(sample)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        lib.compute(sample)
        times.append(time.perf_counter() - t0)
    t = statistics.median(times)
    value = sample.batch_size / t
    cores = host_cores()
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "systems/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * t, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "global_batch": args.systems,
                   "sample_per_step": sample.batch_size},
        "cpu_baseline": {"value": value, "unit": "systems/s", "cores": cores, "kind": "reference",
                         "sample": f"{sample.batch_size} evenly spaced systems of the 4096-system batch per step, cpu_threads=0 (affinity count, capped at 64)"},
        "e2e": {"value": value, "unit": "systems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def time_form(lib, args, world, stream, dev_batch, outs_d, host_batch, host_outs):
    """Times one execution form: K device-resident steps (CUDA events on the
    context stream, max over ranks); K more with the engine's per-stage CUDA
    events on (the stage breakdown and the roofline; graph replay is off while
    they are recorded); then K end-to-end steps with host buffers."""
    import torch
    opts = lib.make_options()
    fetch(lib, "kernel_timing_off")
    for _ in range(args.warmup):
        lib.compute(dev_batch, opts, outs_d)
    torch.cuda.synchronize()
    fetch(lib, "reset_counters")
    barrier(world)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        lib.compute(dev_batch, opts, outs_d)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = allreduce_max(e0.elapsed_time(e1) / args.steps, world)
    launches = int(fetch(lib, "launch_count")[0])
    # profiled pass: per-stage CUDA events
    fetch(lib, "kernel_timing_on")
    fetch(lib, "reset_counters")
    barrier(world)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        lib.compute(dev_batch, opts, outs_d)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms_prof = allreduce_max(e0.elapsed_time(e1) / args.steps, world)
    stage = fetch(lib, "kernel_times").reshape(-1, 2)
    timing_on = True
    fetch(lib, "kernel_timing_off")
    lib.compute(host_batch, opts, host_outs)
    torch.cuda.synchronize()
    barrier(world)
    e0.record(stream)
    for _ in range(args.steps):
        lib.compute(host_batch, opts, host_outs)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms_e2e = allreduce_max(e0.elapsed_time(e1) / args.steps, world)
    return {"ms": ms, "ms_e2e": ms_e2e, "ms_profiled": ms_prof, "stage": stage, "launches": launches,
            "timing_on": timing_on}


def time_gfn1(args, world, local, stream):
    """GFN1-xTB, spin-polarised: the 2048-radical workload (doublets, 15 %
    with Cl/Br), FP64, graph replay, inputs resident in HBM; K timed calls
    after W warm-up calls (CUDA events on the context stream)."""
    import torch
    from xtbloom_b200 import library_path
    dev = torch.device("cuda", local)
    b = W.config4(2048, seed=4)
    B, N = b.batch_size, b.total_atoms
    pos_d = torch.from_numpy(b.positions).to(dev)
    db = abi.RaggedBatch(b.atom_offsets, b.atomic_numbers, pos_d, b.molecular_charges,
                         b.unpaired_electrons, b.spin_channels)
    outs = {"energies": torch.empty(B, dtype=torch.float64, device=dev),
            "forces": torch.empty(3 * N, dtype=torch.float64, device=dev),
            "atomic_charges": torch.empty(N, dtype=torch.float64, device=dev),
            "scc_iterations": torch.empty(B, dtype=torch.int32, device=dev),
            "scc_converged": torch.empty(B, dtype=torch.uint8, device=dev),
            "per_system_status": torch.empty(B, dtype=torch.int32, device=dev)}
    lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=local, stream=stream.cuda_stream)
    lib.set_execution(abi.PRECISION_FP64, capture_graphs=True)
    opts = lib.make_options(model=abi.MODEL_GFN1)
    for _ in range(max(1, min(args.warmup, 2))):
        lib.compute(db, opts, outs)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    steps = max(1, min(args.steps, 3))
    e0.record(stream)
    for _ in range(steps):
        lib.compute(db, opts, outs)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = allreduce_max(e0.elapsed_time(e1) / steps, world)
    st = outs["per_system_status"].cpu().numpy()
    it = outs["scc_iterations"].cpu().numpy()
    lib.close()
    return {"workload": "GFN1-xTB E+F+q, 2048 radicals C_nH_(2n+1) (n 4..45, doublets, two spin "
                        "channels, 15% with 1-3 H -> Cl/Br), seed 4; SCC 1e-6/1e-8, 300 K",
            "value": world * B / (ms / 1e3), "unit": "systems/s", "ms_per_step": ms, "steps": steps,
            "converged": int(np.sum(st == 0)), "systems": int(B),
            "mean_scc_iterations": float(np.mean(it))}


def _device_outs(torch, dev, B, N):
    return {"energies": torch.empty(B, dtype=torch.float64, device=dev),
            "forces": torch.empty(3 * N, dtype=torch.float64, device=dev),
            "atomic_charges": torch.empty(N, dtype=torch.float64, device=dev),
            "scc_iterations": torch.empty(B, dtype=torch.int32, device=dev),
            "scc_converged": torch.empty(B, dtype=torch.uint8, device=dev),
            "per_system_status": torch.empty(B, dtype=torch.int32, device=dev)}


def time_autograd(args, world, local, stream):
    """Energies and their gradients through the torch.autograd function: 1024
    C20H42 conformers, each in 200 point charges (dE/dR, dE/dR_pc, dE/dQ_pc);
    one step = forward + backward over the batch, inputs resident in HBM."""
    import torch
    from xtbloom_b200.autograd import gfn2_energy
    dev = torch.device("cuda", local)
    b = W.config2(1024, seed=2)
    B = b.batch_size
    z = torch.from_numpy(b.atomic_numbers).to(dev)
    off = torch.from_numpy(b.atom_offsets).to(dev)
    pos = torch.from_numpy(b.positions.reshape(-1, 3)).to(dev).requires_grad_(True)
    poff = torch.from_numpy(b.point_charge_offsets).to(dev)
    ppos = torch.from_numpy(b.point_charge_positions.reshape(-1, 3)).to(dev).requires_grad_(True)
    pq = torch.from_numpy(b.point_charge_values).to(dev).requires_grad_(True)
    pg = torch.from_numpy(b.point_charge_gammas).to(dev)

    def step():
        pos.grad = ppos.grad = pq.grad = None
        e = gfn2_energy(z, off, pos, poff, ppos, pq, pg)
        e.sum().backward()
        return e

    for _ in range(max(1, min(args.warmup, 2))):
        e = step()
    torch.cuda.synchronize()
    barrier(world)
    steps = max(1, min(args.steps, 3))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        e = step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier(world)
    ms = allreduce_max(e0.elapsed_time(e1) / steps, world)
    ok = int(torch.isfinite(e).sum().item())
    return {"workload": "GFN2-xTB energy + dE/dR, dE/dR_pc, dE/dQ_pc via torch.autograd.Function; 1024 "
                        "C20H42 conformers (seed 2), each in 200 point charges (8-20 bohr shell)",
            "value": world * B / (ms / 1e3), "unit": "systems/s", "ms_per_step": ms, "steps": steps,
            "converged": ok, "systems": int(B)}


def time_water(args, world, local, stream):
    """Precision stress: 256 water clusters (H2O)_N, N uniform in 100..200
    (600-1200 AOs), seed 3.  One device-resident call per step in the FP64
    and split-precision forms, and each form's largest output difference from
    the FP64 fixed point (charge tolerance 1e-10, untimed)."""
    import torch
    from xtbloom_b200 import library_path
    dev = torch.device("cuda", local)
    b = W.config3(256, seed=3)
    B, N = b.batch_size, b.total_atoms
    db = abi.RaggedBatch(b.atom_offsets, b.atomic_numbers, torch.from_numpy(b.positions).to(dev),
                         b.molecular_charges, b.unpaired_electrons)
    lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=local, stream=stream.cuda_stream)
    fixed = lib.compute(b, lib.make_options(ctol=1e-10, etol=1e-13))
    line = {"workload": "GFN2-xTB E+F+q, 256 water clusters (H2O)_N, N uniform in 100..200 "
                        "(600-1200 AOs), seed 3; SCC 1e-6/1e-8, 300 K", "unit": "systems/s", "forms": {}}
    okat_fixed = np.repeat(fixed["per_system_status"] == 0, np.diff(b.atom_offsets))
    for form, prec in (("fp64", abi.PRECISION_FP64), ("mixed", abi.PRECISION_MIXED)):
        lib.set_execution(prec, capture_graphs=args.graphs)
        outs = _device_outs(torch, dev, B, N)
        lib.compute(db, lib.make_options(), outs)
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lib.compute(db, lib.make_options(), outs)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        ms = allreduce_max(e0.elapsed_time(e1), world)
        o = {k: v.cpu().numpy() for k, v in outs.items()}
        ok = (o["per_system_status"] == 0) & (fixed["per_system_status"] == 0)
        okat = np.repeat(ok, np.diff(b.atom_offsets)) & okat_fixed
        line["forms"][form] = {
            "value": world * B / (ms / 1e3), "ms_per_step": ms, "steps": 1,
            "converged": int(np.sum(o["per_system_status"] == 0)),
            "vs_fp64_fixed_point": {
                "max_abs_dE_Eh": float(np.abs(o["energies"][ok] - fixed["energies"][ok]).max()),
                "max_abs_dF_Eh_per_bohr": float(np.abs(o["forces"].reshape(-1, 3)[okat]
                                                       - fixed["forces"].reshape(-1, 3)[okat]).max()),
                "max_abs_dq_e": float(np.abs(o["atomic_charges"][okat] - fixed["atomic_charges"][okat]).max())}}
    lib.close()
    return line


def time_strong(args, world, rank, local, stream):
    """One 4096-system batch over all ranks (strong scaling): the systems are
    partitioned by predicted cost (n_AO^3 per channel and iteration); one
    untimed pass over the n^3-only partition gives every system's iteration
    count, which re-weights the partition that is timed.  K device-resident
    calls of each rank's shard, CUDA events, max over ranks."""
    import torch
    import torch.distributed as dist
    from xtbloom_b200 import library_path
    from xtbloom_b200 import sharding as S
    dev = torch.device("cuda", local)
    full = W.config1(args.systems, seed=1)
    lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=local, stream=stream.cuda_stream)
    lib.set_execution(abi.PRECISION_FP64, capture_graphs=args.graphs)
    first = S.plan_shards(full, world)
    out = lib.compute(S.shard(full, first[rank]))
    gathered = [None] * world
    dist.all_gather_object(gathered, {"scc_iterations": out["scc_iterations"]})
    iters = S.scatter_back(full, first, gathered)["scc_iterations"]
    cost = S.predicted_cost(full, iterations=iters)
    shards = S.plan_shards(full, world, cost)
    mine = S.shard(full, shards[rank])
    B, N = mine.batch_size, mine.total_atoms
    db = abi.RaggedBatch(mine.atom_offsets, mine.atomic_numbers, torch.from_numpy(mine.positions).to(dev),
                         mine.molecular_charges, mine.unpaired_electrons)
    outs = {"energies": torch.empty(B, dtype=torch.float64, device=dev),
            "forces": torch.empty(3 * N, dtype=torch.float64, device=dev),
            "atomic_charges": torch.empty(N, dtype=torch.float64, device=dev),
            "scc_iterations": torch.empty(B, dtype=torch.int32, device=dev),
            "scc_converged": torch.empty(B, dtype=torch.uint8, device=dev),
            "per_system_status": torch.empty(B, dtype=torch.int32, device=dev)}
    opts = lib.make_options()
    for _ in range(max(1, min(args.warmup, 2))):
        lib.compute(db, opts, outs)
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        lib.compute(db, opts, outs)
    e1.record(stream)
    torch.cuda.synchronize()
    mine_ms = e0.elapsed_time(e1) / args.steps
    barrier(world)
    ms = allreduce_max(mine_ms, world)
    lib.close()
    loads = [float(cost[s].sum()) for s in shards]
    return {"workload": f"one {args.systems}-system batch over {world} ranks (same batch as the headline, seed 1)",
            "value": args.systems / (ms / 1e3), "unit": "systems/s", "ms_per_step": ms,
            "scaling": "strong", "partition": "LPT over n_AO^3 x (channels x iterations + 2), "
                                              "iterations from one untimed pass",
            "systems_per_rank": [int(len(s)) for s in shards],
            "predicted_load_imbalance": max(loads) / (sum(loads) / world)}


def run_ours(args, world, rank, local):
    import torch
    from xtbloom_b200 import library_path
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    batch = W.config1(args.systems, seed=1 + 1000 * rank)
    if args.once and args.indices:
        batch = W.subset(W.config1(4096, seed=1 + 1000 * rank),
                         np.array([int(x) for x in args.indices.split(",")]))
    B, N = batch.batch_size, batch.total_atoms
    stream = torch.cuda.current_stream(dev)
    pos_d = torch.from_numpy(batch.positions).to(dev)
    dev_batch = abi.RaggedBatch(batch.atom_offsets, batch.atomic_numbers, pos_d,
                                batch.molecular_charges, batch.unpaired_electrons)

    def new_outs_d():
        return {"energies": torch.empty(B, dtype=torch.float64, device=dev),
                "forces": torch.empty(3 * N, dtype=torch.float64, device=dev),
                "atomic_charges": torch.empty(N, dtype=torch.float64, device=dev),
                "scc_iterations": torch.empty(B, dtype=torch.int32, device=dev),
                "scc_converged": torch.empty(B, dtype=torch.uint8, device=dev),
                "per_system_status": torch.empty(B, dtype=torch.int32, device=dev)}

    def new_host_outs():
        return {"energies": np.empty(B), "forces": np.empty(3 * N), "atomic_charges": np.empty(N),
                "scc_iterations": np.empty(B, np.int32), "scc_converged": np.empty(B, np.uint8),
                "per_system_status": np.empty(B, np.int32)}

    if args.once:
        lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=local,
                          stream=stream.cuda_stream)
        lib.set_execution(abi.PRECISION_MIXED if args.form == "mixed" else abi.PRECISION_FP64,
                          capture_graphs=args.graphs)
        if args.workload == "hetero":
            lib.compute(dev_batch, lib.make_options(), new_outs_d())
        else:
            other = (W.config3(256, seed=3) if args.workload == "water" else W.config4(2048, seed=4))
            other = W.subset(other, np.arange(min(args.systems, other.batch_size)))
            model = abi.MODEL_GFN1 if args.workload == "radicals" else abi.MODEL_GFN2
            lib.compute(other, lib.make_options(model=model))
        torch.cuda.synchronize()
        lib.close()
        return
    forms = {}
    results = {}
    probe = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=local,
                        stream=stream.cuda_stream)
    fp64_peak = float(fetch(probe, "fp64_peak", 4)[0])
    # the FP64 fixed point of the batch (charge tolerance 1e-10, not timed):
    # both execution forms are compared with it
    fixed = new_host_outs()
    probe.compute(batch, probe.make_options(ctol=1e-10, etol=1e-13), fixed)
    probe.close()
    clocks = ClockSampler(local)
    for form in (["fp64", "mixed"] if args.form == "both" else [args.form]):
        lib = abi.Library(library_path(), backend=abi.BACKEND_CUDA, device_id=local,
                          stream=stream.cuda_stream)
        lib.set_execution(abi.PRECISION_MIXED if form == "mixed" else abi.PRECISION_FP64,
                          capture_graphs=args.graphs)
        host_outs = new_host_outs()
        forms[form] = time_form(lib, args, world, stream, dev_batch, new_outs_d(), batch, host_outs)
        split = lib.fetch("split_iterations", capacity=B)
        results[form] = (host_outs, split)
        lib.close()
        torch.cuda.synchronize()
    # the GFN1, autograd and water-cluster lines characterise one GPU; with
    # several ranks the run times the headline batch per rank and one batch
    # split over the ranks, and stays short while every GPU is held
    single = world == 1
    gfn1_line = time_gfn1(args, world, local, stream) if single and not args.no_gfn1 else None
    autograd_line = time_autograd(args, world, local, stream) if single and not args.no_autograd else None
    water_line = time_water(args, world, local, stream) if single and not args.no_water else None
    strong = time_strong(args, world, rank, local, stream) if world > 1 else None
    clk = clocks.stop()
    h2d = (B + 1) * 8 + N * 4 + 3 * N * 8 + B * 8 + B * 4
    d2h = B * 8 + 3 * N * 8 + N * 8 + B * 4 + B + B * 4
    if rank != 0:
        return
    # headline: the FP64 form (exact, and the faster form on this workload);
    # the split-precision form is reported beside it in "forms"
    head = "fp64" if "fp64" in forms else "mixed"
    main = forms[head]
    host_outs, split = results[head]
    energies = host_outs["energies"]
    status = host_outs["per_system_status"]
    iters = host_outs["scc_iterations"]
    n_ao = np.array([int(np.sum([{1: 1}.get(int(z), 4) for z in W.molecule(batch, i)[0]]))
                     for i in range(B)])
    nocc = n_ao // 2 + 1
    work = stage_work(n_ao, iters, nocc)
    ms = main["ms"]
    stage = main["stage"]
    timing_on = main["timing_on"]
    per_stage_ms = {STAGES[i]: float(stage[i, 0]) / args.steps for i in range(len(STAGES))} if timing_on else {}
    total_stage = sum(per_stage_ms.values()) or 1.0
    peaks = load_peaks()
    roofline = None
    if timing_on:
        # The stage times come from the profiled pass (per-stage events, size
        # buckets one after another, no graph replay); they are scaled to the
        # timed graph pass by the ratio of the two step times.
        scale = main["ms"] / main["ms_profiled"]
        dom = max(per_stage_ms, key=per_stage_ms.get)
        dom_ms = per_stage_ms[dom] * scale
        calls = float(stage[STAGES.index(dom), 1]) / args.steps
        if dom in work:
            byts, flops = work[dom]["bytes"], work[dom]["flops"]
            gbs = byts / (dom_ms / 1e3) / 1e9
            tfs = flops / (dom_ms / 1e3) / 1e12
            f_hbm = gbs / peaks["hbm_gbs"]
            f_fp64 = tfs / fp64_peak if fp64_peak else 0.0
            compute = f_fp64 > f_hbm
            roofline = {"kernel": dom, "bound": "tensor" if compute else "hbm",
                        "compute_pipe": "fp64" if compute else None,
                        "achieved": tfs if compute else gbs,
                        "peak": fp64_peak if compute else peaks["hbm_gbs"],
                        "unit": "TFLOP/s" if compute else "GB/s",
                        "frac": max(f_hbm, f_fp64),
                        "traffic": (byts / calls * TRIDIAG_DRAM_PER_ALG_BYTE) if dom == "tridiag" and calls else None,
                        "frac_hbm": f_hbm, "frac_fp64": f_fp64,
                        "achieved_gbs": gbs, "achieved_fp64_tflops": tfs,
                        "peak_hbm_gbs": peaks["hbm_gbs"], "peak_hbm_source": peaks["source"],
                        "peak_fp64_tflops": fp64_peak,
                        "peak_fp64_source": "FP64 FMA probe on this device (xtbloom_b200_debug_fetch fp64_peak)",
                        "share_of_step": per_stage_ms[dom] / main["ms_profiled"],
                        "launches_per_step": calls,
                        "algorithmic_bytes_per_launch": byts / calls if calls else None,
                        "timed_in": "profiled pass per-stage CUDA events, scaled to the timed graph pass"}
        else:
            roofline = {"kernel": dom, "bound": "hbm", "achieved": None, "peak": peaks["hbm_gbs"],
                        "unit": "GB/s", "frac": None, "traffic": None, "share_of_step": dom_ms / ms}
    cpu = None
    dE = None
    if world == 1 and not args.no_cpu_baseline and REF_LIB.exists():
        sample, idx = reference_sample(batch, args.cpu_sample)
        t, ref = cpu_run(sample, 0)
        ok = (ref["per_system_status"] == 0) & (status[idx] == 0)
        dE = float(np.max(np.abs(ref["energies"][ok] - energies[idx][ok]))) if ok.any() else None
        cpu = {"value": sample.batch_size / t, "unit": "systems/s", "cores": host_cores(),
               "kind": "reference",
               "sample": (f"{sample.batch_size} evenly spaced systems of the same batch, "
                          "median of 3 calls after one warm-up call, cpu_threads=0 (affinity count)")}
        sample1, _ = reference_sample(batch, args.cpu_sample_1t)
        t1, _ = cpu_run(sample1, 1)
        cpu["cpu_threads_1"] = {"value": sample1.batch_size / t1, "unit": "systems/s", "cores": 1,
                                "sample": f"{sample1.batch_size} evenly spaced systems, median of 3 calls"}
    form_lines = {}
    for name, f in forms.items():
        form_lines[name] = {"value": world * B / (f["ms"] / 1e3), "ms_per_step": f["ms"],
                            "ms_per_step_profiled": f["ms_profiled"],
                            "e2e_value": world * B / (f["ms_e2e"] / 1e3),
                            "split_iteration_fraction": float(results[name][1].sum() / max(results[name][0]["scc_iterations"].sum(), 1))}
    def vs_fixed(o):
        ok = (o["per_system_status"] == 0) & (fixed["per_system_status"] == 0)
        okat = np.repeat(ok, np.diff(batch.atom_offsets))
        return {"max_abs_dE_Eh": float(np.abs(o["energies"][ok] - fixed["energies"][ok]).max()),
                "max_abs_dF_Eh_per_bohr": float(np.abs(o["forces"].reshape(-1, 3)[okat]
                                                       - fixed["forces"].reshape(-1, 3)[okat]).max()),
                "max_abs_dq_e": float(np.abs(o["atomic_charges"][okat] - fixed["atomic_charges"][okat]).max())}
    for name in forms:
        form_lines[name]["vs_fp64_fixed_point"] = vs_fixed(results[name][0])
    mixed_vs = None
    if "mixed" in results and "fp64" in results:
        a, b = results["fp64"][0], results["mixed"][0]
        ok = (a["per_system_status"] == 0) & (b["per_system_status"] == 0)
        okat = np.repeat(ok, np.diff(batch.atom_offsets))
        mixed_vs = {"speedup": forms["fp64"]["ms"] / forms["mixed"]["ms"],
                    "speedup_e2e": forms["fp64"]["ms_e2e"] / forms["mixed"]["ms_e2e"],
                    "max_abs_dE_Eh": float(np.abs(a["energies"][ok] - b["energies"][ok]).max()),
                    "max_abs_dF_Eh_per_bohr": float(np.abs(a["forces"].reshape(-1, 3)[okat] - b["forces"].reshape(-1, 3)[okat]).max()),
                    "max_abs_dq_e": float(np.abs(a["atomic_charges"][okat] - b["atomic_charges"][okat]).max()),
                    "status_equal": bool(np.array_equal(a["per_system_status"], b["per_system_status"]))}
    line = {
        "metric": METRIC, "value": world * B / (ms / 1e3), "unit": "systems/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "global_batch": world * B, "atoms_per_rank": int(N),
                   "path": ("split-precision GEMMs (3xTF32 tensor cores) until the residual is below 1e-5, "
                            "then FP64; FP64 eigensolver, mixer and reductions") if head == "mixed"
                           else "FP64 (all stages)",
                   "graphs": bool(args.graphs),
                   "l2": "inputs larger than L2 (~11 GB of packed matrices per step)",
                   "parallelism": f"dp{world} (independent systems, no collective)"},
        "forms": form_lines,
        "mixed_vs_fp64": mixed_vs,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": {"value": world * B / (main["ms_e2e"] / 1e3), "unit": "systems/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": main["launches"],
        "clocks": clk,
        "parity": {"max_abs_dE_vs_reference_Eh": dE,
                   "converged": int(np.sum(status == 0)), "systems": int(B),
                   "mean_scc_iterations": float(np.mean(iters))},
        "gfn1_radicals": gfn1_line,
        "point_charges_autograd": autograd_line,
        "water_clusters": water_line,
        "one_batch_over_ranks": strong,
        "stage_ms_per_step": per_stage_ms,
        "stage_share": {k: v / total_stage for k, v in per_stage_ms.items()},
    }
    print(json.dumps(line))
    sys.stdout.flush()


def main():
    args = parse()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference(args, world, rank)
    else:
        run_ours(args, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
