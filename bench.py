"""Benchmark: B target-evaluations per second of the fast-multipole Biot-Savart solve.

Workload (the headline precision configuration): a solid torus (R = 2, a = 0.5, axis z),
tensor-product quadrature 512 toroidal x 128 poloidal x 256 radial = 2^24 sources with the
poloidal current, J = 1 A/m^2; the targets are the source points themselves (self term
excluded); order p = 16, leaf capacity 64; FP32 pipeline with the M2L contraction in the
selected mode. One step = one full solve (tree build, P2M, M2M, M2L, L2L, L2P + near field)
with inputs already in HBM; the inputs (2^24 points) are larger than L2.

Multi-GPU: every rank solves its own copy of the workload (replicas, weak scaling); the
aggregate is the units all ranks processed divided by the slowest rank's time.

`--impl reference` times the reference's own CPU FMM (FastMultipoleSolver, FP32, p = 16,
built from the reference sources into oracle/_ref/) on a bounded sample of the workload.

`--extra` adds the other workload families to the same JSON line under "workloads" (each with
its own timing, accuracy against the FP64 direct sum and tree statistics):
  c1     FP64, torus 128x32x16 = 65,536 sources (azimuthal J), 32^3 grid on [-3,3]^3, p = 10, leaf 32
  c2     FP32, torus 256x64x64 = 2^20 sources, 2^20 seeded targets in [-3,3]^3, p = 12, leaf 64
  batch  FP32 + split-BF16 M2L, 256 independent tori (log-uniform 2^12..2^18 points, random pose,
         2^14 targets each), p = 8, leaf 32: eager solve and CUDA-graph replay on the fixed forest
  c5     FP32 differentiation: loss = 1/2 sum |B - B*|^2 on 2^18 targets, N = 2^20, p = 12; forward
         + adjoint (dLoss/dJ, dLoss/dx) against the FP64 direct-sum adjoint on 64 seeded sources
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "B evals/s (N=2^24, p=16) split-BF16 vs FP32 FMM at rel err<=1e-6; adjoint/forward"
UNIT = "target-evals/s"
SEED = 20260002
# DRAM bytes (read + write) per M2L pair of the tensor-core M2L, from an ncu capture of the
# 128 x 32 x 64 torus at p = 16 (536.6 MB read + 54.2 MB written for 1,271,544 pairs;
# profiles/m2l_tc_bf16x3_torus2e18_p16.md)
M2L_DRAM_BYTES_PER_PAIR = 590.78e6 / 1271544
# bounded CPU samples of the same workload family (torus points, targets = sources): 32 x 8 x 8 = 2,048 for
# each step of the reference arm (25 steps stay within a few minutes), 32 x 8 x 16 = 4,096 for the main
# line's cpu_baseline (~15 s)
CPU_SAMPLE = (32, 8, 8)
CPU_BASELINE_SAMPLE = (32, 8, 16)
# the reference CPU FMM's throughput against N, measured once on the 8-core Xeon of the build container
# (oracle/_ref/libref_fmm_f32_p16.so, p = 16, leaf 64, targets = sources): it falls as the tree deepens
# (more M2L pairs per target), so a small sample overstates the reference at N = 2^24
CPU_TREND = {"2048": 357.3, "4096": 274.3, "8192": 154.5, "16384": 142.1, "65536": 81.6}


def m2l_flops_per_pair(p, cut):
    """FLOPs of one M2L box pair with the operator the kernels execute: the three components x 2 x the
    operator's entries (l, lambda) with l + lambda <= cut (output degree l, input degree lambda <= p)."""
    return 6 * sum((2 * l + 1) * (2 * lam + 1) for l in range(p + 1) for lam in range(p + 1) if l + lam <= cut)


def fp32_core_peak_tflops(sm_mhz):
    """Nominal FP32 FMA peak of the CUDA cores: 148 SMs x 128 lanes x 2 FLOPs x the SM clock."""
    return 148 * 128 * 2 * sm_mhz * 1e6 / 1e12


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_setup():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device(f"cuda:{local}"))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """The maximum of x over the ranks (device times are reported as the slowest rank's)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate(units_per_rank, ms_per_rank, world):
    """Whole-job throughput: the units all ranks processed over the slowest rank's time."""
    ms = max_over_ranks(ms_per_rank, world)
    return world * units_per_rank / (ms / 1000.0), ms


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.proc:
            return out
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for k, name in enumerate(names):
                if r[5 + k].lower() == "active":
                    reasons.add(name)
        out["sm_mhz"] = statistics.median(sm) if sm else None
        out["sm_max_mhz"] = max(mx) if mx else None
        out["reasons"] = sorted(reasons)
        out["samples"] = len(rows)
        return out


def make_workload(n_phi, n_theta, n_rho):
    from bachelors_b200 import geometry as G
    xyz, w, J = G.torus(n_phi, n_theta, n_rho, 2.0, 0.5, current="poloidal")
    return xyz.astype(np.float32), w.astype(np.float32), J.astype(np.float32)


def cpu_reference_run(sample=CPU_SAMPLE):
    """One run of the reference's CPU FMM (FP32, p = 16, leaf 64/64) on the sample; returns
    (target-evals/s, seconds, n)."""
    from oracle.oracle import Reference
    ref = Reference("f32", 16)
    xyz, w, _ = make_workload(*sample)
    t0 = time.perf_counter()
    _, found, _ = ref.fmm(np.c_[xyz, w].astype(np.float64), xyz.astype(np.float64), 64, 64, 1.0)
    dt = time.perf_counter() - t0
    return len(xyz) / dt, dt, len(xyz)


def run_reference(args, world, rank):
    if rank != 0:
        return
    from oracle.oracle import Reference
    cores = os.cpu_count()
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    if not Reference.available("f32", 16):
        print(json.dumps({"impl": "reference", "unavailable": "reference CPU build oracle/_ref/libref_fmm_f32_p16.so "
                          "missing (built by oracle/ref/build_ref.sh from the reference sources)"}))
        return
    for _ in range(args.warmup):
        cpu_reference_run()
    times = []
    n = 0
    for _ in range(args.steps):
        _, dt, n = cpu_reference_run()
        times.append(dt)
    ms = 1000 * sum(times) / len(times)
    value = n / (ms / 1000)
    sample = f"torus {CPU_SAMPLE[0]}x{CPU_SAMPLE[1]}x{CPU_SAMPLE[2]} = {n} sources, targets = sources, p=16, leaf 64/64, FP32"
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "torus 512x128x256 (2^24) targets=sources p=16 leaf 64 (reference: bounded sample)",
                   "sample": sample},
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _timed(fn, steps, world):
    """Device time per call of fn() (CUDA events, max over ranks)."""
    import torch
    torch.cuda.synchronize()
    barrier(world)
    e0, e1 = _events()
    e0.record()
    for _ in range(steps):
        out = fn()
    e1.record()
    torch.cuda.synchronize()
    return max_over_ranks(e0.elapsed_time(e1) / steps, world), out


def _tree_stats(plan):
    st = plan.stats()
    return {k: st[k] for k in ("nodes", "levels", "v_pairs", "p2p_pairs", "coils")}


def extra_c1(local, world, steps):
    """FP64 plain FMM: torus 128x32x16 (azimuthal current, the reference's direction), 32^3 grid."""
    import torch
    from bachelors_b200 import Plan, geometry as G
    xyz, w, _ = G.torus(128, 32, 16, 2.0, 0.5, current="azimuthal")
    tgt = G.cube_grid(32, -3.0, 3.0)
    dev = f"cuda:{local}"
    plan = Plan(order=10, leaf_capacity=32, precision="fp64", device=local)
    plan.set_sources(torch.from_numpy(xyz).to(dev), torch.from_numpy(w).to(dev), None)
    plan.set_targets(torch.from_numpy(tgt).to(dev))
    for _ in range(3):
        B, _ = plan.solve(1.0, 1)
    ms, (B, _) = _timed(lambda: plan.solve(1.0, 1), steps, world)
    D, _ = plan.direct(1.0, 1)
    err = float(torch.linalg.norm(B - D) / torch.linalg.norm(D))
    res = {"workload": "FP64 torus 128x32x16 = 65536 sources (azimuthal J), 32^3 grid on [-3,3]^3, p=10, leaf 32",
           "value": world * len(tgt) / (ms / 1000), "unit": UNIT, "ms_per_step": ms, "steps": steps,
           "rel_l2_vs_fp64_direct": err, "error_samples": "all 32768 targets", "tree": _tree_stats(plan)}
    plan.close()
    return res


def extra_c2(local, world, steps):
    """FP32 plain FMM at 2^20 sources and 2^20 seeded targets, p = 12, leaf 64 (CUDA-core and split-BF16 M2L)."""
    import torch
    from bachelors_b200 import Plan, geometry as G
    xyz, w, J = make_workload(256, 64, 64)
    tgt = G.uniform_points(1 << 20, -3.0, 3.0, 20260002).astype(np.float32)
    dev = f"cuda:{local}"
    dx, dw, dJ, dt = (torch.from_numpy(a).to(dev) for a in (xyz, w, J, tgt))
    rng = np.random.default_rng(20260002)
    idx = rng.choice(len(tgt), size=4096, replace=False)
    out = {"workload": "FP32 torus 256x64x64 = 2^20 sources, 2^20 targets U[-3,3]^3 (seed 20260002), p=12, leaf 64",
           "unit": UNIT, "error_samples": "4096 seeded targets vs FP64 direct"}
    Bd = None
    for mode in ("simt", "bf16x3"):
        plan = Plan(order=12, leaf_capacity=64, precision="fp32", m2l=mode, device=local)
        plan.set_sources(dx, dw, dJ)
        plan.set_targets(dt)
        for _ in range(3):
            plan.solve(1.0, 1)
        ms, (B, _) = _timed(lambda: plan.solve(1.0, 1), steps, world)
        if Bd is None:
            Bd = plan.direct_fp64(tgt[idx].astype(np.float64), current=1.0)
        Bh = B.cpu().numpy().astype(np.float64)[idx]
        out[f"m2l_{mode}"] = {"value": world * len(tgt) / (ms / 1000), "ms_per_step": ms, "steps": steps,
                              "rel_l2_vs_fp64_direct": float(np.linalg.norm(Bh - Bd) / np.linalg.norm(Bd)),
                              "phases_ms": {k: plan.stats()[k] for k in ("ms_tree", "ms_upward", "ms_m2l",
                                                                         "ms_downward", "ms_near")}}
        out["tree"] = _tree_stats(plan)
        plan.close()
    out["value"] = out["m2l_simt"]["value"]
    return out


def extra_batch(local, world, steps):
    """256 independent tori in one plan: eager full solves and CUDA-graph replays on the fixed forest."""
    import torch
    from bachelors_b200 import Plan, geometry as G
    xyz, w, J, tgt, so, to, prm = G.torus_batch(256, seed=20260004, params=True)
    dev = f"cuda:{local}"
    dx, dw, dJ, dt = (torch.from_numpy(a.astype(np.float32)).to(dev) for a in (xyz, w, J, tgt))
    plan = Plan(order=8, leaf_capacity=32, precision="fp32", m2l="bf16x3", device=local)
    plan.set_sources(dx, dw, dJ)
    plan.set_targets(dt)
    plan.set_coils(so, to)
    for _ in range(3):
        plan.solve(1.0, 1)
    ms, (B, _) = _timed(lambda: plan.solve(1.0, 1), steps, world)
    phases = {k: plan.stats()[k] for k in ("ms_tree", "ms_upward", "ms_m2l", "ms_downward", "ms_near", "ms_total")}
    plan.graph_capture(1)
    for _ in range(3):
        plan.graph_launch(1.0)
    gms, (Bg, _) = _timed(lambda: plan.graph_launch(1.0), steps, world)
    # accuracy: 16 seeded targets per coil against the FP64 direct sum over that coil's sources
    rng = np.random.default_rng(20260004)
    pick = np.concatenate([rng.choice(np.arange(to[c], to[c + 1]), size=16, replace=False) for c in range(256)])
    # the reference sum takes the solver's own FP32 inputs (rounded positions of coils ~17 units from the origin
    # move by ~1e-6, which is 3e-4 of the point spacing of the densest coils: input rounding, not solver error)
    r32 = lambda a: a.astype(np.float32).astype(np.float64)
    ref = Plan(order=1, leaf_capacity=1 << 30, precision="fp64", device=local)
    ref.set_sources(r32(xyz), r32(w), r32(J))
    ref.set_targets(r32(tgt[pick]))
    ref.set_coils(so, np.arange(0, 16 * 257, 16))
    Bd, _ = ref.direct(1.0, 1)
    ref.close()
    Bh = B.cpu().numpy().astype(np.float64)[pick]
    err = float(np.linalg.norm(Bh - Bd) / np.linalg.norm(Bd))
    per_coil = [float(np.linalg.norm(Bh[16 * c:16 * c + 16] - Bd[16 * c:16 * c + 16]) /
                      max(np.linalg.norm(Bd[16 * c:16 * c + 16]), 1e-300)) for c in range(256)]
    # the same errors against each coil's field scale B0 = MU0 |J| a: a poloidal current's field almost
    # vanishes outside its torus, where most targets lie, so per-coil relative errors are ill-conditioned
    mu0 = 1.2566370614e-6
    per_coil_b0 = [float(np.sqrt(np.mean(np.sum((Bh[16 * c:16 * c + 16] - Bd[16 * c:16 * c + 16]) ** 2, axis=1))) /
                         (mu0 * prm[c, 2] * prm[c, 1])) for c in range(256)]
    res = {"workload": f"256 tori (R~U(1,3), a~U(0.2,0.6), random axis, centre U[-10,10]^3, log-uniform "
                       f"2^12..2^18 points, J poloidal |J|~U(0.5,2)), {len(w)} sources, 2^14 targets each = "
                       f"{len(tgt)} targets; p=8, leaf 32, FP32 + BF16X3 M2L; seed 20260004",
           "value": world * len(tgt) / (ms / 1000), "unit": UNIT, "ms_per_step": ms, "steps": steps,
           "graph_replay": {"value": world * len(tgt) / (gms / 1000), "ms_per_step": gms,
                            "note": "P2M..L2P + near field replayed on the fixed forest (new strengths, same points)"},
           "rel_l2_vs_fp64_direct": err, "max_coil_rel_l2": max(per_coil),
           "max_coil_rms_err_over_field_scale": max(per_coil_b0), "field_scale_bar": 1e-4,
           "field_scale": "B0 = MU0 |J| a per coil (a = minor radius)",
           "error_samples": "16 seeded targets per coil (4096) vs the FP64 direct sum over the coil's sources, both "
                            "from the same FP32 inputs",
           "phases_ms": phases, "tree": _tree_stats(plan)}
    plan.close()
    return res


def extra_c5(local, world, steps):
    """Differentiation workload: forward + adjoint of loss = 1/2 sum |B - B*|^2."""
    import torch
    from bachelors_b200 import Plan, geometry as G
    xyz, w, J = G.torus(256, 64, 64, 2.0, 0.5, current="poloidal")
    rng = np.random.default_rng(20260005)
    Jstar = J * (1 + 0.05 * rng.normal(size=(len(J), 1)))
    tgt = G.uniform_points(1 << 18, -3.0, 3.0, 20260005)
    dev = f"cuda:{local}"
    f32 = lambda a: torch.from_numpy(a.astype(np.float32)).to(dev)
    plan = Plan(order=12, leaf_capacity=64, precision="fp32", m2l="bf16x3", device=local)
    plan.set_sources(f32(xyz), f32(w), f32(Jstar))
    plan.set_targets(f32(tgt))
    Bstar, _ = plan.solve(1.0, 1)
    Bstar = Bstar.clone()
    plan.update_sources(f32(w), f32(J))

    def step():
        B, _ = plan.solve(1.0, 1)
        g = B - Bstar
        return plan.adjoint(g, 1.0)
    for _ in range(3):
        step()
    ms, (dJ, dX) = _timed(step, steps, world)
    fms, _ = _timed(lambda: plan.solve(1.0, 1), steps, world)
    B, _ = plan.solve(1.0, 1)
    g = (B - Bstar).cpu().numpy().astype(np.float64)
    # FP64 direct-sum adjoint for 64 seeded sources (each source's gradient involves only itself
    # and the targets, so a plan holding just those sources gives their exact gradients)
    pick = rng.choice(len(xyz), size=64, replace=False)
    ref = Plan(order=1, leaf_capacity=1 << 30, precision="fp64", device=local)
    ref.set_sources(xyz[pick], w[pick], J[pick])
    ref.set_targets(tgt)
    rJ, rX = ref.adjoint_direct(g, 1.0)
    ref.close()
    gJ = dJ.cpu().numpy().astype(np.float64)[pick]
    gX = dX.cpu().numpy().astype(np.float64)[pick]
    res = {"workload": "FP32 torus 256x64x64 = 2^20 sources, 2^18 targets U[-3,3]^3, loss 1/2 sum|B - B*|^2 with "
                       "B* from J (1 + 0.05 N(0,1)), p=12, leaf 64, BF16X3 M2L; seed 20260005",
           "value": world * len(tgt) / (ms / 1000), "unit": "loss+gradient evals/s (targets)", "ms_per_step": ms,
           "forward_ms": fms, "adjoint_over_forward": (ms - fms) / fms, "steps": steps,
           "rel_l2_dLdJ_vs_fp64_direct_adjoint": float(np.linalg.norm(gJ - rJ) / np.linalg.norm(rJ)),
           "rel_l2_dLdx_vs_fp64_direct_adjoint": float(np.linalg.norm(gX - rX) / np.linalg.norm(rX)),
           "error_samples": "64 seeded sources (g from this run's B)"}
    plan.close()
    return res


def extra_batch_sharded(local, world, steps):
    """The 256-coil batch split over the ranks by whole coils (fmm_batch_partition), each rank solving its
    shard with one batched plan and the fields gathered over NCCL into every rank (strong scaling: the same
    batch whatever the rank count); time = the slowest rank's, CUDA events around solve + gather."""
    import torch
    from bachelors_b200 import geometry as G
    from bachelors_b200.sharding import gather_fields, partition_coils, Shard, solve_shard_on_gpu
    xyz, w, J, tgt, so, to = G.torus_batch(256, seed=20260004)
    part = partition_coils(so, to, world)
    rank = int(os.environ.get("RANK", "0"))
    f32 = lambda a: a.astype(np.float32)
    shard = Shard(f32(xyz), f32(w), f32(J), f32(tgt), so, to, part, rank)

    def step():
        B = solve_shard_on_gpu(shard, order=8, leaf_capacity=32, precision="fp32", m2l="bf16x3", device=local)
        return gather_fields(shard, B, len(tgt), rank, world) if world > 1 else B
    for _ in range(3):
        step()
    ms, B = _timed(step, steps, world)
    work = np.bincount(part, weights=np.diff(so) + np.diff(to), minlength=world)
    return {"workload": "the 256-coil batch (see batch) split by whole coils over the ranks, fields gathered to "
                        "every rank", "value": len(tgt) / (ms / 1000), "unit": UNIT, "ms_per_step": ms,
            "steps": steps, "scaling": "strong", "coils_per_rank": np.bincount(part, minlength=world).tolist(),
            "work_imbalance": float(work.max() / work.mean()),
            "note": "includes plan creation and tree build per step (each rank's shard is solved from its points)"}


EXTRAS = {"c1": extra_c1, "c2": extra_c2, "batch": extra_batch, "c5": extra_c5, "batch_sharded": extra_batch_sharded}


def count_launches(plan):
    """Kernels one solve launches (from the CUDA profiler), excluding library kernels."""
    import torch
    from torch.profiler import ProfilerActivity, profile
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        plan.solve(1.0, 1)
        torch.cuda.synchronize()
    names = [e.name for e in prof.events() if e.device_type == torch.autograd.DeviceType.CUDA]
    kernels = [n for n in names if not n.lower().startswith(("memcpy", "memset"))]
    ours = [n for n in kernels if "fmm" in n or "kM2L" in n or "kP2" in n]
    return len(kernels), len(ours), sorted(set(ours))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--m2l", default="auto", choices=["auto", "simt", "bf16x3", "bf16x6"])
    ap.add_argument("--size", default="512,128,256", help="torus n_phi,n_theta,n_rho")
    ap.add_argument("--order", type=int, default=16)
    ap.add_argument("--leaf", type=int, default=64)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP32 comparison solve")
    ap.add_argument("--no-launch-count", action="store_true", help="skip the profiler-based launch count")
    ap.add_argument("--no-adjoint", action="store_true", help="skip the adjoint timing")
    ap.add_argument("--no-tune", action="store_true", help="keep the default tile choices (no autotuning)")
    ap.add_argument("--extra", default="c1,c2,batch,c5",
                    help="comma list of further workloads to measure into 'workloads' (c1, c2, batch, c5; '' = none)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return

    import torch
    world, rank, local = dist_setup()
    torch.cuda.set_device(local)
    from bachelors_b200 import FastMultipoleSolver, Plan

    size = tuple(int(v) for v in args.size.split(","))
    xyz, w, J = make_workload(*size)
    n = len(xyz)
    m2l = "bf16x3" if args.m2l == "auto" else args.m2l
    dev = f"cuda:{local}"
    d_xyz = torch.from_numpy(xyz).to(dev)
    d_w = torch.from_numpy(w).to(dev)
    d_J = torch.from_numpy(J).to(dev)
    plan = Plan(order=args.order, leaf_capacity=args.leaf, precision="fp32", m2l=m2l, device=local)
    plan.set_sources(d_xyz, d_w, d_J)
    plan.set_targets_to_sources()   # targets = the source points (the plan reuses their sorted order)
    B, _ = plan.solve(1.0, 1)
    # the project's autotuner picks the tile choices on this workload (outside the timed region)
    tuning = plan.autotune() if not args.no_tune else plan.tuning()
    for _ in range(args.warmup):
        B, _ = plan.solve(1.0, 1)
    torch.cuda.synchronize()

    # timed region: K full solves, inputs resident in HBM
    clocks = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    m2l_ms = []
    phase = []
    ev0.record()
    for _ in range(args.steps):
        B, _ = plan.solve(1.0, 1)
        st = plan.stats()
        m2l_ms.append(st["ms_m2l"])
        phase.append(st)
    ev1.record()
    torch.cuda.synchronize()
    barrier(world)
    clk = clocks.stop()
    ms = ev0.elapsed_time(ev1) / args.steps
    value, ms_max = aggregate(n, ms, world)

    st = phase[-1]
    L = (args.order + 1) ** 2
    cut = args.order + 8            # the FP32 plans' default M2L degree cutoff (l + lambda <= p + 8)
    per_pair = m2l_flops_per_pair(args.order, cut)
    flops_m2l = st["v_pairs"] * per_pair
    flops_dense = st["v_pairs"] * 3 * 2 * L * L
    flops_reftrunc = st["v_pairs"] * m2l_flops_per_pair(args.order, args.order)
    m2l_avg = sum(m2l_ms) / len(m2l_ms)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak_src = "measured" if "bf16_tflops" in peaks else "fallback"
    bf16_peak = peaks.get("bf16_tflops", 1590.0)
    bf16_sustained = peaks.get("bf16_tflops_sustained", 1400.0)
    if m2l == "simt":
        # the CUDA-core form: its peak is the FP32 FMA rate (not measured by the driver; nominal)
        peak_src = "nominal FP32 FMA (148 SMs x 128 lanes x 2 x max SM clock)"
        bf16_peak = bf16_sustained = fp32_core_peak_tflops(peaks.get("sm_max_mhz", 1965.0))
    achieved = flops_m2l / (m2l_avg / 1000.0) / 1e12

    # accuracy against the FP64 direct sum on 4096 seeded targets
    rng = np.random.default_rng(SEED)
    idx = rng.choice(n, size=min(4096, n), replace=False)
    Bh = B.cpu().numpy().astype(np.float64)
    Bd = plan.direct_fp64(xyz[idx].astype(np.float64), current=1.0)
    rel_err = float(np.linalg.norm(Bh[idx] - Bd) / np.linalg.norm(Bd))

    # the metric's own terms (accuracy bar, split-BF16 / plain FP32 ratio, adjoint / forward), filled in
    # below; kept inside "config" as well as at the top level so that a reader of the parsed line sees them
    terms = {"rel_l2_vs_fp64_direct": rel_err, "rel_l2_bar": 1e-6, "error_samples": "4096 seeded targets"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded torus quadrature)",
        "rel_l2_vs_fp64_direct": rel_err,
        "config": {"workload": f"torus {size[0]}x{size[1]}x{size[2]} = {n} sources, targets = sources (self excluded), "
                               f"p={args.order}, leaf {args.leaf}, M2L {m2l}",
                   "m2l": m2l, "order": args.order, "leaf": args.leaf, "n_sources": n, "n_targets": n,
                   "l2_flush": "inputs larger than L2 (2^24 points)", "parallelism": f"replicas x{world}",
                   "measured_terms": terms},
        "roofline": {"kernel": f"M2L ({m2l})", "bound": "fp32" if m2l == "simt" else "tensor", "achieved": achieved,
                     "peak": bf16_peak,
                     "unit": "TFLOP/s", "frac": achieved / bf16_peak,
                     "frac_sustained": achieved / bf16_sustained, "peak_sustained": bf16_sustained,
                     "traffic": M2L_DRAM_BYTES_PER_PAIR * st["v_pairs"] if m2l == "bf16x3" else None,
                     "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one ncu capture of the "
                                       "kernel on the 128x32x64 torus (465 B per M2L pair), scaled by the pairs "
                                       "of this launch",
                     "flops_per_launch": flops_m2l, "flops_per_pair": per_pair,
                     "dense_equiv_flops_per_launch": flops_dense,
                     "reference_truncation_flops_per_launch": flops_reftrunc,
                     "note": f"algorithmic FLOPs = V pairs x 3 components x 2 x the entries of the executed operator "
                             f"(l + lambda <= p + 8 = {cut}); dense_equiv counts (p+1)^4, reference_truncation "
                             f"l + lambda <= p; peak = {peak_src} (bf16: MEASURED_PEAKS.json dense, burst for frac, "
                             f"sustained for frac_sustained); achieved over the M2L phase time (CUDA events)"},
        "clocks": clk,
        "tuning": tuning,
        "phases_ms": {k: st[k] for k in ("ms_tree", "ms_upward", "ms_m2l", "ms_downward", "ms_near", "ms_total")},
        "tree": {k: st[k] for k in ("nodes", "levels", "v_pairs", "p2p_pairs", "m2l_tiles", "m2l_tile_offsets")},
    }

    # adjoint FMM (dLoss/dJ and dLoss/d(source positions)) for g = B - B*, with B* = 1.01 B: one
    # warm-up and K timed adjoint calls, against the forward solve's time
    if not args.no_adjoint:
        g = (B * 0.01).contiguous()
        plan.adjoint(g, 1.0)
        torch.cuda.synchronize()
        barrier(world)
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        a0.record()
        for _ in range(args.steps):
            dJ, dx = plan.adjoint(g, 1.0)
        a1.record()
        torch.cuda.synchronize()
        ams = max_over_ranks(a0.elapsed_time(a1) / args.steps, world)
        line["adjoint"] = {"ms_per_step": ams, "adjoint_over_forward": ams / ms_max,
                           "outputs": "dLoss/dJ and dLoss/d(source positions), 2 x [N,3]"}
        terms["adjoint_over_forward"] = ams / ms_max
        del dJ, dx, g

    # the other M2L forms on the same workload (one warm-up and one timed solve each): the plain
    # FP32 FMM (M2L on the CUDA cores) for the split-BF16 ratio, the six-piece split and one TF32 pass
    def one_mode(mode, steps=1, warmup=1):
        pplan = Plan(order=args.order, leaf_capacity=args.leaf, precision="fp32", m2l=mode, device=local)
        pplan.set_sources(d_xyz, d_w, d_J)
        pplan.set_targets_to_sources()
        for _ in range(warmup):
            Bp, _ = pplan.solve(1.0, 1)
        torch.cuda.synchronize()
        barrier(world)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        m2l = []
        e0.record()
        for _ in range(steps):
            Bp, _ = pplan.solve(1.0, 1)
            m2l.append(pplan.stats()["ms_m2l"])
        e1.record()
        torch.cuda.synchronize()
        pms = max_over_ranks(e0.elapsed_time(e1) / steps, world)
        Bph = Bp.cpu().numpy().astype(np.float64)
        res = {"value": world * n / (pms / 1000.0), "ms_per_step": pms, "steps": steps, "warmup": warmup,
               "rel_l2_vs_fp64_direct": float(np.linalg.norm(Bph[idx] - Bd) / np.linalg.norm(Bd)),
               "ms_m2l": sum(m2l) / len(m2l)}
        pplan.close()
        return res

    if not args.no_plain:
        for mode in ("simt", "bf16x3", "bf16x6", "tf32"):
            if mode == m2l:
                continue
            key = "plain_fp32" if mode == "simt" else f"m2l_{mode}"
            # the plain FP32 comparator is timed like the headline (same steps, warm-ups up to 3); the other
            # forms once
            line[key] = one_mode(mode, args.steps, min(args.warmup, 3)) if mode == "simt" else one_mode(mode)
        if "plain_fp32" in line:
            pf = line["plain_fp32"]
            line["speedup_vs_plain_fp32"] = line["value"] / pf["value"]
            terms["speedup_vs_plain_fp32"] = line["speedup_vs_plain_fp32"]
            terms["plain_fp32_rel_l2_vs_fp64_direct"] = pf["rel_l2_vs_fp64_direct"]
            # the comparator's own roofline: the same executed M2L operator on the CUDA cores (FP32 FMA)
            fp32_peak = fp32_core_peak_tflops(peaks.get("sm_max_mhz", 1965.0))
            ach32 = flops_m2l / (pf["ms_m2l"] / 1000.0) / 1e12
            pf["roofline"] = {"kernel": "M2L (simt, kM2LSimt)", "bound": "fp32", "achieved": ach32, "peak": fp32_peak,
                              "unit": "TFLOP/s", "frac": ach32 / fp32_peak,
                              "note": "peak = nominal FP32 FMA rate of the CUDA cores, 148 SMs x 128 lanes x 2 x "
                                      "max SM clock (not in MEASURED_PEAKS.json); same FLOP count as the headline"}
            terms["plain_fp32_m2l_frac_of_fp32_peak"] = ach32 / fp32_peak

    if rank == 0 and not args.no_launch_count:
        try:
            total, ours, names = count_launches(plan)
            line["gpu_launches"] = ours * args.steps
            line["gpu_launch_names"] = names
            line["library_launches_per_step"] = total - ours
        except Exception as e:  # profiler unavailable
            line["gpu_launches"] = None
            line["gpu_launch_error"] = str(e)[:200]

    # end to end through the public API: pinned host inputs, H2D + solve + D2H each step
    if not args.no_e2e:
        hx = torch.from_numpy(xyz).pin_memory().numpy()
        hw = torch.from_numpy(w).pin_memory().numpy()
        hJ = torch.from_numpy(J).pin_memory().numpy()
        s = FastMultipoleSolver((hx, hw, hJ), hx, quadratureOctreeLeafCapacity=args.leaf,
                                calculationPointOctreeLeafCapacity=args.leaf, order=args.order, precision="fp32",
                                m2l=m2l, device=local)
        # the same warm-up steps as the device-resident line: the plan's page-locked result buffers (one per
        # result the caller still holds) are made before the timed steps
        for _ in range(max(args.warmup, 2)):
            s.plan.set_sources(hx, hw, hJ, asynchronous=True)
            s.plan.set_targets_to_sources()
            Bh2 = s.solve(1.0, "B")
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            # page-locked inputs: the points cross the bus first, the weights and directions under the
            # tree build (fmm_set_sources_async)
            s.plan.set_sources(hx, hw, hJ, asynchronous=True)
            s.plan.set_targets_to_sources()   # the targets are the source points: moved once
            Bh2 = s.solve(1.0, "B")
        torch.cuda.synchronize()
        e2e_ms = (time.perf_counter() - t0) * 1000 / args.steps
        e2e_ms = max_over_ranks(e2e_ms, world)
        line["e2e"] = {"value": world * n / (e2e_ms / 1000.0), "unit": UNIT,
                       "h2d_bytes_per_step": int(xyz.nbytes + w.nbytes + J.nbytes),
                       "d2h_bytes_per_step": int(Bh2.nbytes), "ms_per_step": e2e_ms,
                       "note": "page-locked inputs through fmm_set_sources_async: the points cross first, the "
                               "weights and directions under the tree build; B back into page-locked memory"}
        s.plan.close()

    extras = [e for e in args.extra.split(",") if e]
    if world > 1 and extras and "batch_sharded" not in extras:
        extras.append("batch_sharded")   # the one workload that shards across ranks
    if extras:
        line["workloads"] = {}
        for e in extras:
            try:
                line["workloads"][e] = EXTRAS[e](local, world, args.steps)
            except Exception as ex:  # keep the headline line even if a secondary workload fails
                line["workloads"][e] = {"error": f"{type(ex).__name__}: {str(ex)[:300]}"}

    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            from oracle.oracle import Reference
            if Reference.available("f32", 16):
                s = CPU_BASELINE_SAMPLE
                v, dt, ns = cpu_reference_run(s)
                line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                                        "sample": f"torus {s[0]}x{s[1]}x{s[2]} = {ns} sources, targets = sources, "
                                                  f"p=16, leaf 64/64, FP32, {dt:.1f} s; the reference's M2L/L2L/L2P "
                                                  "run on one thread by design",
                                        "trend_evals_per_s_by_n": CPU_TREND,
                                        "trend_note": "measured once on the build container's 8-core Xeon: the "
                                                      "reference's evals/s falls with N (~N^-0.3), so at N = 2^24 "
                                                      "it is lower than any bounded sample and the ratio against "
                                                      "a sample understates the speed-up"}
        except Exception as e:
            line["cpu_baseline"] = {"error": str(e)[:200]}
    plan.close()
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
