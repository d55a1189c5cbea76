#!/usr/bin/env python
"""Jacobian builds/s of the Newton-shooting solver on B200.

Workload (the metric's configuration): D = 4, Ntau = 1024, NLeft = NRight =
4000 (8000 spatial points), Gauss-Legendre IRK2, PrecisionIRK 1e-15 -- the
reference's data/simulation_4D_1024.json setup -- with seeded free data.  One
step = one finite-difference Jacobian build: 768 columns, each a two-sided
shoot (1536 IRK sweeps of 4000 steps), as NewtonSolver::assembleJacobian
(NewtonSolver.cpp:615-702) computes it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

Multi-GPU: one process per GPU; every rank builds the Jacobian of its own
seeded solve (independent work, no data-path collective) and `value` is all
ranks' builds divided by the slowest rank's device time (weak scaling).
Under torchrun (WORLD_SIZE set) the ranks are torchrun's; `--gpus N` with
N > 1 and no WORLD_SIZE re-launches this script as N local ranks through
torch.distributed.run (127.0.0.1 rendezvous, NCCL).  `--dry-run` runs the
rank launch and the multi-rank host logic (column partition, all-gather,
max-over-ranks) on gloo without a GPU.
--impl reference times the reference's own CPU implementation (oracle/_ref,
OpenMP over Jacobian columns, all host threads) on a bounded column sample.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
PKG = REPO / "parallel-critical-collapse_b200"
sys.path.insert(0, str(PKG))

METRIC = "Jacobian builds/s at Nτ=1024×8000 pts, mixed vs FP64; p50/p99 solve latency"
FIXTURE = REPO / "tests" / "golden" / "ref_c3_fixture.npz"


def f_rhs(n):
    """Algorithmic FP64 flops of one RHS evaluation: 7 complex FFTs of length
    Ntau (5 N log2 N each) + 100 flops per point of pointwise work."""
    return 7 * 5 * n * np.log2(n) + 100 * n


def workload(seed, amp):
    """C3 config and seeded free data.  Free data: the reference's near-solution
    (data/simulation_4D_1024.json, packed) plus perturb()'s seeded noise."""
    d = np.load(FIXTURE)
    cfg = json.loads(str(d["config"]))
    return cfg, perturb(d["in0"], np.random.default_rng(seed), amp)


# Seeds of the C3 free data whose base shoot converges (checked on a B200 over
# seeds 1024..1199: at perturbation amplitude 0.1 most seeds march into an IRK
# failure).  Rank r of a multi-GPU run with the default seed takes the r-th,
# so that every GPU builds the Jacobian of a solve of its own.
C3_SEEDS = (1024, 1031, 1034, 1046, 1058, 1075, 1090, 1091, 1100, 1117, 1122, 1124, 1128, 1156, 1163, 1178)


def rank_seed(seed, rank):
    """The free-data seed of a rank: the validated list for the default seed,
    else seed + rank."""
    if seed == C3_SEEDS[0]:
        return C3_SEEDS[rank % len(C3_SEEDS)]
    return seed + rank


def perturb(z, rng, amp):
    """The free-data perturbation of workload(): per field, amp * |c_lead| *
    N(0,1) * exp(-k/8) on the coefficient of mode k (Delta and the shared
    cosine slot unchanged)."""
    z = np.array(z, dtype=np.float64)
    third = z.size // 3
    islot = 2 * third + 2
    for f in range(3):
        blk = z[f * third:(f + 1) * third]
        modes = np.arange(third) // 2 * 2 + (1 if f < 2 else 0)
        lead = np.max(np.abs(blk[:2]))
        noise = amp * lead * rng.standard_normal(third) * np.exp(-modes / 8.0)
        if f == 2:
            noise[islot - 2 * third] = 0.0
            noise[1] = 0.0
        z[f * third:(f + 1) * third] = blk + noise
    return z


SEEDS = REPO / "bench_data" / "dscan_seeds_128.npz"

# Fewest spatial points at which the reference's IRK fixed-point iteration
# converges on this problem, per Ntau (checked on the compiled reference: at
# Ntau = 1024 the converged fixture fails with 4000 and 6000 points, at the
# right boundary and mid-grid).  The workloads draw points from [min, 8000].
MIN_POINTS = {128: 2000, 256: 2000, 512: 4000, 1024: 8000}


def seed_request(eng, seeds, dim, ntau, points):
    """SimulationConfig and initial unknowns for dimension `dim`: the converged
    continuation solution at the nearest tabulated D (Ntau 128, 1000+1000
    points, bench_data/make_dscan_seeds.py), spectrally resampled to Ntau
    (create_simulation_data.py double) on NLeft = NRight = points/2."""
    i = int(np.argmin(np.abs(seeds["D"] - dim)))
    cfg = json.loads(str(seeds["config"]))
    cfg.update({"Dim": float(seeds["D"][i]), "Ntau": int(ntau), "NLeft": int(points) // 2,
                "NRight": int(points) // 2, "EpsNewton": 1e-7 if ntau <= 256 else 1e-8})
    fields = np.array([seeds["Up"][i], seeds["psic"][i], seeds["fc"][i]])
    if ntau != fields.shape[1]:
        fields = eng.resample(fields, ntau)
    z = eng.pack(ntau, fields[0], fields[1], fields[2])
    z[2 * z.size // 3 + 2] = seeds["delta"][i]
    return cfg, z


class Clocks:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(",") for r in Path(self.f.name).read_text().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].strip().replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].strip().replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            if len(r) < 9:
                continue
            for k, nm in enumerate(names):
                if "Active" in r[5 + k] and "Not" not in r[5 + k]:
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def traffic_per_launch():
    """DRAM bytes per launch of the march kernel from the committed ncu summary."""
    p = REPO / "profiles" / "march_c3.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.startswith("traffic_bytes_per_full_launch:"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1 and args.impl == "reference":
        return world, rank, local  # the CPU arm: rank 0 alone works, no collective is taken
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if args.dry_run:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        else:
            os.environ.setdefault("NCCL_DEBUG", "INFO")  # one communicator line per rank in the log
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def launch_ranks(args, argv):
    """`--gpus N` without an outer launcher: runs this script as N local ranks
    (one process per GPU) through torch.distributed.run on 127.0.0.1 and
    returns its exit code.  The ranks see WORLD_SIZE and do not re-launch."""
    import socket

    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={args.gpus}",
           "--master-addr=127.0.0.1", f"--master-port={port}", str(Path(__file__).resolve())] + argv
    env = dict(os.environ)
    env.setdefault("NCCL_DEBUG", "INFO")  # communicator set-up lines: one per rank
    env.setdefault("OMP_NUM_THREADS", "1")
    return subprocess.run(cmd, env=env).returncode


def run_dry(args, world, rank):
    """The multi-rank host path without a GPU (gloo): every rank partitions
    the C3 Jacobian's 768 columns, fills its block with known values, the
    all-gather assembles J, and the max-over-ranks reduction takes every
    rank's time; rank 0 prints the line the GPU run would print, marked dry."""
    import torch

    nn = 768
    blocks = column_blocks(nn, world)
    c0, c1 = blocks[rank]
    nb = max(b - a for a, b in blocks)
    local = torch.zeros(nb * nn, dtype=torch.float64)
    cols = torch.arange(c0, c1, dtype=torch.float64)[:, None] * nn + torch.arange(nn, dtype=torch.float64)[None, :]
    local[:(c1 - c0) * nn] = cols.reshape(-1)
    J = gather_columns(local, nn, blocks, world)
    expect = (torch.arange(nn, dtype=torch.float64)[None, :] * nn + torch.arange(nn, dtype=torch.float64)[:, None])
    ok = bool(torch.equal(J, expect))
    ok_all = max_over_ranks(world, 0.0 if ok else 1.0) == 0.0
    t = max_over_ranks(world, 1.0 + rank)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "dry_run": True, "n_gpus": world, "steps": args.steps,
                          "warmup": args.warmup, "blocks": blocks, "gather_ok": ok_all, "max_over_ranks": t,
                          "config": workload_config(args, world)}))


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def _dist_device():
    import torch.distributed as dist

    return "cuda" if dist.get_backend() == "nccl" else "cpu"


def max_over_ranks(world, v):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist

    t = torch.tensor([v], dtype=torch.float64, device=_dist_device())
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def column_blocks(nn, world):
    """Contiguous column partition of a Jacobian over `world` ranks (block
    sizes differ by at most one)."""
    base, extra = divmod(nn, world)
    out, c = [], 0
    for r in range(world):
        k = base + (1 if r < extra else 0)
        out.append((c, c + k))
        c += k
    return out


def gather_columns(local, nn, blocks, world):
    """All-gather of the ranks' column-major blocks (each padded to the largest
    block) -> the full J, row-major, on every rank."""
    import torch

    if world > 1:
        import torch.distributed as dist

        parts = [torch.empty_like(local) for _ in range(world)]
        dist.all_gather(parts, local)
    else:
        parts = [local]
    cols = [parts[r][:(c1 - c0) * nn].view(c1 - c0, nn) for r, (c0, c1) in enumerate(blocks)]
    return torch.cat(cols, 0).t().contiguous()


def workload_config(args, world):
    """The `config` of the bench line, the same dict in the engine and the
    reference arm: what the workload is, not how a run went."""
    return {"workload": "C3: D=4, Ntau=1024, 4000+4000 points, 768-column FD Jacobian, IRK2",
            "ntau": 1024, "points": 8000, "columns": 768, "seed": args.seed,
            "rank_seeds": [rank_seed(args.seed, r) for r in range(world)], "amp": args.amp,
            "l2": "GPU arm: flushed (256 MB write) before every timed build",
            "parallelism": f"{world} independent solves, one per GPU"}


def run_shard(args, world, rank, local):
    """One Jacobian split over the ranks by column blocks: every
    rank builds its contiguous block of columns of the same seeded C3 solve
    with one persistent launch, then one all-gather assembles J on every GPU.
    Strong scaling; time = max over ranks of (build + gather) device time."""
    import torch

    import pcc

    torch.cuda.set_device(local)
    eng = pcc.Engine(local)
    cfg, in0 = workload(args.seed, args.amp)  # the same solve on every rank
    solve = eng.solve(pcc.SolveDesc.from_config(cfg))
    nn = solve.nn
    out0 = solve.shoot(in0)
    blocks = column_blocks(nn, world)
    c0, c1 = blocks[rank]
    nb = max(b - a for a, b in blocks)
    d_in0 = torch.tensor(in0, dtype=torch.float64, device="cuda")
    d_out0 = torch.tensor(out0, dtype=torch.float64, device="cuda")
    d_cols = torch.zeros(nb * nn, dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step():
        solve.jacobian_columns_device(d_in0.data_ptr(), d_out0.data_ptr(), c0, c1, d_cols.data_ptr())
        st = solve.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        J = gather_columns(d_cols, nn, blocks, world)
        e1.record()
        torch.cuda.synchronize()
        return st["ms_total"] + e0.elapsed_time(e1), J

    for _ in range(args.warmup):
        step()
    barrier(world)
    ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        barrier(world)
        t, J = step()
        ms.append(t)
    total = max_over_ranks(world, float(np.sum(ms)))
    finite = bool(torch.isfinite(J).all().item())
    if rank == 0:
        print(json.dumps({"metric": METRIC, "value": args.steps / (total * 1e-3), "unit": "builds/s",
                          "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                          "ms_per_step": total / args.steps, "higher_is_better": True, "scaling": "strong",
                          "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded free data)",
                          "config": {"workload": "C3 Jacobian, columns sharded over the GPUs, one all-gather",
                                     "blocks": blocks, "finite": finite}}))
    solve.close()
    eng.close()


NATIVE_REF = REPO / "oracle" / "_ref" / "native" / "libpcc_ref.so"


def host_id():
    """This host and its CPU model, to tell whether a -march=native build of
    the reference was made here."""
    import platform

    model = ""
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                model = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    return f"{platform.node()} | {model}"


def build_native_reference():
    """Rebuilds the compiled reference's library -march=native on this host
    (as the reference's own build does), from the sources copied into
    oracle/_ref; returns (path or None, note).  Not timed."""
    NATIVE_REF.parent.mkdir(parents=True, exist_ok=True)
    if NATIVE_REF.exists():
        NATIVE_REF.unlink()
    env = dict(os.environ, PCC_REF_NATIVE="1")
    try:
        r = subprocess.run(["bash", str(REPO / "oracle" / "build_ref.sh")], env=env, capture_output=True,
                           text=True, timeout=900)
    except (OSError, subprocess.TimeoutExpired) as e:
        return None, f"native build failed ({e}); portable x86-64-v3 build used"
    if r.returncode != 0 or not NATIVE_REF.exists():
        return None, "native build failed (" + r.stderr.strip()[-200:] + "); portable x86-64-v3 build used"
    (NATIVE_REF.parent / "host.txt").write_text(host_id())
    return NATIVE_REF, "-march=native, built on this host before timing"


def reference_library():
    """The compiled reference to time: the -march=native build if it was made
    on this host, else the portable one."""
    marker = NATIVE_REF.parent / "host.txt"
    if NATIVE_REF.exists() and marker.exists() and marker.read_text() == host_id():
        return NATIVE_REF, "-march=native, built on this host"
    return REPO / "oracle" / "_ref" / "libpcc_ref.so", "portable x86-64-v3 build"


def cpu_reference(cfg, in0, out0, columns, threads, lib=None):
    """Times the reference's own OpenMP Jacobian loop on columns [0, columns):
    (seconds, the columns as rows x columns)."""
    sys.path.insert(0, str(REPO / "tests" / "golden"))
    from ref_lib import RefLib  # compiled reference (oracle/_ref)

    R = RefLib(lib) if lib else RefLib()
    t = time.perf_counter()
    cols = R.jacobian_columns(cfg, in0, out0, 0, columns, threads)
    return time.perf_counter() - t, cols


def run_reference(args, world, rank):
    if rank != 0:
        return
    cfg, in0 = workload(args.seed, args.amp)
    nn = in0.size
    sys.path.insert(0, str(REPO / "tests" / "golden"))
    from ref_lib import RefLib

    if not (REPO / "oracle" / "_ref" / "libpcc_ref.so").exists():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libpcc_ref.so was not built"}))
        return
    lib, build_note = build_native_reference()
    if lib is None:
        lib = REPO / "oracle" / "_ref" / "libpcc_ref.so"
    R = RefLib(lib)
    out0 = R.shoot(cfg, in0)
    threads = os.cpu_count() or 1
    cols = min(args.ref_columns or threads, nn)
    for _ in range(args.warmup):
        R.jacobian_columns(cfg, in0, out0, 0, 1, 1)
    times = [cpu_reference(cfg, in0, out0, cols, threads, lib)[0] for _ in range(args.steps)]
    per_build = np.array(times) * nn / cols
    value = 1.0 / float(np.mean(per_build))
    sample = (f"{cols} of {nn} Jacobian columns per step on {threads} threads, extrapolated x{nn / cols:.1f} "
              f"(a full 768-column build measured on 8 cores took 1.17x the extrapolation of an 8-column "
              f"sample: short samples run at burst clocks)"
              if cols < nn else f"all {nn} Jacobian columns per step on {threads} threads (full build)")
    line = {"metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": float(np.mean(per_build)) * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded free data)",
            "impl": "reference",
            "config": workload_config(args, world),
            "cpu_baseline": {"value": value, "unit": "builds/s", "cores": threads, "kind": "reference",
                             "sample": sample, "build": build_note},
            "e2e": {"value": value, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def variant_build(eng, cfg, in0, out0, J_head, steps, flush, **over):
    """C3 Jacobian builds of a solve with the SimulationConfig keys over
    changed: builds/s, RHS evaluations and the difference of its Jacobian
    from the headline build's J_head, relative to max |J|."""
    import torch

    import pcc

    s = eng.solve(pcc.SolveDesc.from_config(dict(cfg, **over)))
    nn = s.nn
    d_in0 = torch.tensor(in0, dtype=torch.float64, device="cuda")
    d_out0 = torch.tensor(out0, dtype=torch.float64, device="cuda")
    d_J = torch.empty((nn, nn), dtype=torch.float64, device="cuda")
    s.jacobian_device(d_in0.data_ptr(), d_out0.data_ptr(), d_J.data_ptr())
    s.sync()
    ms, rhs = [], 0
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        s.jacobian_device(d_in0.data_ptr(), d_out0.data_ptr(), d_J.data_ptr())
        st = s.sync()
        ms.append(st["ms_total"])
        rhs += st["rhs_evals"]
    J = d_J.cpu().numpy()
    s.close()
    return {"builds_per_s": steps / (float(np.sum(ms)) * 1e-3), "ms_per_build": float(np.mean(ms)),
            "rhs_evals_per_build": rhs / steps,
            "J_diff_vs_headline_rel_max": float(np.max(np.abs(J - J_head)) / np.max(np.abs(J_head))),
            "J_identical": bool(np.array_equal(J, J_head))}


def predictor_build(eng, cfg, in0, out0, J_head, steps, flush):
    """C3 Jacobian builds with the optional stage predictor (each step's
    fixed-point iteration starts from the previous step's collocation
    polynomial; not in the reference)."""
    r = variant_build(eng, cfg, in0, out0, J_head, steps, flush, IRKPredictor=True)
    r["note"] = ("stage iteration started from the previous step's collocation polynomial (not in the "
                 "reference); same fixed point to PrecisionIRK")
    return r


def both_sides_build(eng, cfg, in0, out0, J_head, steps, flush):
    """C3 Jacobian builds in the reference's schedule: every column marches
    both sides (ShootBothSides); the headline build marches only the side a
    column's free datum feeds and takes the other from the base shoot."""
    import pcc

    r = variant_build(eng, cfg, in0, out0, J_head, steps, flush, ShootBothSides=True)
    n = int(cfg["Ntau"])
    nn = 3 * n // 4
    r["sweeps_per_build"] = int(len(pcc.sweep_plan(n, 0, nn, shoot_both_sides=True)))
    r["headline_sweeps_per_build"] = int(len(pcc.sweep_plan(n, 0, nn)))
    r["note"] = "every column shoots both sides (NewtonSolver.cpp:615-650 schedule); J_identical compares bits"
    return r


def newton_compare(eng, cfg, in0, out0, J):
    """C3 Newton steps: the batched form (base shoot and all 768 columns in one
    persistent launch, device-side Newton update) with the mixed-precision and
    the FP64 solve, against the plain FP64 GPU form (one march launch per
    shoot, 2 sweeps each, FP64 LU), timed on a column sample and extrapolated."""
    import pcc

    s = eng.solve(dict(cfg, PrecisionNewton=1e-30, MaxIterNewton=1000))
    nn = s.nn
    out = {"workload": "C3 (Ntau 1024, 4000+4000 points), one Newton iteration from the bench's seeded data"}
    for name, prec in [("batched_mixed", pcc.PREC_MIXED), ("batched_fp64", pcc.PREC_FP64)]:
        s.newton_begin(in0)
        t = time.perf_counter()
        st = eng.newton_iterate([s], precision=prec)[0]
        out[f"ms_{name}"] = (time.perf_counter() - t) * 1e3
        if prec == pcc.PREC_MIXED:
            out["mixed_lu_refinement_steps"] = st["lu_refinement_steps"]
            out["mixed_lu_fell_back_to_fp64"] = st["lu_fell_back"]
    sample = 8
    t = time.perf_counter()
    for c in range(sample):
        s.jacobian_columns(in0, out0, c, c + 1)
    per_col = (time.perf_counter() - t) / sample
    b = -np.asarray(out0)
    for prec in (pcc.PREC_FP64, pcc.PREC_MIXED):
        eng.lu_solve(J, b, precision=prec)  # first calls set the kernels' shared-memory limits
    t = time.perf_counter()
    x64, rep64 = eng.lu_solve(J, b, precision=pcc.PREC_FP64)
    lu_ms = (time.perf_counter() - t) * 1e3
    xm, rep = eng.lu_solve(J, b, precision=pcc.PREC_MIXED)
    old_tc = os.environ.get("PCC_LU_TC")
    os.environ["PCC_LU_TC"] = "0"
    eng.lu_solve(J, b, precision=pcc.PREC_MIXED)
    xc, repc = eng.lu_solve(J, b, precision=pcc.PREC_MIXED)
    if old_tc is None:
        os.environ.pop("PCC_LU_TC")
    else:
        os.environ["PCC_LU_TC"] = old_tc
    x_lapack = np.linalg.solve(J, b)  # LAPACK dgesv (numpy)
    out["lu"] = {"n": nn, "ms_fp64": rep64["ms"], "ms_mixed_tensor_cores": rep["ms"],
                 "ms_mixed_cuda_cores": repc["ms"], "refinement_steps": rep["refinement_steps"],
                 "fell_back_to_fp64": rep["fell_back_to_fp64"],
                 "mixed_tc_dx_rel_err_vs_lapack_dgesv": float(np.linalg.norm(xm - x_lapack) /
                                                              np.linalg.norm(x_lapack)),
                 "mixed_cuda_cores_dx_rel_err_vs_lapack_dgesv": float(np.linalg.norm(xc - x_lapack) /
                                                                      np.linalg.norm(x_lapack)),
                 "what": "device time of one solve (factorisation, solve, refinement) on the timed build's J; "
                         "mixed = FP32 LU (trailing updates on tcgen05 TF32 high/low, or on the CUDA cores) "
                         "+ FP64 refinement"}
    out["ms_plain_fp64"] = per_col * (nn + 1) * 1e3 + lu_ms
    out["plain_form"] = (f"one march launch per shoot (base + {nn} columns); {sample} columns timed, "
                         f"extrapolated; FP64 LU {lu_ms:.1f} ms")
    out["speedup_batched_mixed_vs_plain_fp64"] = out["ms_plain_fp64"] / out["ms_batched_mixed"]
    out["speedup_batched_mixed_vs_batched_fp64"] = out["ms_batched_fp64"] / out["ms_batched_mixed"]
    out["mixed_dx_rel_err_vs_fp64"] = float(np.linalg.norm(xm - x64) / np.linalg.norm(x64))
    out["mixed_dx_rel_err_vs_lapack_dgesv"] = float(np.linalg.norm(xm - x_lapack) / np.linalg.norm(x_lapack))
    out["fp64_dx_rel_err_vs_lapack_dgesv"] = float(np.linalg.norm(x64 - x_lapack) / np.linalg.norm(x_lapack))
    s.close()
    return out


def run_dscan(eng, args):
    """C4: 16 solves, D = 3.25, 3.35, .., 4.75, Ntau drawn from {128, 256, 512,
    1024} and points from {2000, 4000, 6000, 8000} (seeded; at least
    MIN_POINTS[Ntau]), seeded free data, batched: one Newton iteration of all
    16 in one batch launch timed alone (Jacobian builds/s), then all 16 to
    convergence (NewtonSolver::run for each, every iteration's shoots of every
    running solve in one launch, mixed-precision solve)."""
    import pcc

    if not SEEDS.exists():
        return {"unavailable": "bench_data/dscan_seeds_128.npz missing (bench_data/make_dscan_seeds.py)"}
    seeds = np.load(SEEDS)
    rng = np.random.default_rng(args.seed + 4)
    dims = 3.25 + 0.1 * np.arange(16)
    ns = rng.choice([128, 256, 512, 1024], 16)
    pts = [int(rng.choice([p for p in (2000, 4000, 6000, 8000) if p >= MIN_POINTS[int(n)]])) for n in ns]
    solves, xs, rejects, cfgs = [], [], [], []
    for d, n, p in zip(dims, ns, pts):
        for attempt in range(4):
            cfg, z = seed_request(eng, seeds, d, int(n), int(p))
            z = perturb(z, rng, args.dscan_amp)
            s = eng.solve(dict(cfg, PrecisionNewton=1e-30, MaxIterNewton=1000))
            try:
                s.shoot(z)  # the base shoot must converge (else re-draw, logged)
                break
            except pcc.PccError as e:
                rejects.append({"D": float(d), "ntau": int(n), "points": int(p), "why": e.name})
                s.close()
                s = None
        if s is not None:
            solves.append(s)
            xs.append(z)
            cfgs.append(cfg)
    for s, z in zip(solves, xs):  # warm-up iteration
        s.newton_begin(z)
    eng.newton_iterate(solves, precision=pcc.PREC_MIXED)
    for s, z in zip(solves, xs):
        s.newton_begin(z)
    st = pcc.Stats()
    t = time.perf_counter()
    eng.newton_iterate(solves, precision=pcc.PREC_MIXED, stats=st)
    wall = time.perf_counter() - t
    for s in solves:
        s.close()
    # the same 16 solves to convergence
    tol = 1e-10
    conv = [eng.solve(dict(c, PrecisionNewton=tol, MaxIterNewton=args.dscan_iters)) for c in cfgs]
    t = time.perf_counter()
    x_out, states = eng.newton_solve(conv, xs, precision=pcc.PREC_MIXED)
    wall_conv = time.perf_counter() - t
    for s in conv:
        s.close()
    return {"solves": len(solves), "rejected_draws": rejects,
            "ntau": [int(c["Ntau"]) for c in cfgs], "points": [int(c["NLeft"] + c["NRight"]) for c in cfgs],
            "dims_requested": [float(d) for d in dims], "dims": [float(c["Dim"]) for c in cfgs],
            "wall_s": wall, "jacobian_builds_per_s": len(solves) / wall, "ms_batch_march": st.ms_sweep,
            "rhs_evals": st.rhs_evals,
            "sweeps": int(sum(len(pcc.sweep_plan(int(c["Ntau"]), 0, 3 * int(c["Ntau"]) // 4)) for c in cfgs)),
            "converge": {"tolerance": tol, "max_iterations": args.dscan_iters, "wall_s": wall_conv,
                         "states": [x["state"] for x in states], "iterations": [x["iterations"] for x in states],
                         "err": [x["err"] for x in states],
                         "delta": [float(x[2 * x.size // 3 + 2]) for x in x_out]},
            "free_data_amp": args.dscan_amp, "lu": "mixed (FP32 LU on tensor cores + FP64 refinement)"}


def serving_requests(eng, args, n_req):
    """C5's seeded request stream: D ~ U[3.25, 4.75] (the nearest dimension of
    the seed table, 0.01 apart), Ntau from {128, 256, 512, 1024}, points ~
    U[MIN_POINTS[Ntau], 8000] (even)."""
    seeds = np.load(SEEDS)
    rng = np.random.default_rng(args.seed + 5)
    reqs = []
    for _ in range(n_req):
        d = rng.uniform(3.25, 4.75)
        n = int(rng.choice([128, 256, 512, 1024]))
        p = 2 * int(rng.integers(MIN_POINTS[n] // 2, 4001))
        cfg, z = seed_request(eng, seeds, d, n, p)
        cfg.update({"PrecisionNewton": 1e-10, "MaxIterNewton": 10})
        reqs.append((cfg, z, d))
    return reqs, rng


def run_serving(eng, args, rate, n_req, precision="fp64"):
    """C5 at one arrival rate: a seeded Poisson stream of whole Newton solves;
    latency = submit -> result (host clock), service = latency minus the time
    queued before admission."""
    import pcc

    if not SEEDS.exists():
        return {"unavailable": "bench_data/dscan_seeds_128.npz missing (bench_data/make_dscan_seeds.py)"}
    reqs, rng = serving_requests(eng, args, n_req)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, n_req))
    prec = pcc.PREC_MIXED if precision == "mixed" else pcc.PREC_FP64
    eng.serve_start()
    t0 = time.perf_counter()
    tickets = []
    for (cfg, z, _), a in zip(reqs, arrivals):
        dt = t0 + a - time.perf_counter()
        if dt > 0:
            time.sleep(dt)
        tickets.append(eng.submit(cfg, z, precision=prec))
    res = [eng.wait(t, 3600.0)[0] for t in tickets]
    span = time.perf_counter() - t0
    info = eng.serve_stats()
    eng.serve_stop()
    lat = np.array([r["ms_latency"] for r in res])
    svc = np.array([r["ms_latency"] - r["ms_queued"] for r in res])
    q = np.array([r["ms_queued"] for r in res])
    return {"rate_per_s": rate, "requests": n_req, "precision": precision,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "service_p50_ms": float(np.percentile(svc, 50)),
            "service_p99_ms": float(np.percentile(svc, 99)), "queued_p50_ms": float(np.percentile(q, 50)),
            "queued_p99_ms": float(np.percentile(q, 99)),
            "throughput_solves_per_s": n_req / span, "span_s": span,
            "converged": int(sum(r["newton"]["state"] == "CONVERGED" for r in res)),
            "statuses": sorted(set(r["status_name"] for r in res)),
            "iterations_mean": float(np.mean([r["newton"]["iterations"] for r in res])),
            "ntau": [c["Ntau"] for c, _, _ in reqs], "dims_requested": [float(d) for _, _, d in reqs],
            "dims": [float(c["Dim"]) for c, _, _ in reqs], "launches": info["launches"],
            "sweeps": info["sweeps"], "newton_tolerance": 1e-10,
            "note": "percentiles over `requests` draws (with 16 the p99 is the maximum)"}


def run_lu_case(args, local):
    """A profiling case for the dense solve: a seeded n x n system with
    singular values graded from 1 to 1e-6, solved in FP64 and in mixed
    precision; prints the refine reports and the errors against numpy's
    LAPACK dgesv."""
    import torch

    import pcc

    torch.cuda.set_device(local)
    eng = pcc.Engine(local)
    n = args.lu
    rng = np.random.default_rng(768)
    u, _ = np.linalg.qr(rng.standard_normal((n, n)))
    v, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (u * np.logspace(0, -6, n)) @ v.T
    b = rng.standard_normal(n)
    xn = np.linalg.solve(A, b)
    for prec in (pcc.PREC_FP64, pcc.PREC_MIXED):
        x, rep = eng.lu_solve(A, b, precision=prec)
        print(json.dumps({"lu_case": n, "precision": prec, **rep,
                          "rel_err_vs_dgesv": float(np.linalg.norm(x - xn) / np.linalg.norm(xn))}))
    eng.close()


def run_serving_only(args, local):
    """C5 alone, for a longer measurement than the bench line carries: one
    JSON line per (rate, precision)."""
    import torch

    import pcc

    torch.cuda.set_device(local)
    eng = pcc.Engine(local)
    for prec, rates in (("fp64", args.rates), ("mixed", args.mixed_rates)):
        for r in rates.split(","):
            if r:
                print(json.dumps({"serving": run_serving(eng, args, float(r), args.requests, prec)}), flush=True)
    eng.close()


def run_engine(args, world, rank, local):
    import torch

    import pcc

    torch.cuda.set_device(local)
    eng = pcc.Engine(local)
    cfg, in0 = workload(rank_seed(args.seed, rank), args.amp)
    solve = eng.solve(pcc.SolveDesc.from_config(dict(cfg, ShootBothSides=args.both_sides)))
    nn, n = solve.nn, solve.ntau
    out0 = solve.shoot(in0)  # base shoot (the Newton step's, outside the build)

    d_in0 = torch.tensor(in0, dtype=torch.float64, device="cuda")
    d_out0 = torch.tensor(out0, dtype=torch.float64, device="cuda")
    d_J = torch.empty((nn, nn), dtype=torch.float64, device="cuda")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    torch.cuda.synchronize()

    if args.columns:
        # a profiling case: columns [0, C) through the host ABI, one march launch per step
        for _ in range(args.warmup + args.steps):
            st = {}
            solve.jacobian_columns(in0, out0, 0, args.columns, stats=st)
            print(json.dumps({"profile_case": True, "columns": args.columns, **st}))
        solve.close()
        eng.close()
        return

    for _ in range(args.warmup):
        solve.jacobian_device(d_in0.data_ptr(), d_out0.data_ptr(), d_J.data_ptr())
        solve.sync()

    clocks = Clocks(local)
    barrier(world)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dev_ms, sweep_ms, rhs = [], [], 0
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        solve.jacobian_device(d_in0.data_ptr(), d_out0.data_ptr(), d_J.data_ptr())
        st = solve.sync()
        dev_ms.append(st["ms_total"])
        sweep_ms.append(st["ms_sweep"])
        rhs += st["rhs_evals"]
    torch.cuda.synchronize()
    barrier(world)
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    total_ms = max_over_ranks(world, float(np.sum(dev_ms)))
    ms_per_step = total_ms / args.steps
    value = world * args.steps / (total_ms * 1e-3)

    # end to end: the host C-ABI call with pinned host buffers, copies included
    h_in0 = torch.tensor(in0, dtype=torch.float64).pin_memory()
    h_out0 = torch.tensor(out0, dtype=torch.float64).pin_memory()
    h_J = torch.empty((nn, nn), dtype=torch.float64).pin_memory()
    lib = pcc.load()
    D = pcc._D
    import ctypes

    def ptr(t):
        return ctypes.cast(ctypes.c_void_p(t.data_ptr()), D)

    st_e = pcc.Stats()
    barrier(world)
    t1 = time.perf_counter()
    for _ in range(args.steps):
        r = lib.pcc_jacobian(solve.h, ptr(h_in0), ptr(h_out0), ptr(h_J), ctypes.byref(st_e))
        if r != 0:
            raise pcc.PccError(r, lib.pcc_last_error(eng.ctx).decode())
    barrier(world)
    e2e_s = max_over_ranks(world, time.perf_counter() - t1)
    e2e = {"value": world * args.steps / e2e_s, "unit": "builds/s", "h2d_bytes_per_step": 2 * nn * 8,
           "d2h_bytes_per_step": nn * nn * 8}
    if not np.all(np.isfinite(h_J.numpy())):
        raise RuntimeError("non-finite Jacobian")

    peak = eng.fp64_peak_tflops()
    flops_per_launch = (rhs / args.steps) * f_rhs(n)
    achieved = flops_per_launch / (np.mean(sweep_ms) * 1e-3) / 1e12
    roofline = {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "traffic": traffic_per_launch(), "kernel": "march_kernel<1024,2>",
                "peak_source": "in-run FP64 FMA probe (MEASURED_PEAKS.json has no FP64 figure)",
                "flops_per_launch": flops_per_launch, "rhs_evals_per_launch": rhs / args.steps,
                "flop_convention": "7*5*N*log2(N) + 100*N per RHS evaluation (reference algorithm)"}

    # the further sections go into rank 0's line only, so only rank 0 runs
    # them (after the last collective): another rank's seed need not suit them
    extras = rank == 0 and not args.quick
    predictor = predictor_build(eng, cfg, in0, out0, h_J.numpy().copy(), args.steps, flush) if extras else None
    both_sides = both_sides_build(eng, cfg, in0, out0, h_J.numpy().copy(), args.steps, flush) if extras else None
    newton = newton_compare(eng, cfg, in0, out0, h_J.numpy().copy()) if extras else None
    dscan = run_dscan(eng, args) if extras else None
    serving = None
    if extras:
        serving = [run_serving(eng, args, float(r), args.requests) for r in args.rates.split(",") if r]
        serving += [run_serving(eng, args, float(r), args.requests, "mixed") for r in args.mixed_rates.split(",")
                    if r]

    cpu, parity = None, None
    if rank == 0 and world == 1 and not args.no_cpu:
        ref_so = REPO / "oracle" / "_ref" / "libpcc_ref.so"
        threads = os.cpu_count() or 1
        cols = min(threads, nn)
        if ref_so.exists():
            lib, build_note = reference_library()
            t, J_ref = cpu_reference(cfg, in0, out0, cols, threads, lib)
            cpu = {"value": (cols / nn) / t, "unit": "builds/s", "cores": threads, "kind": "reference",
                   "sample": f"{cols} of {nn} Jacobian columns on {threads} threads ({t:.1f} s), extrapolated",
                   "build": build_note}
            # the timed build's own columns against the reference's on the same input
            J_gpu = h_J.numpy()[:, :cols]
            parity = {"J_rel": float(np.max(np.abs(J_gpu - J_ref)) / np.max(np.abs(J_ref))), "columns": cols,
                      "tolerance": 2e-5,
                      "what": "max |J_gpu[:, c] - J_ref[:, c]| / max |J_ref| over the CPU baseline's columns "
                              "c < columns of this input (reference: oracle/_ref, NewtonSolver::shoot per column)"}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded free data)",
                "config": workload_config(args, world),
                "run": {"sweep_ctas": st_e.sweep_ctas, "wall_s": wall, "march_schedule": eng.march_tuning(n, 2),
                        "sweeps_per_build": int(len(pcc.sweep_plan(n, 0, nn, shoot_both_sides=args.both_sides))),
                        "side_reuse": not args.both_sides},
                "clocks": clk, "e2e": e2e, "gpu_launches": 4 * args.steps, "roofline": roofline,
                "cpu_baseline": cpu, "parity": parity, "predictor": predictor, "both_sides": both_sides, "newton_step": newton,
                "dscan16": dscan, "serving": serving}
        print(json.dumps(line))
    solve.close()
    eng.close()


def main():
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--seed", type=int, default=1024)
    ap.add_argument("--amp", type=float, default=0.1)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--quick", action="store_true", help="only the Jacobian build line (no Newton/C4/C5 sections)")
    ap.add_argument("--rates", default="0.25,1,4,16",
                    help="C5 Poisson arrival rates (requests/s), FP64 Newton solves; 0.25 is below capacity")
    ap.add_argument("--mixed-rates", default="4", help="C5 rates served again with the mixed-precision solve")
    ap.add_argument("--requests", type=int, default=16, help="C5 requests per rate")
    ap.add_argument("--dscan-iters", type=int, default=20, help="C4: Newton iteration cap of the convergence run")
    ap.add_argument("--dscan-amp", type=float, default=0.01, help="C4 free-data perturbation amplitude")
    ap.add_argument("--shard", choices=["solves", "columns"], default="solves",
                    help="multi-GPU: independent solves per GPU (weak scaling, default) or one Jacobian's "
                         "columns split over the GPUs and all-gathered (strong scaling)")
    ap.add_argument("--ref-columns", type=int, default=0,
                    help="--impl reference: columns timed per step (default one per host thread; "
                         "the Jacobian's column count times a full build)")
    ap.add_argument("--columns", type=int, default=0,
                    help="profiling aid: build only the first C columns (not a benchmark line)")
    ap.add_argument("--both-sides", action="store_true",
                    help="every Jacobian column marches both sides (ShootBothSides, the reference's schedule) "
                         "instead of only the side its free datum feeds; with --columns 148 a profiling case of "
                         "exactly 296 sweeps (one wave)")
    ap.add_argument("--lu", type=int, default=0,
                    help="profiling aid: pcc_lu_solve, FP64 then mixed, on a seeded n x n system of condition "
                         "number 1e6 (prints the refine reports, not a benchmark line)")
    ap.add_argument("--serving-only", action="store_true",
                    help="only C5: one JSON line per rate (--rates FP64, --mixed-rates mixed), no bench line")
    ap.add_argument("--dry-run", action="store_true",
                    help="no GPU: the rank launch and multi-rank host logic on gloo (a test of the launcher)")
    args = ap.parse_args()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(launch_ranks(args, sys.argv[1:]))
    world, rank, local = dist_setup(args)
    if world != args.gpus and rank == 0:
        print(f"bench.py: {world} ranks for --gpus {args.gpus}; the line reports the ranks that ran",
              file=sys.stderr)
    try:
        if args.dry_run:
            run_dry(args, world, rank)
        elif args.serving_only:
            run_serving_only(args, local)
        elif args.lu:
            run_lu_case(args, local)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        elif args.shard == "columns":
            run_shard(args, world, rank, local)
        else:
            run_engine(args, world, rank, local)
    finally:
        if world > 1 and args.impl != "reference":
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()
