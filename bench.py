#!/usr/bin/env python
"""Benchmark of the B200 iSVD hot path (one JSON line on rank 0).

Workload (default): the plain-FP64-at-scale configuration -- A = U_r diag(sigma)
V_r' + 1e-4 G with m = 100000, n = 20000 (16 GB FP64, row-major), r = 200,
sigma_j = exp(-j/30); k = 50, p = 14 (l = 64), N = 64 sketches (sketch GEMM
100000 x 20000 x 4096); Gramian orthogonalizer, row-block Gramian
Kolmogorov-Nagumo integrator (tol 1e-6, at most 256 iterations), row-block
Gramian former.  A step is one whole solve (Omega drawn on the device, sketch,
orthogonalize, integrate, form) with A resident in HBM.  Synthetic data
(seeded; no dataset exists for this path).  A (16 GB) is larger than L2, so no
flush is needed between steps.

Arms:
  default            this build (libmcnla_b200.so); value = iSVD/s over all ranks
  --impl reference   the reference's own CPU stages (oracle/_ref, built from the
                     reference sources; the numpy restatement when absent) on a
                     bounded row sample of the same workload, all host threads
N > 1 runs independent replicas (one solve per GPU per step, no collective in
the data path: the one-GPU solve does not shard); torch.distributed is used for
the barrier and the max-over-ranks time only.
"""
import argparse
import ctypes
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "iSVD/s & A-read GB/s, mixed vs FP64 plain on B200 at σ err≤1e-6; p50/p99 ms"

# dram bytes (read + write) per row of A for one launch of the sketch GEMM, from
# one ncu capture (dram__bytes_read.sum + dram__bytes_write.sum: 22.48 GB +
# 0.53 GB) of the 16384 x 20000 x 4096 case with the 64 x 128 two-CTA tile;
# scaled by rows to the benchmark's m (A is re-read ~8.6x through L2)
SKETCH_TRAFFIC_PER_ROW = (22.475526e9 + 0.534837e9) / 16384


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--m", type=int, default=100000)
    ap.add_argument("--n", type=int, default=20000)
    ap.add_argument("--k", type=int, default=50)
    ap.add_argument("--p", type=int, default=14)
    ap.add_argument("--N", type=int, default=64)
    ap.add_argument("--rank-r", type=int, default=200)
    ap.add_argument("--integrator", default="rb_gramian_kn")
    ap.add_argument("--former", default="rb_gramian")
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--maxit", type=int, default=256)
    ap.add_argument("--colmajor", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--no-row-block", action="store_true", help="N > 1: skip the row-block (one matrix over all ranks) leg")
    ap.add_argument("--cpu-rows", type=int, default=0, help="row sample of the CPU baseline (0: auto)")
    ap.add_argument("--ref-budget", type=float, default=420.0,
                    help="reference arm: seconds of timed full solves; no step starts that would end past it")
    ap.add_argument("--quick", action="store_true", help="small shape for a smoke run")
    ap.add_argument("--no-serving", action="store_true", help="skip the batched / served leg")
    ap.add_argument("--kernel", choices=["sketch_bf16", "gkn", "trace", "grouped", "served_trace", "gkn_scaling",
                                         "ingest", "syev", "inverse"],
                    default=None,
                    help="time one kernel alone (profiling case) instead of the benchmark: the BF16 sketch GEMM "
                         "on --m x --n x (--k + --p) --N with --parts parts, or the persistent row-block Gramian "
                         "KN integrator on the sketches of a seeded --m x --n matrix (sigma_j = 1/j, tol 1e-5); "
                         "trace: per-kernel device time (CUPTI activity records, no replay) of one FP64 and one "
                         "mixed solve of the workload, and the per-iteration share from maxit 65 vs 257")
    ap.add_argument("--only-serving", action="store_true", help="run the batched / served leg alone")
    ap.add_argument("--batch-count", type=int, default=1024, help="matrices in the uneven batch")
    ap.add_argument("--serve-workers", type=int, default=8, help="concurrent solves of the server")
    ap.add_argument("--serve-pool", type=int, default=256, help="distinct resident matrices the requests use")
    ap.add_argument("--serve-rates", default="200,1000,5000", help="Poisson arrival rates, requests/s")
    ap.add_argument("--serve-rates-fp64", default="200,1000",
                    help="arrival rates also served in plain FP64 (the same arrivals as the mixed ones)")
    ap.add_argument("--serve-seconds", type=float, default=0.5, help="arrival window per rate (>= 400 requests)")
    ap.add_argument("--serve-integrator", default="rb_gramian_kn", help="KN integrator of the batched / served solves")
    ap.add_argument("--serve-former", default="rb_gramian",
                    help="former of the batched / served solves (the row-block driver's pairing by default)")
    ap.add_argument("--parts", type=int, default=2, help="BF16 parts of A in the mixed leg (2: 16 bits, 3: 24 bits)")
    ap.add_argument("--former-parts", type=int, default=3, choices=[0, 1, 2, 3],
                    help="BF16 parts of A' for the mixed leg's former (0: the former reads the FP64 A)")
    ap.add_argument("--serve-parts", type=int, default=3, help="BF16 parts of A in the batched / served mixed solves")
    args = ap.parse_args()
    if args.quick:
        args.m, args.n, args.k, args.p, args.N, args.rank_r = 8192, 4096, 16, 8, 16, 64
        args.batch_count, args.serve_pool, args.serve_seconds = 64, 32, 0.1
    return args


def workload(args):
    l = args.k + args.p
    return {
        "workload": "plain FP64 iSVD, A = U diag(exp(-j/30)) V' + 1e-4 G, m=%d n=%d r=%d, k=%d p=%d N=%d"
                    % (args.m, args.n, args.rank_r, args.k, args.p, args.N),
        "m": args.m, "n": args.n, "k": args.k, "p": args.p, "l": l, "N": args.N,
        "sketch_gemm": "%dx%dx%d" % (args.m, args.n, l * args.N),
        "stages": "GaussianProjection(device Philox) / Gramian / %s (tol %g, maxit %d) / %s"
                  % (args.integrator, args.tol, args.maxit, args.former),
        "layout": "column-major" if args.colmajor else "row-major",
        "l2": "inputs larger than L2 (A is %.1f GB)" % (args.m * args.n * 8 / 1e9),
    }


# ------------------------------------------------------------------------------------------------
# distributed plumbing
# ------------------------------------------------------------------------------------------------
def dist_init(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if args.impl == "b200":
            torch.cuda.set_device(local)
        dist.init_process_group("nccl" if args.impl == "b200" else "gloo",
                                timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    """Largest value of x over the ranks (a CUDA tensor on NCCL, a CPU tensor on gloo)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# ------------------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ["clocks.sm", "clocks.max.sm", "power.draw", "clocks_event_reasons.hw_slowdown",
              "clocks_event_reasons.hw_thermal_slowdown", "clocks_event_reasons.sw_thermal_slowdown",
              "clocks_event_reasons.sw_power_cap"]

    def __init__(self, device_index):
        import torch
        self.proc = None
        try:
            uuid = "GPU-" + str(torch.cuda.get_device_properties(device_index).uuid)
        except Exception:
            uuid = str(device_index)
        self.cmd = ["nvidia-smi", "-i", uuid, "--query-gpu=" + ",".join(self.FIELDS),
                    "--format=csv,noheader,nounits", "-lms", "200"]

    def start(self):
        try:
            self.proc = subprocess.Popen(self.cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) != len(self.FIELDS):
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": max(mx), "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------------------
# this build
# ------------------------------------------------------------------------------------------------
def _measured_peak(key):
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)[key])
    except Exception:
        return {"bf16_tflops": 1590.0, "hbm_gbs": 6650.0}.get(key)


def fp64_peak_tflops():
    """cuBLAS DGEMM throughput on this GPU (the FP64 roofline denominator; no FP64
    figure is in the measured-peaks file).  Best of 5 at 8192^3, after warm-up."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    c = a @ b
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b, c
    return 2 * n ** 3 / best / 1e12


def stage_rooflines(m, n, k, l, N, integrator, former, stages, peak_tflops, hbm_gbs):
    """Per-stage roofline of the FP64 solve: algorithmic flops and HBM bytes of each
    stage (the minimum any implementation must do), the stage's roofline time
    max(flops / FP64 tensor peak, bytes / HBM peak), and frac = roofline time /
    measured time.  Integrator flops count the products each iteration needs at
    this shape, times the measured iteration count."""
    L = N * l
    it = stages["integrate_iterations"]
    per_it = {
        # B = Qs'Qc, X = Qs B - Qc D, Z = X'X, Qc+ = [Qc X][C; inv(C)]
        "kn": 4 * m * L * l + 8 * m * l * l,
        # G = Qs B / N, Bg = Qs'G, Q+ = [Qc G][F; inv(C)], D, Dg
        "rb_kn": 4 * m * L * l + 4 * m * l * l + 4 * L * l * l,
        # Bg = Bs B, [D | Dg] = B'[B | Bg], E~+, B+
        "rb_gramian_kn": 2 * L * L * l + 4 * L * l * l + 8 * L * l * l,
        "rb_wy": 4 * m * L * l + 8 * m * l * l,
        "rb_gramian_wy": 2 * L * L * l + 12 * L * l * l,
    }[integrator]
    once = {"rb_gramian_kn": L * L * m + 2 * m * L * l, "rb_gramian_wy": L * L * m + 2 * m * L * l}.get(integrator, 0)
    integ_bytes = 8 * m * L + 8 * m * l + (8 * L * L if "gramian" in integrator else 0)
    if former == "svd":
        form_flops = 2 * m * n * l + 2 * m * l * k
    else:
        form_flops = 2 * m * n * l + 2 * n * l * l + 2 * m * l * k + 2 * n * l * k
    rows = {
        "sketch": (2 * m * n * L, 8 * (m * n + n * L + m * L), stages["sketch_gemm_s"]),
        "orthogonalize": (4 * m * l * L, 8 * 3 * m * L, stages["orthogonalize_s"]),
        "integrate": (once + per_it * it, integ_bytes, stages["integrate_s"]),
        "form": (form_flops, 8 * (m * n + m * l + n * k + m * k), stages["form_s"]),
    }
    out = {}
    for name, (fl, by, t) in rows.items():
        t_c, t_m = fl / (peak_tflops * 1e12), by / (hbm_gbs * 1e9)
        out[name] = {"bound": "tensor" if t_c >= t_m else "hbm", "flops": float(fl), "bytes": float(by),
                     "s": round(t, 6), "achieved_tflops": round(fl / t / 1e12, 3),
                     "achieved_gbs": round(by / t / 1e9, 1), "frac": round(max(t_c, t_m) / t, 4)}
    out["peaks"] = {"fp64_tflops": round(peak_tflops, 3), "hbm_gbs": hbm_gbs,
                    "source": "FP64: cuBLAS DGEMM measured in this run; HBM: MEASURED_PEAKS.json hbm_gbs of measured"}
    return out


def run_config1_b200(args, dev):
    """Configuration 1 in full on this build: device-resident A and Omega (value), and the same
    through mcnla_b200_isvd_host with pinned host A and Omega in and S/U/V out (e2e)."""
    import torch
    from mcnla_b200 import isvd
    a_np, om_np = config1_inputs()
    a = torch.as_tensor(a_np, device=dev)
    om = torch.as_tensor(om_np, device=dev)
    stream = torch.cuda.current_stream(dev)
    kw = dict(integrator="kn", former="svd", maxit=256, tol=1e-4)
    for _ in range(max(1, args.warmup)):
        s, u, v, it = isvd.solve(a, 10, 10, 16, omega=om, **kw)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s, u, v, it = isvd.solve(a, 10, 10, 16, omega=om, **kw)
    e1.record(stream)
    torch.cuda.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / args.steps
    a_h = torch.from_numpy(a_np).pin_memory()
    om_h = torch.from_numpy(om_np).pin_memory()
    out = (torch.empty(10, dtype=torch.float64, pin_memory=True),
           torch.empty(1000, 10, dtype=torch.float64, pin_memory=True),
           torch.empty(2000, 10, dtype=torch.float64, pin_memory=True))
    isvd.solve_host(a_h, om_h, 10, 10, 16, out=out, device=dev, **kw)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        isvd.solve_host(a_h, om_h, 10, 10, 16, out=out, device=dev, **kw)
    e1.record(stream)
    torch.cuda.synchronize()
    t_e2e = e0.elapsed_time(e1) / 1e3 / args.steps
    return {**CONFIG1, "value": round(1.0 / t, 3), "unit": "iSVD/s", "ms_per_step": round(t * 1e3, 4),
            "steps": args.steps, "iterations": it,
            "e2e": {"value": round(1.0 / t_e2e, 3), "unit": "iSVD/s", "h2d_bytes_per_step": int((a_np.size + om_np.size) * 8),
                    "d2h_bytes_per_step": int((10 + 1000 * 10 + 2000 * 10) * 8)},
            "reconstruction_rel_err": reconstruction_error_torch(a, s, u, v),
            "sigma": [float(x) for x in s[:3].tolist()]}


def _svd_metrics(s, u, s_ref, u_ref):
    """sigma relative error, largest principal angle between the U subspaces, ||U'U - I||_F."""
    import numpy as np
    k = s.shape[0]
    rel = float(np.max(np.abs(s - s_ref[:k]) / s_ref[:k]))
    cosmin = np.clip(np.linalg.svd(u_ref[:, :k].T @ u, compute_uv=False).min(), -1.0, 1.0)
    orth = float(np.linalg.norm(u.T @ u - np.eye(k)))
    return {"sigma_rel_err": rel, "max_principal_angle_U": float(np.arccos(cosmin)), "UtU_minus_I_fro": orth}


def run_config3_b200(args, dev):
    """The precision form at the configuration-1 shape with an ill-conditioned spectrum: m = 1000,
    n = 2000, sigma_j = 10^(-6 (j-1)/199) for j <= 200 plus a 1e-8 G noise floor, k = 64, p = 16,
    N = 32; A stored in FP32 (the FP64 path reads its exact FP64 widening) and as BF16 parts of A
    and A' (resident, split once).  Gramian orthogonalizer, row-block Gramian KN (tol 1e-6), SVD
    former (the mixed solve: the precision former).  Timed solves of both paths (CUDA events),
    and for each the sigma relative error, the largest principal angle of U and ||U'U - I||
    against LAPACK dgesvd of the same FP64 matrix, plus mixed against FP64 on the same Omega."""
    import numpy as np
    import scipy.linalg
    import torch
    from mcnla_b200 import isvd, synthetic
    m, n, k, p, N = 1000, 2000, 64, 16, 32
    a32 = torch.as_tensor(synthetic.lowrank_np(m, n, synthetic.config3_sigma(), seed=3, noise=1e-8),
                          device=dev).float()
    a64 = a32.double()
    a_np = a64.cpu().numpy()
    u_ref, s_ref, _ = scipy.linalg.svd(a_np, full_matrices=False, lapack_driver="gesvd")
    split, fsplit = isvd.resident_parts(a32, 3)
    seed = 11
    _, _, omega = isvd.gaussian_bf16(n, (k + p) * N, seed, dev, with_fp64=True)
    kw = dict(integrator="rb_gramian_kn", former="svd", tol=1e-6, maxit=256)
    stream = torch.cuda.current_stream(dev)

    def timed(fn, steps):
        for _ in range(2):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3 / steps

    steps = max(3, args.steps)
    (s64, u64, _, it64), t64 = timed(lambda: isvd.solve(a64, k, p, N, omega=omega, **kw), steps)
    (smx, umx, _, itmx), tmx = timed(lambda: isvd.solve_mixed(a64, k, p, N, seed=seed, split=split,
                                                              former_split=fsplit, **kw), steps)
    s64, u64, smx, umx = (x.cpu().numpy() for x in (s64, u64, smx, umx))
    fp64 = dict(_svd_metrics(s64, u64, s_ref, u_ref), value=round(1.0 / t64, 3), unit="iSVD/s", iterations=it64)
    mixed = dict(_svd_metrics(smx, umx, s_ref, u_ref), value=round(1.0 / tmx, 3), unit="iSVD/s", iterations=itmx)
    mixed["vs_fp64_same_A_Omega"] = _svd_metrics(smx, umx, s64, u64)
    del split, fsplit, a32, a64, omega
    torch.cuda.empty_cache()
    return {"workload": "precision form, m=1000 n=2000, sigma_j=10^(-6(j-1)/199) j<=200 + 1e-8 G, k=64 p=16 N=32, "
                        "A in FP32 + resident BF16 parts (3 of A, 3 of A')",
            "stages": "Gramian / RowBlockGramianKolmogorovNagumo (tol 1e-6) / Svd (mixed: precision former)",
            "oracle": "LAPACK dgesvd (scipy.linalg.svd, lapack_driver='gesvd') of the FP64 widening of A",
            "fp64": fp64, "mixed": mixed, "speedup_mixed_vs_fp64": round(t64 / tmx, 3)}


def run_colblock_b200(args, dev, a_rm):
    """Configuration 2 in the column-block layout (the reference's isvd_dense_cb: column-major
    A, column-block Gramian former) with the Kolmogorov-Nagumo and Wen-Yin integrators: a
    column-major copy of the same A, one warm-up and `steps` timed solves each (CUDA events),
    sigma against the row-major solve with the same Omega seed."""
    import torch
    from mcnla_b200 import isvd
    a_cm = a_rm.t().contiguous().t()
    stream = torch.cuda.current_stream(dev)
    out = {}
    for integ in ("rb_gramian_kn", "rb_wy"):
        kw = dict(integrator=integ, former="cb_gramian", maxit=args.maxit, tol=args.tol)
        isvd.solve(a_cm, args.k, args.p, args.N, seed=0, **kw)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        steps = 2
        e0.record(stream)
        for step in range(steps):
            s, u, v, it = isvd.solve(a_cm, args.k, args.p, args.N, seed=100 + step, **kw)
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3 / steps
        entry = {"value": round(1.0 / t, 4), "unit": "iSVD/s", "iterations": it}
        if integ == args.integrator:
            s_rm = isvd.solve(a_rm, args.k, args.p, args.N, seed=100 + steps - 1, integrator=integ,
                              former=args.former, maxit=args.maxit, tol=args.tol)[0]
            entry["sigma_rel_diff_vs_row_major"] = float(((s - s_rm).abs() / s_rm).max().item())
        out[integ] = entry
    del a_cm
    torch.cuda.empty_cache()
    return {"layout": "column-major A (isvd_dense_cb), ColBlockGramianFormer", "integrators": out}


def run_row_block_b200(args, world, rank, local):
    """One matrix of the workload split by rows over the ranks (the reference's row-block
    decomposition): every rank sketches its rows with the same Omega and the stages sum their
    partial products through the library's NCCL communicator (NVLink / NVSwitch).  K timed
    solves, CUDA events on each rank, the max over ranks."""
    import torch
    from mcnla_b200 import isvd, rowblock
    dev = torch.device("cuda", local)
    full = workload_matrix(args, 0, device=dev)
    r0, r1 = rowblock.row_range(args.m, world, rank)
    a = full[r0:r1].contiguous() if not args.colmajor else full[r0:r1].t().contiguous().t()
    del full
    torch.cuda.empty_cache()
    ctx = isvd.context(dev)
    rowblock.attach_nccl(ctx, rank=rank, world=world)
    stream = torch.cuda.current_stream(dev)
    try:
        def solve(seed):
            return rowblock.solve_row_block(a, args.k, args.p, args.N, seed=seed, integrator=args.integrator,
                                            former=args.former, maxit=args.maxit, tol=args.tol)
        for w in range(max(1, args.warmup)):
            solve(w)
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for step in range(args.steps):
            s, u, v, it = solve(100 + step)
        e1.record(stream)
        torch.cuda.synchronize()
        t = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
        n_ar = rowblock.allreduces(ctx)
    finally:
        rowblock.detach(ctx)
    del a
    torch.cuda.empty_cache()
    return {"value": round(args.steps / t, 5), "unit": "iSVD/s (one matrix over all ranks)",
            "ms_per_step": round(t / args.steps * 1e3, 3), "rows_per_rank": [r1 - r0], "iterations": it,
            "collective": "the library's NCCL communicator: all-reduce of W, Bs and Z per solve",
            "allreduces_per_rank": int(n_ar), "scaling": "strong"}


def run_b200(args, world, rank, local):
    import numpy as np
    import torch
    from mcnla_b200 import isvd, synthetic, _lib

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    m, n, k, p, N = args.m, args.n, args.k, args.p, args.N
    l = k + p
    L = l * N
    sigma = np.exp(-np.arange(1, args.rank_r + 1) / 30.0)
    a = synthetic.lowrank_torch(m, n, sigma, seed=1000 + rank, noise=1e-4, device=dev, colmajor=args.colmajor)
    torch.cuda.synchronize()
    ctx = isvd.context(dev)
    stream = torch.cuda.current_stream(dev)

    def one_solve(seed):
        return isvd.solve(a, k, p, N, seed=seed, integrator=args.integrator, former=args.former, maxit=args.maxit,
                          tol=args.tol, with_v=True)

    # warm-up (also allocates the workspaces once)
    for w in range(max(args.warmup, 1)):
        s, u, v, it = one_solve(w)
    torch.cuda.synchronize()

    # ---- timed region: K whole solves, inputs resident in HBM
    clocks = ClockSampler(local)
    k0 = ctx.kernels_launched()
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    per_step = []
    iters = []
    ev0.record(stream)
    for step in range(args.steps):
        e_a, e_b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_a.record(stream)
        s, u, v, it = one_solve(100 + step)
        e_b.record(stream)
        per_step.append((e_a, e_b))
        iters.append(it)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    barrier(world)
    launches = ctx.kernels_launched() - k0
    total = ev0.elapsed_time(ev1) / 1e3
    step_ms = sorted(x.elapsed_time(y) for x, y in per_step)
    total = max_over_ranks(total, world)
    value = world * args.steps / total

    # ---- per-stage breakdown and the sketch roofline (stage API, CUDA events on the same stream)
    prm = isvd.Parameters(device=dev).setSize(m, n).setRank(k).setOverRank(p).setNumSketch(N).sync()
    sk = isvd.RowBlockGaussianProjectionSketcher(prm, 7) if not args.colmajor else \
        isvd.ColBlockGaussianProjectionSketcher(prm, 7)
    sk.initialize()
    q = prm.createCollectionQ()
    sketch_t = []
    for _ in range(3):
        sk(a, q)
        sketch_t.append(sk.times()[1])      # "projection" part: the sketch GEMM alone
    sketch_s = sum(sketch_t) / len(sketch_t)
    orth = isvd.RowBlockGramianOrthogonalizer(prm)
    orth.initialize()
    orth(q)
    integ_cls = {"kn": isvd.KolmogorovNagumoIntegrator, "rb_kn": isvd.RowBlockKolmogorovNagumoIntegrator,
                 "rb_gramian_kn": isvd.RowBlockGramianKolmogorovNagumoIntegrator,
                 "rb_wy": isvd.RowBlockWenYinIntegrator,
                 "rb_gramian_wy": isvd.RowBlockGramianWenYinIntegrator}[args.integrator]
    integ = integ_cls(prm, args.maxit, args.tol)
    integ.initialize()
    qbar = prm.createMatrixQbar()
    integ(q, qbar)
    former_cls = {"svd": isvd.SvdFormer, "gramian": isvd.GramianFormer, "rb_gramian": isvd.RowBlockGramianFormer,
                  "cb_gramian": isvd.ColBlockGramianFormer}[args.former]
    former = former_cls(prm)
    former.initialize()
    former(a, qbar)
    stages = {"sketch_s": sk.time(), "sketch_gemm_s": sketch_s, "orthogonalize_s": orth.time(),
              "integrate_s": integ.time(), "integrate_iterations": integ.iteration(), "form_s": former.time()}
    # every integrator on the same orthonormal sketches (tol and maxit of the workload)
    variants = {}
    if world == 1 and not args.quick:
        for name, cls in (("kn", isvd.KolmogorovNagumoIntegrator),
                          ("rb_kn", isvd.RowBlockKolmogorovNagumoIntegrator),
                          ("rb_gramian_kn", isvd.RowBlockGramianKolmogorovNagumoIntegrator),
                          ("rb_wy", isvd.RowBlockWenYinIntegrator),
                          ("rb_gramian_wy", isvd.RowBlockGramianWenYinIntegrator)):
            if "wy" in name and l > _lib.MAX_DIM_SKETCH_WENYIN:
                continue
            it_ = cls(prm, args.maxit, args.tol)
            it_.initialize()
            it_(q, qbar)
            variants[name] = {"s": round(it_.time(), 5), "iterations": it_.iteration(),
                              "s_per_iteration": round(it_.time() / max(1, it_.iteration()), 7)}
    peak64 = fp64_peak_tflops()
    flops = 2.0 * m * n * L
    achieved = flops / sketch_s / 1e12
    traffic = None
    if SKETCH_TRAFFIC_PER_ROW is not None:
        traffic = SKETCH_TRAFFIC_PER_ROW * m
    # ---- mixed precision: BF16 (hi + lo) tcgen05 sketch, FP64 elsewhere; A kept resident as BF16 parts
    mixed = None
    if not args.no_mixed:
        torch.cuda.synchronize()
        e_s0, e_s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_s0.record(stream)
        split = isvd.split_bf16(a, args.parts)
        fsplit = isvd.split_bf16(a.t(), args.former_parts) if args.former_parts else None
        e_s1.record(stream)
        torch.cuda.synchronize()
        split_s = e_s0.elapsed_time(e_s1) / 1e3

        def mixed_solve(seed):
            return isvd.solve_mixed(a, k, p, N, seed=seed, integrator=args.integrator, former=args.former,
                                    maxit=args.maxit, tol=args.tol, split=split, former_split=fsplit)
        for w in range(max(args.warmup, 1)):
            mixed_solve(w)
        torch.cuda.synchronize()
        barrier(world)
        m0e, m1e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0e.record(stream)
        for step in range(args.steps):
            sm_, um_, vm_, itm_ = mixed_solve(100 + step)
        m1e.record(stream)
        torch.cuda.synchronize()
        t_mixed = max_over_ranks(m0e.elapsed_time(m1e) / 1e3, world)
        # sketch kernel alone (tcgen05 BF16 x 2 parts) for its roofline
        om_t, ldo, om64 = isvd.gaussian_bf16(n, L, 77, dev, with_fp64=True)
        prm_c = _lib.Params(m, n, k, p, N)
        qb = torch.empty(m, L, dtype=torch.float64, device=dev)
        sk_t = []
        for _ in range(3):
            _lib.check(ctx.lib.mcnla_b200_sketch_bf16(ctx.bind(), ctypes.byref(prm_c), isvd._ptr(split.hi),
                                                      isvd._ptr(split.lo), isvd._ptr(split.lo2), split.ld,
                                                      isvd._ptr(om_t), ldo, isvd._ptr(qb)), "sketch_bf16")
            sk_t.append(ctx.last_times()[1])
        sk_bf16 = sum(sk_t) / len(sk_t)
        # accuracy of the mixed solve against the FP64 solve on the same A and Omega
        s64, u64, v64, it64 = isvd.solve(a, k, p, N, omega=om64, integrator=args.integrator, former=args.former,
                                         maxit=args.maxit, tol=args.tol)
        smx, umx, vmx, itmx = isvd.solve_mixed(a, k, p, N, seed=77, integrator=args.integrator,
                                               former=args.former, maxit=args.maxit, tol=args.tol, split=split,
                                               former_split=fsplit)
        rel = ((smx - s64).abs() / s64).max().item()
        ang = float(torch.arccos(torch.clamp(torch.linalg.svdvals(u64.t() @ umx).min(), -1, 1)).item())
        orth = float(torch.linalg.norm(umx.t() @ umx - torch.eye(k, dtype=torch.float64, device=dev)).item())
        bf16_peak = _measured_peak("bf16_tflops")
        ach = args.parts * 2.0 * m * n * L / sk_bf16 / 1e12
        mixed = {"value": round(world * args.steps / t_mixed, 5), "unit": "iSVD/s",
                 "ms_per_step": round(t_mixed / args.steps * 1e3, 3),
                 "speedup_vs_fp64": round((world * args.steps / t_mixed) / value, 3),
                 "sketch": "A as %d BF16 parts (%d bits), Omega BF16, tcgen05 FP32 accumulation, FP64 out"
                           % (args.parts, 8 * args.parts),
                 "former": ("Q' A on tcgen05 from A' as %d BF16 parts and Qbar as 3, split over K, FP64 sums "
                            "of FP32 chunks" % args.former_parts) if fsplit is not None else "FP64 from A",
                 "gramian": "Qs' Qs from 3 BF16 parts of Qs, then one FP64 re-orthonormalization of Qbar"
                            if "gramian" in args.integrator else None,
                 "split_s": round(split_s, 5), "sketch_gemm_s": round(sk_bf16, 5),
                 "sketch_roofline": {"bound": "tensor", "achieved": round(ach, 2),
                                     "peak": bf16_peak, "unit": "TFLOP/s",
                                     "frac": round(ach / bf16_peak, 4) if bf16_peak else None,
                                     "peak_source": "MEASURED_PEAKS.json bf16_tflops (burst) of measured",
                                     "counted": "%d parts x 2 m n N l tensor-pipe flops" % args.parts,
                                     "achieved_algorithmic": round(ach / args.parts, 2),
                                     "frac_algorithmic": round(ach / args.parts / bf16_peak, 4) if bf16_peak else None,
                                     "algorithmic": "2 m n N l flops (one product; the parts are an accuracy "
                                                    "choice)"},
                 "accuracy_vs_fp64_same_A_Omega": {"sigma_rel_err": rel, "max_principal_angle_U": ang,
                                                   "UtU_minus_I_fro": orth, "iterations": [itmx, it64]}}
        del split, fsplit, qb, om_t, om64

    stage_roof = stage_rooflines(m, n, k, l, N, args.integrator, args.former, stages, peak64,
                                 _measured_peak("hbm_gbs"))
    roofline = {"bound": "tensor", "kernel": "dgemm_kernel (sketch Y = A Omega, FP64 DMMA)",
                "achieved": round(achieved, 3), "peak": round(peak64, 3), "unit": "TFLOP/s",
                "frac": round(achieved / peak64, 4), "traffic": traffic,
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (FP64 has no tcgen05 kind; the "
                               "measured-peaks file holds bf16 and HBM only)",
                "algorithmic": "2*m*n*N*l flops per launch"}

    # ---- end to end through the host-buffer C-ABI call (copies inside the timed region)
    e2e = None
    if not args.no_e2e:
        a_host = torch.empty(m, n, dtype=torch.float64, pin_memory=True) if not args.colmajor else \
            torch.empty(n, m, dtype=torch.float64, pin_memory=True)
        a_host.copy_(a.t() if args.colmajor else a)
        om_host = torch.empty(n, L, dtype=torch.float64, pin_memory=True)
        om_host.copy_(synthetic.omega_torch(n, L, seed=3, device=dev))
        out = (torch.empty(k, dtype=torch.float64, pin_memory=True),
               torch.empty(m, k, dtype=torch.float64, pin_memory=True),
               torch.empty(n, k, dtype=torch.float64, pin_memory=True))
        isvd.solve_host(a_host, om_host, k, p, N, integrator=args.integrator, former=args.former,
                        maxit=args.maxit, tol=args.tol, out=out, colmajor=args.colmajor)
        torch.cuda.synchronize()
        barrier(world)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            isvd.solve_host(a_host, om_host, k, p, N, integrator=args.integrator, former=args.former,
                            maxit=args.maxit, tol=args.tol, out=out, colmajor=args.colmajor)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(world)
        t_e2e = max_over_ranks(e0.elapsed_time(e1) / 1e3, world)
        e2e = {"value": round(world * args.steps / t_e2e, 5), "unit": "iSVD/s",
               "h2d_bytes_per_step": int(a_host.numel() * 8 + om_host.numel() * 8),
               "d2h_bytes_per_step": int((k + m * k + n * k) * 8),
               "path": "mcnla_b200_isvd_host (pinned host A and Omega in, S/U/V out)"}
        del a_host, om_host

    recon = reconstruction_error_torch(a, s, u, v)
    c1 = run_config1_b200(args, dev) if world == 1 and not args.quick else None
    c3 = colblock = None
    if world == 1 and not args.quick:
        for name, fn in (("config3", lambda: run_config3_b200(args, dev) if not args.no_mixed else None),
                         ("colblock", lambda: run_colblock_b200(args, dev, a) if not args.colmajor else None)):
            try:
                r_ = fn()
            except Exception as e:          # an extra leg's failure is reported, not fatal
                r_ = {"error": "%s: %s" % (type(e).__name__, e)}
                torch.cuda.synchronize()
            c3, colblock = (r_, colblock) if name == "config3" else (c3, r_)
    row_block = None
    if world > 1 and not args.no_row_block:
        del a
        torch.cuda.empty_cache()
        try:
            row_block = run_row_block_b200(args, world, rank, local)
        except Exception as e:              # reported on the line; the replicas' value stands
            row_block = {"error": "%s: %s" % (type(e).__name__, e)}
    result = {
        "metric": METRIC, "value": round(value, 5), "unit": "iSVD/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total / args.steps * 1e3, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, on device)",
        "config": dict(workload(args), parallelism="replicas" if world > 1 else "single GPU"),
        "a_read_gbs": round(2 * m * n * 8 * world * args.steps / total / 1e9, 2),
        "p50_ms": round(step_ms[len(step_ms) // 2], 3),
        "p99_ms": round(step_ms[min(len(step_ms) - 1, int(0.99 * len(step_ms)))], 3),
        "iterations": iters[-1], "stages": stages, "integrators": variants, "mixed": mixed, "roofline": roofline,
        "stage_roofline": stage_roof, "e2e": e2e,
        "gpu_launches": int(launches), "clocks": clk,
        "reconstruction_rel_err": recon, "config1": c1, "config3": c3, "colblock": colblock, "row_block": row_block,
    }
    return result


# ------------------------------------------------------------------------------------------------
# batched and served solves: uneven FP32 matrices through mcnla_b200_server_*
# ------------------------------------------------------------------------------------------------
def _pct(xs, q):
    xs = sorted(xs)
    return xs[min(len(xs) - 1, int(q * len(xs)))] if xs else None


def run_serving(args, dev):
    """Uneven batch (1024 FP32 matrices, m ~ U[512,16384], n ~ U[256,4096], k in {8,16,32,64},
    p = k/2, N = 8, sigma_j = j^-alpha, KN tol 1e-5, SVD former) through the server:
    per-request plain FP64 (one worker), batched FP64 and batched mixed precision (W
    workers), then Poisson arrivals at each rate with 5 % large requests (65536 x 8192,
    k = 128, p = 32, N = 16), mixed precision, 150 GB admission cap, and the same arrivals
    again in plain FP64 at the --serve-rates-fp64 rates.  A stays resident in HBM as FP32
    (and, for the mixed requests, as BF16 parts); wall-clock times on the host with the
    device synchronized on both sides (the solves run on the workers' own streams)."""
    import numpy as np
    import torch
    from mcnla_b200 import isvd, synthetic

    W = args.serve_workers
    budget = int(150e9)   # the configuration's 150 GB admission cap
    shapes = synthetic.batch_shapes(args.batch_count, seed=4)
    pool = [synthetic.lowrank_torch(sh["m"], sh["n"], sh["sigma"], seed=sh["seed"], device=dev, dtype=torch.float32)
            for sh in shapes]
    torch.cuda.synchronize()

    def request(i, mixed, a=None, sh=None, parts=None):
        sh = shapes[i] if sh is None else sh
        sp, fsp = parts if parts is not None else (None, None)
        return isvd.Request(pool[i] if a is None else a, sh["k"], sh["p"], sh["N"], seed=sh["seed"],
                            integrator=args.serve_integrator, former=args.serve_former, maxit=256, tol=1e-5,
                            mixed=mixed, split=sp, former_split=fsp)

    order = sorted(range(len(shapes)), key=lambda i: -shapes[i]["m"] * shapes[i]["n"] * shapes[i]["k"])

    def timed_batch(workers, mixed, grouped, runs=2):
        """grouped: the whole batch through mcnla_b200_isvd_grouped (grouped integrator kernel);
        else one worker pool of the server (per-request solves).  The batch runs `runs` times
        (host-side noise from the box moves a single pass by up to 1.5x); the fastest counts,
        and every pass's seconds are reported."""
        phases = None
        passes = []
        if grouped:
            isvd.solve_grouped([request(i, mixed) for i in order[:64]], workers=workers, budget_bytes=budget)
            torch.cuda.synchronize()
            for _ in range(runs):
                reqs = [request(i, mixed) for i in range(len(shapes))]
                t0 = time.perf_counter()
                isvd.solve_grouped(reqs, workers=workers, budget_bytes=budget)
                torch.cuda.synchronize()
                passes.append(time.perf_counter() - t0)
                if passes[-1] == min(passes):
                    phases = isvd.grouped_times()
            st = {"peak_bytes": 0}
        else:
            with isvd.Server(workers=workers, budget_bytes=budget, device=dev) as srv:
                warm = [request(i, mixed) for i in order[:2 * workers]]        # grow every worker's buffers
                for r in warm:
                    srv.submit(r)
                for r in warm:
                    srv.wait(r)
                torch.cuda.synchronize()
                for _ in range(runs):
                    reqs = [request(i, mixed) for i in range(len(shapes))]
                    t0 = time.perf_counter()
                    for r in reqs:
                        srv.submit(r)
                    for r in reqs:
                        srv.wait(r)
                    torch.cuda.synchronize()
                    passes.append(time.perf_counter() - t0)
                st = srv.stats()
        t = min(passes)
        bad = sum(1 for r in reqs if r.result.status != 0)
        its = [r.result.iteration for r in reqs]
        svc = [r.result.seconds for r in reqs]
        a_bytes = sum(shapes[i]["m"] * shapes[i]["n"] * 4 for i in range(len(shapes)))
        return reqs, {"workers": workers, "solves_per_s": round(len(reqs) / t, 2), "seconds": round(t, 4),
                      "passes_s": [round(x, 4) for x in passes],
                      "a_read_gbs": round(2 * a_bytes / t / 1e9, 2), "failed": bad,
                      "iterations_mean": round(float(np.mean(its)), 2), "iterations_max": int(max(its)),
                      "service_p50_ms": round(_pct(svc, 0.5) * 1e3, 3),
                      "service_p99_ms": round(_pct(svc, 0.99) * 1e3, 3),
                      "peak_admitted_gb": round(st["peak_bytes"] / 1e9, 3),
                      "path": "grouped batch (mcnla_b200_isvd_grouped)" if grouped else "worker pool (server)",
                      "phases_s": phases}

    _, serial64 = timed_batch(1, False, False, runs=1)
    _, batched64 = timed_batch(W, False, False)
    mixed_reqs, batched_mx = timed_batch(W, args.serve_parts, False)
    _, grouped64 = timed_batch(W, False, True)
    _, grouped_mx = timed_batch(W, args.serve_parts, True)

    # accuracy of the mixed results against FP64 solves on the same A and Omega (BF16 Omega
    # drawn from the same seed, FP64 copy), and against FP64 dgesvd singular values of A
    acc = {"sigma_rel_err": 0.0, "max_principal_angle_U": 0.0, "UtU_minus_I_fro": 0.0, "sampled": 0,
           "sigma_rel_err_vs_dgesvd": 0.0, "sampled_dgesvd": 0}
    for i in range(min(16, len(shapes))):
        sh, r = shapes[i], mixed_reqs[i]
        k, L = sh["k"], (sh["k"] + sh["p"]) * sh["N"]
        a64 = pool[i].double()
        _, _, om64 = isvd.gaussian_bf16(sh["n"], L, sh["seed"], dev, with_fp64=True)
        s64, u64, _, _ = isvd.solve(a64, k, sh["p"], sh["N"], omega=om64, integrator=args.serve_integrator,
                                    former=args.serve_former, maxit=256, tol=1e-5)
        acc["sigma_rel_err"] = max(acc["sigma_rel_err"], ((r.s - s64).abs() / s64).max().item())
        cosmin = torch.linalg.svdvals(u64.t() @ r.u).min().clamp(-1, 1)
        acc["max_principal_angle_U"] = max(acc["max_principal_angle_U"], float(torch.arccos(cosmin).item()))
        eye = torch.eye(k, dtype=torch.float64, device=dev)
        acc["UtU_minus_I_fro"] = max(acc["UtU_minus_I_fro"], float(torch.linalg.norm(r.u.t() @ r.u - eye).item()))
        acc["sampled"] += 1
        if sh["m"] * sh["n"] <= (1 << 23) and acc["sampled_dgesvd"] < 4:
            sv = torch.linalg.svdvals(a64, driver="gesvd")[:k]
            acc["sigma_rel_err_vs_dgesvd"] = max(acc["sigma_rel_err_vs_dgesvd"], ((r.s - sv).abs() / sv).max().item())
            acc["sampled_dgesvd"] += 1
        del a64, om64
    del mixed_reqs

    # ---- served: Poisson arrivals, mixed precision, 5 % large requests
    keep = max(1, min(args.serve_pool, len(pool)))
    del pool[keep:]
    torch.cuda.empty_cache()
    lsh = [synthetic.large_shape(seed=s) for s in (1, 2)]
    large = [synthetic.lowrank_torch(x["m"], x["n"], x["sigma"], seed=x["seed"], device=dev, dtype=torch.float32)
             for x in lsh]
    torch.cuda.synchronize()
    # per-request plain FP64 service time of the large request, for the mix's FP64 reference rate
    # (one warm single-worker server: the second solve is the steady-state service time)
    t_large = []
    with isvd.Server(workers=1, budget_bytes=budget, device=dev) as srv:
        for _ in range(2):
            r = request(0, False, a=large[0], sh=lsh[0])
            srv.submit(r)
            srv.wait(r)
            t_large.append(r.result.seconds)
    t_small = serial64["seconds"] / len(shapes)
    fp64_mix_rate = 1.0 / (0.95 * t_small + 0.05 * t_large[-1])
    served = []
    rates = [float(x) for x in args.serve_rates.split(",") if x]
    # resident matrices keep their BF16 parts (A for the sketch, A' for the precision former), split once
    t_split = time.perf_counter()
    resident = [isvd.resident_parts(pool[i], args.serve_parts) for i in range(keep)]
    large_parts = [isvd.resident_parts(x, args.serve_parts) for x in large]
    torch.cuda.synchronize()
    t_split = time.perf_counter() - t_split
    n_resident = keep + len(large)
    with isvd.Server(workers=W, budget_bytes=budget, device=dev) as srv:
        warm = [request(0, args.serve_parts, a=large[j], sh=lsh[j], parts=large_parts[j]) for j in range(2)] + \
               [request(i, args.serve_parts, parts=resident[i]) for i in range(min(keep, 2 * W))]
        for r in warm:
            srv.submit(r)
        for r in warm:
            srv.wait(r)
        def serve(rate, mixed):
            """Poisson arrivals at `rate` (seeded by the rate: the same arrivals, sizes and
            matrices for every precision), submitted as they arrive; latency per request."""
            rng = np.random.default_rng(int(rate))
            count = max(400, int(rate * args.serve_seconds)) if not args.quick else 64
            arrivals = np.cumsum(rng.exponential(1.0 / rate, count))
            is_large = rng.random(count) < 0.05
            pick = rng.integers(0, keep, count)
            reqs = [request(0, mixed, a=large[j % 2], sh=lsh[j % 2], parts=large_parts[j % 2] if mixed else None)
                    if is_large[j] else
                    request(int(pick[j]), mixed, parts=resident[int(pick[j])] if mixed else None)
                    for j in range(count)]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            for r, ta in zip(reqs, arrivals):
                while time.perf_counter() - t0 < ta:
                    pass
                srv.submit(r)
            for r in reqs:
                srv.wait(r)
            torch.cuda.synchronize()
            t = time.perf_counter() - t0
            lat = [r.result.latency for r in reqs]
            lat_small = [r.result.latency for r, big in zip(reqs, is_large) if not big]
            return {"rate_per_s": rate, "requests": count, "large": int(is_large.sum()),
                    "solves_per_s": round(count / t, 2), "seconds": round(t, 4),
                    "p50_ms": round(_pct(lat, 0.5) * 1e3, 3), "p99_ms": round(_pct(lat, 0.99) * 1e3, 3),
                    "p50_ms_small": round(_pct(lat_small, 0.5) * 1e3, 3),
                    "p99_ms_small": round(_pct(lat_small, 0.99) * 1e3, 3),
                    "failed": sum(1 for r in reqs if r.result.status != 0)}

        for rate in rates:
            served.append(serve(rate, args.serve_parts))
        st = srv.stats()
    # the same arrivals in plain FP64 (the server widens each FP32 A per request), on a server
    # whose admission cap leaves room for the resident FP32 matrices once the BF16 parts are freed
    del resident, large_parts
    torch.cuda.empty_cache()
    budget64 = int(min(budget, torch.cuda.mem_get_info(dev)[0] - 12e9))
    with isvd.Server(workers=W, budget_bytes=budget64, device=dev) as srv:
        served64 = [serve(rate, False) for rate in [float(x) for x in args.serve_rates_fp64.split(",") if x]]
    del large, pool
    torch.cuda.empty_cache()
    return {
        "workload": "%d uneven FP32 matrices (m~U[512,16384], n~U[256,4096], k in {8,16,32,64}, p=k/2, N=8, "
                    "sigma_j=j^-alpha over j=1..min(m,n), alpha~U[0.5,2]), %s tol 1e-5, %s former"
                    % (len(shapes), args.serve_integrator, args.serve_former),
        "timing": "host wall clock, device synchronized on both sides; solves on the workers' own streams",
        "per_request_fp64": serial64, "batched_fp64": batched64, "batched_mixed": batched_mx,
        "grouped_fp64": grouped64, "grouped_mixed": grouped_mx,
        "grouped_mixed_speedup_vs_grouped_fp64": round(grouped_mx["solves_per_s"] / grouped64["solves_per_s"], 3),
        "mixed_speedup_vs_per_request_fp64": round(batched_mx["solves_per_s"] / serial64["solves_per_s"], 3),
        "mixed_speedup_vs_batched_fp64": round(batched_mx["solves_per_s"] / batched64["solves_per_s"], 3),
        "accuracy_mixed_vs_fp64_same_A_Omega": acc,
        "served": {"precision": "mixed, A as %d BF16 parts and A' as 3, resident (split once: %.2f s for the %d "
                                "matrices)" % (args.serve_parts, t_split, n_resident),
                   "workers": W, "admission_cap_gb": budget / 1e9,
                   "large": "5%% of requests: 65536 x 8192 FP32, k=128 p=32 N=16 (%s)" % "two resident matrices",
                   "resident_pool": keep, "fp64_per_request_solves_per_s_same_mix": round(fp64_mix_rate, 2),
                   "fp64_large_request_s": round(t_large[-1], 4), "rates": served,
                   "fp64_same_arrivals": served64, "fp64_admission_cap_gb": round(budget64 / 1e9, 1),
                   "mixed_speedup_vs_fp64_same_arrivals": [
                       {"rate_per_s": x["rate_per_s"], "solves_per_s": round(x["solves_per_s"] / y["solves_per_s"], 3),
                        "p50": round(y["p50_ms"] / x["p50_ms"], 3)}
                       for x in served for y in served64 if x["rate_per_s"] == y["rate_per_s"]],
                   "peak_admitted_gb": round(st["peak_bytes"] / 1e9, 3)},
    }


# ------------------------------------------------------------------------------------------------
# single-kernel cases (profiling)
# ------------------------------------------------------------------------------------------------
def run_trace(args, dev):
    """Device time per kernel (CUPTI activity records through torch.profiler: every launch's own
    start and end on the GPU, no replay, the autotuner sees ordinary launches) for one FP64 and one
    mixed solve of the workload after two warm-up solves each, and each kernel's time per
    integrator iteration from the difference of solves capped at 257 and 65 iterations."""
    import collections
    import numpy as np
    import torch
    from torch.profiler import profile, ProfilerActivity
    from mcnla_b200 import isvd, synthetic
    m, n, k, p, N = args.m, args.n, args.k, args.p, args.N
    a = synthetic.lowrank_torch(m, n, np.exp(-np.arange(1, args.rank_r + 1) / 30.0), seed=1, noise=1e-4, device=dev)
    sp = isvd.split_bf16(a, args.parts)
    fs = isvd.split_bf16(a.t(), args.former_parts) if args.former_parts else None

    def solve(mixed, maxit):
        kw = dict(seed=3, integrator=args.integrator, former=args.former, tol=args.tol, maxit=maxit)
        if mixed:
            return isvd.solve_mixed(a, k, p, N, split=sp, former_split=fs, **kw)
        return isvd.solve(a, k, p, N, **kw)

    def kernels(mixed, maxit):
        solve(mixed, maxit)
        solve(mixed, maxit)
        torch.cuda.synchronize()
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            solve(mixed, maxit)
            torch.cuda.synchronize()
        agg = collections.defaultdict(lambda: [0, 0.0])
        for e in prof.events():
            if e.device_type.name == "CUDA" and e.time_range.end > e.time_range.start:
                key = e.name.replace("(anonymous namespace)::", "").split("(")[0]
                agg[key][0] += 1
                agg[key][1] += (e.time_range.end - e.time_range.start) / 1e3   # ms
        return agg

    out = {"workload": workload(args)["workload"], "timing": "CUPTI activity records (device start/end per "
           "launch), one solve after two warm-up solves"}
    for name, mixed in (("fp64", False), ("mixed", True)):
        full, short = kernels(mixed, args.maxit), kernels(mixed, 65)
        rows = []
        for key in sorted(full, key=lambda x: -full[x][1]):
            c1, t1 = full[key]
            c0, t0 = short.get(key, [0, 0.0])
            rows.append({"kernel": key[-110:], "launches": c1, "ms": round(t1, 3),
                         "us_per_iteration": round((t1 - t0) * 1e3 / max(1, args.maxit - 65), 2)})
        out[name] = {"kernel_ms_total": round(sum(r["ms"] for r in rows), 3), "kernels": rows[:20]}
    return out


def run_served_trace(args, dev, count=500):
    """The served mix in throughput mode: `count` requests (5 % large: 65536 x 8192, k = 128,
    p = 32, N = 16; the rest from 256 resident matrices of the uneven batch) submitted at once to
    a --serve-workers server, mixed (3 BF16 parts, resident) and FP64; wall time, mean service
    time per request kind, and per-kernel device time of a second pass (CUPTI activity records
    through torch.profiler: every launch's own start and end, no replay)."""
    import collections
    import numpy as np
    import torch
    from torch.profiler import profile, ProfilerActivity
    from mcnla_b200 import isvd, synthetic
    W = args.serve_workers
    shapes = synthetic.batch_shapes(256, seed=4)
    pool = [synthetic.lowrank_torch(sh["m"], sh["n"], sh["sigma"], seed=sh["seed"], device=dev, dtype=torch.float32)
            for sh in shapes]
    lsh = [synthetic.large_shape(seed=s_) for s_ in (1, 2)]
    large = [synthetic.lowrank_torch(x["m"], x["n"], x["sigma"], seed=x["seed"], device=dev, dtype=torch.float32)
             for x in lsh]
    parts = [isvd.resident_parts(a_, 3) for a_ in pool]
    lparts = [isvd.resident_parts(a_, 3) for a_ in large]
    torch.cuda.synchronize()
    rng = np.random.default_rng(1000)
    is_large = rng.random(count) < 0.05
    pick = rng.integers(0, len(pool), count)

    def request(j, mixed):
        big = bool(is_large[j])
        i = j % 2 if big else int(pick[j])
        sh = lsh[i] if big else shapes[i]
        sp, fsp = ((lparts[i] if big else parts[i]) if mixed else (None, None))
        return isvd.Request(large[i] if big else pool[i], sh["k"], sh["p"], sh["N"], seed=sh["seed"],
                            integrator="rb_gramian_kn", former="rb_gramian", maxit=256, tol=1e-5, mixed=mixed,
                            split=sp, former_split=fsp)

    out = {}
    for name, mixed in (("mixed", 3), ("fp64", False)):
        cap = int(min(90e9, torch.cuda.mem_get_info(dev)[0] - 12e9))   # room left by the resident matrices
        with isvd.Server(workers=W, budget_bytes=cap, device=dev) as srv:
            warm = [request(j, mixed) for j in range(32)]
            for r in warm:
                srv.submit(r)
            for r in warm:
                srv.wait(r)
            torch.cuda.synchronize()
            reqs = [request(j, mixed) for j in range(count)]
            t0 = time.perf_counter()
            for r in reqs:
                srv.submit(r)
            for r in reqs:
                srv.wait(r)
            torch.cuda.synchronize()
            wall = time.perf_counter() - t0
            kinds = collections.defaultdict(list)
            for j, r in enumerate(reqs):
                kinds["large" if is_large[j] else "k%d" % shapes[int(pick[j])]["k"]].append(r.result.seconds)
            reqs = [request(j, mixed) for j in range(count)]
            with profile(activities=[ProfilerActivity.CUDA]) as prof:
                for r in reqs:
                    srv.submit(r)
                for r in reqs:
                    srv.wait(r)
                torch.cuda.synchronize()
        agg = collections.defaultdict(lambda: [0, 0.0])
        for e in prof.events():
            if e.device_type.name == "CUDA" and e.time_range.end > e.time_range.start:
                key = e.name.replace("(anonymous namespace)::", "").split("(")[0][:90]
                agg[key][0] += 1
                agg[key][1] += (e.time_range.end - e.time_range.start) / 1e3
        top = sorted(agg.items(), key=lambda kv: -kv[1][1])[:16]
        out[name] = {"wall_s": round(wall, 3), "solves_per_s": round(count / wall, 1),
                     "kernel_ms_total": round(sum(v[1] for v in agg.values()), 1),
                     "service_mean_ms": {k_: round(1e3 * float(np.mean(v)), 2) for k_, v in sorted(kinds.items())},
                     "kernels": [{"name": k_, "launches": v[0], "ms": round(v[1], 1)} for k_, v in top]}
    del pool, large, parts, lparts
    torch.cuda.empty_cache()
    return {"case": "served mix, throughput mode, %d requests, %d workers" % (count, W), **out}


def run_gkn_scaling(args, dev):
    """The persistent row-block Gramian KN integrator's time per iteration against its CTA share
    (mcnla_b200_set_cta_limit) for l = 96, 48, 24 (N = 8, m = 8448, n = 2176, sigma_j = 1/j,
    tol 1e-5): stage part timer, best of three calls."""
    import numpy as np
    import torch
    from mcnla_b200 import isvd, synthetic
    ctx = isvd.context(dev)
    rows = []
    for k, p in ((64, 32), (32, 16), (16, 8)):
        m, n, N = 8448, 2176, 8
        l, L = k + p, (k + p) * N
        a = synthetic.lowrank_torch(m, n, np.arange(1, min(m, n) + 1) ** -1.0, seed=1, device=dev)
        prm = isvd.Parameters(device=dev).setSize(m, n).setRank(k).setOverRank(p).setNumSketch(N).sync()
        sk = isvd.RowBlockGaussianProjectionSketcher(prm, 7)
        sk.initialize()
        q = prm.createCollectionQ()
        sk(a, q)
        orth = isvd.RowBlockGramianOrthogonalizer(prm)
        orth.initialize()
        orth(q)
        try:
            for ctas in (18, 37, 74, 0):
                ctx.set_cta_limit(ctas)
                integ = isvd.RowBlockGramianKolmogorovNagumoIntegrator(prm, 256, 1e-5)
                integ.initialize()
                qbar = prm.createMatrixQbar()
                integ(q, qbar)
                t = 1e9
                for _ in range(3):
                    integ(q, qbar)
                    t = min(t, integ.times()[1])
                it = integ.iteration()
                flops = 2.0 * L * L * l + 6.0 * L * l * l
                rows.append({"l": l, "L": L, "ctas": ctas or torch.cuda.get_device_properties(dev).multi_processor_count, "iterations": it,
                             "us_per_iteration": round(t / it * 1e6, 2), "tflops": round(flops * it / t / 1e12, 3)})
        finally:
            ctx.set_cta_limit(0)
        del a, q
    return {"kernel": "k_gkn_persistent", "rows": rows}


def run_ingest(args, dev):
    """Streamed ingest (mcnla_b200_isvd_stream) of an MCNLA binary file of the --m x --n workload
    matrix, against reading the file alone and the host-buffer solve of the same A already in
    pinned memory: wall seconds of each (best of 2; the file is read once before, so it comes
    from the page cache)."""
    import tempfile
    import numpy as np
    import torch
    from mcnla_b200 import io, isvd, synthetic
    m, n, k, p, N = args.m, args.n, args.k, args.p, args.N
    L = (k + p) * N
    a = workload_matrix(args, 0, device=dev).cpu().numpy()
    omega = synthetic.omega_torch(n, L, seed=5, device=dev).cpu().pin_memory()
    kw = dict(integrator=args.integrator, former=args.former, maxit=args.maxit, tol=args.tol)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "a.bin")
        io.save_binary(path, a)
        _, _, read_rows = io.binary_row_reader(path)
        buf = torch.empty(min(m, 8192), n, dtype=torch.float64, pin_memory=True)

        def read_all():
            for r0 in range(0, m, buf.shape[0]):
                read_rows(r0, min(buf.shape[0], m - r0), buf.data_ptr())

        def best(fn):
            t = 1e9
            for _ in range(2):
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                fn()
                torch.cuda.synchronize()
                t = min(t, time.perf_counter() - t0)
            return t
        read_all()
        t_read = best(read_all)
        t_stream = best(lambda: isvd.solve_stream(read_rows, m, n, omega, k, p, N, device=dev, **kw))
        a_h = torch.from_numpy(a).pin_memory()
        del a
        t_host = best(lambda: isvd.solve_host(a_h, omega, k, p, N, device=dev, **kw))
    gb = m * n * 8 / 1e9
    return {"case": "streamed ingest of a %d x %d FP64 binary file (%.2f GB), k=%d p=%d N=%d, %s / %s"
                    % (m, n, gb, k, p, N, args.integrator, args.former),
            "read_file_s": round(t_read, 4), "stream_solve_s": round(t_stream, 4),
            "host_buffer_solve_s": round(t_host, 4),
            "overlapped_s": round(max(0.0, t_read + t_host - t_stream), 4),
            "file_gbs": round(gb / t_read, 2)}


def run_inverse(args, dev):
    """The one-CTA Gauss-Jordan inverse (mcnla_b200_inverse_batched, the kernel of the Wen-Yin step's
    2l x 2l solve) on one matrix per launch, n = 16 .. 160: C = M - I / tau with M = [D/2, I/2;
    -Dg/2, -D/2] from seeded Gram-like D, Dg, as the Wen-Yin trial builds it.  CUDA events around
    one call from Python, best of 5, so each time includes the host side of the call (tens of us,
    most of the time at small n); the residual max |C X - I|."""
    import numpy as np
    import torch
    from mcnla_b200 import isvd, _lib
    ctx = isvd.context(dev)
    rows = []
    for n in (16, 32, 64, 96, 128, 160):
        l = n // 2
        rng = np.random.default_rng(n)
        y = rng.standard_normal((4 * l, l)) / np.sqrt(4 * l)
        d = y.T @ y
        dg = d @ d
        eye = np.eye(l)
        c = np.block([[d / 2 - eye / 0.5, eye / 2], [-dg / 2, -d / 2 - eye / 0.5]])
        src = torch.as_tensor(c, device=dev)
        work = src.clone()

        def call():
            work.copy_(src)
            _lib.check(ctx.lib.mcnla_b200_inverse_batched(ctx.bind(), n, 1, isvd._ptr(work)), "inverse_batched")
        call()
        stream = torch.cuda.current_stream(dev)
        best = 1e9
        for _ in range(5):
            work.copy_(src)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            _lib.check(ctx.lib.mcnla_b200_inverse_batched(ctx.bind(), n, 1, isvd._ptr(work)), "inverse_batched")
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        x = work.cpu().numpy()
        rows.append({"n": n, "ms": round(best, 4), "residual": float(np.abs(c @ x - np.eye(n)).max())})
    return {"kernel": "k_inverse (one-CTA Gauss-Jordan, the Wen-Yin step's solve)", "rows": rows}


def run_syev(args, dev):
    """The batched Jacobi eigensolver (mcnla_b200_syev_batched, descending |lambda|, as the
    orthogonalizer and the formers call it) on sketch Gram matrices Y'Y, Y = A Omega with
    sigma_j = 1/j: l = 12 .. 160, 8 matrices (16 for l >= 128).  CUDA events, best of 3; the
    residual max |W v - lambda v| / lambda_1 and max |V'V - I|."""
    import numpy as np
    import torch
    from mcnla_b200 import isvd, _lib
    ctx = isvd.context(dev)
    rows = []
    for l in (12, 24, 48, 64, 96, 128, 160):
        batch = 16 if l >= 128 else 8
        rng = np.random.default_rng(l)
        m, n = 4 * l + 64, 6 * l + 64
        u, _ = np.linalg.qr(rng.standard_normal((m, min(m, n))))
        v, _ = np.linalg.qr(rng.standard_normal((n, min(m, n))))
        a = (u / np.arange(1, min(m, n) + 1)) @ v.T
        grams = []
        for _ in range(batch):
            y = a @ rng.standard_normal((n, l))
            grams.append(y.T @ y)
        g = torch.as_tensor(np.stack(grams), device=dev)
        w = torch.empty(batch, l, dtype=torch.float64, device=dev)
        vv = torch.empty(batch, l, l, dtype=torch.float64, device=dev)

        def call():
            _lib.check(ctx.lib.mcnla_b200_syev_batched(ctx.bind(), l, batch, isvd._ptr(g), isvd._ptr(w), isvd._ptr(vv),
                                                       1), "syev_batched")
        call()
        stream = torch.cuda.current_stream(dev)
        best = 1e9
        for _ in range(3):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(stream)
            call()
            e1.record(stream)
            torch.cuda.synchronize()
            best = min(best, e0.elapsed_time(e1))
        gn, wn, vn = g.cpu().numpy(), w.cpu().numpy(), vv.cpu().numpy()
        resid = max(float(np.abs(gn[b] @ vn[b] - vn[b] * wn[b]).max() / wn[b].max()) for b in range(batch))
        orth = max(float(np.abs(vn[b].T @ vn[b] - np.eye(l)).max()) for b in range(batch))
        rows.append({"l": l, "batch": batch, "ms": round(best, 3), "residual": resid, "orthogonality": orth})
    return {"kernel": "k_syev (batched Jacobi, 1024 threads per matrix)", "rows": rows}


def run_kernel_case(args, dev):
    import numpy as np
    import torch
    from mcnla_b200 import isvd, synthetic, _lib
    m, n, k, p, N = args.m, args.n, args.k, args.p, args.N
    L = (k + p) * N
    ctx = isvd.context(dev)
    if args.kernel == "trace":
        return run_trace(args, dev)
    if args.kernel == "served_trace":
        return run_served_trace(args, dev)
    if args.kernel == "gkn_scaling":
        return run_gkn_scaling(args, dev)
    if args.kernel == "ingest":
        return run_ingest(args, dev)
    if args.kernel == "syev":
        return run_syev(args, dev)
    if args.kernel == "inverse":
        return run_inverse(args, dev)
    if args.kernel == "grouped":
        # the grouped batch integrator on --batch-count copies of one shape (m x n, k, p = k/2, N = 8)
        shapes = [dict(sh, k=k, p=k // 2) for sh in synthetic.batch_shapes(args.batch_count, seed=4)]
        pool = [synthetic.lowrank_torch(m, n, np.arange(1, min(m, n) + 1) ** -1.0, seed=i, device=dev)
                for i in range(min(8, args.batch_count))]
        def reqs():
            return [isvd.Request(pool[i % len(pool)], k, k // 2, 8, seed=i, integrator="rb_gramian_kn",
                                 former="rb_gramian", maxit=args.maxit, tol=1e-5) for i in range(args.batch_count)]
        isvd.solve_grouped(reqs(), workers=args.serve_workers)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rs = isvd.solve_grouped(reqs(), workers=args.serve_workers)
        torch.cuda.synchronize()
        t = time.perf_counter() - t0
        its = [r.result.iteration for r in rs]
        del shapes
        return {"kernel": "k_gkn_grouped (grouped batch)", "m": m, "n": n, "k": k, "count": args.batch_count,
                "s": round(t, 4), "solves_per_s": round(args.batch_count / t, 2), "iterations_mean": float(np.mean(its)),
                "iterations_max": int(max(its)), "phases": isvd.grouped_times()}
    if args.kernel == "sketch_bf16":
        a = torch.randn(m, n, dtype=torch.float64, device=dev)
        sp = isvd.split_bf16(a, args.parts)
        del a
        om_t, ldo, _ = isvd.gaussian_bf16(n, L, 7, dev)
        q = torch.empty(m, L, dtype=torch.float64, device=dev)
        prm = _lib.Params(m, n, k, p, N)
        ts = []
        for _ in range(4):
            _lib.check(ctx.lib.mcnla_b200_sketch_bf16(ctx.bind(), ctypes.byref(prm), isvd._ptr(sp.hi),
                                                      isvd._ptr(sp.lo), isvd._ptr(sp.lo2), sp.ld, isvd._ptr(om_t),
                                                      ldo, isvd._ptr(q)), "sketch_bf16")
            ts.append(ctx.last_times()[1])
        t = min(ts[1:])
        return {"kernel": "bf16_gemm_kernel (sketch)", "shape": "%dx%dx%d" % (m, n, L), "parts": args.parts,
                "ms": round(t * 1e3, 4), "tflops": round(args.parts * 2.0 * m * n * L / t / 1e12, 2)}
    a = synthetic.lowrank_torch(m, n, np.arange(1, min(m, n, 256) + 1) ** -1.0, seed=1, device=dev)
    prm = isvd.Parameters(device=dev).setSize(m, n).setRank(k).setOverRank(p).setNumSketch(N).sync()
    q = prm.createCollectionQ()
    sk = isvd.GaussianProjectionSketcher(prm, 5)
    sk.initialize()
    sk(a, q)
    orth = isvd.GramianOrthogonalizer(prm)
    orth.initialize()
    orth(q)
    integ = isvd.RowBlockGramianKolmogorovNagumoIntegrator(prm, 256, 1e-5)
    integ.initialize()
    qbar = prm.createMatrixQbar()
    runs = []
    for _ in range(2):
        integ(q, qbar)
        runs.append(integ.times())
    return {"kernel": "k_gkn_persistent (row-block Gramian KN integrator)", "m": m, "n": n, "l": k + p, "N": N,
            "iterations": integ.iteration(), "stage_ms": [round(x * 1e3, 4) for x in runs[-1]]}


# ------------------------------------------------------------------------------------------------
# CPU: the reference's own stages on a bounded row sample
# ------------------------------------------------------------------------------------------------
def cpu_sample(args, rows=None):
    """Runs the reference's CPU stages (oracle/_ref when built, else the numpy
    restatement) on the first `rows` rows of a matrix with the workload's
    spectrum and parameters.  Returns (estimated seconds per full solve, info)."""
    import numpy as np
    from mcnla_b200 import synthetic
    from oracle import ref_lib
    m, n, k, p, N = args.m, args.n, args.k, args.p, args.N
    l = k + p
    rows = rows or args.cpu_rows or min(m, max(4 * l, 1024))
    sigma = np.exp(-np.arange(1, args.rank_r + 1) / 30.0)
    a = synthetic.lowrank_np(rows, n, sigma[: min(len(sigma), rows)], seed=5, noise=1e-4)
    omega = synthetic.omega_np(n, l * N, seed=5)
    cores = os.cpu_count() or 1
    scale = m / rows
    kinds = {"kn": 0, "rb_kn": 1, "rb_gramian_kn": 2, "rb_wy": 3, "rb_gramian_wy": 4}
    fkinds = {"svd": 0, "gramian": 1, "rb_gramian": 2, "cb_gramian": 3}
    if ref_lib.available():
        lib = ref_lib.load()
        lib.mref_set_threads(cores)
        t0 = time.perf_counter()
        y, t_sketch = ref_lib.sketch(lib, a, omega)
        q, t_orth = ref_lib.orthogonalize(lib, y, l, N, row_block=True, timing=True)
        qbar, it, t_int = ref_lib.integrate(lib, q, l, N, kinds[args.integrator], args.maxit, args.tol, timing=True)
        s, u, v, t_form = ref_lib.form(lib, a, qbar, k, p, fkinds[args.former], timing=True)
        wall = time.perf_counter() - t0
        # rows-proportional parts scale by m / rows; the Gramian integrators'
        # iteration part works on (N l)^2 matrices and does not
        if args.integrator.startswith("rb_gramian"):
            t_int_scaled = t_int[1] * scale + t_int[2] + t_int[3] * scale
        else:
            t_int_scaled = t_int[0] * scale
        est = t_sketch * scale + t_orth[0] * scale + t_int_scaled + t_form[0] * scale
        kind = "reference"
        detail = {"sketch_s": t_sketch, "orthogonalize_s": t_orth[0], "integrate_s": t_int[0],
                  "integrate_iterations": it, "form_s": t_form[0], "sample_wall_s": wall}
    else:
        from oracle import isvd_oracle as O
        t0 = time.perf_counter()
        r = O.isvd(a, omega, k, p, N, integrator=args.integrator,
                   former="svd" if args.former == "svd" else "gramian", maxit=args.maxit, tol=args.tol)
        wall = time.perf_counter() - t0
        est = wall * scale
        kind = "port"
        cores = 1 if os.environ.get("OMP_NUM_THREADS") == "1" else cores
        detail = {"integrate_iterations": r["iterations"], "sample_wall_s": wall}
    sample = ("first %d of %d rows (same n, k, p, N, spectrum); row-proportional stage times scaled by %.1f"
              % (rows, m, scale))
    return est, {"cores": cores, "kind": kind, "sample": sample, "detail": detail,
                 "sample_iterations": detail.get("integrate_iterations")}


def workload_matrix(args, rank=0, device=None):
    """The workload's A: U_r diag(exp(-j/30)) V_r' + 1e-4 G from the seeded generator of this
    build's arm (rank r uses seed 1000 + r).  Built on `device` (the GPU when given)."""
    import numpy as np
    from mcnla_b200 import synthetic
    sigma = np.exp(-np.arange(1, args.rank_r + 1) / 30.0)
    return synthetic.lowrank_torch(args.m, args.n, sigma, seed=1000 + rank, noise=1e-4,
                                   device=device or "cpu", colmajor=args.colmajor)


def reconstruction_error_np(a, s, u, v, chunk=8192):
    """||A - U diag(S) V'||_F / ||A||_F, the reference drivers' check (src/isvd_dense_rb.cpp:291-315),
    in row chunks of A."""
    import numpy as np
    num = den = 0.0
    us = u * s
    for r0 in range(0, a.shape[0], chunk):
        blk = np.asarray(a[r0:r0 + chunk])
        num += float(np.sum((blk - us[r0:r0 + chunk] @ v.T) ** 2))
        den += float(np.sum(blk * blk))
    return (num / den) ** 0.5


def reconstruction_error_torch(a, s, u, v, chunk=8192):
    """The same check on the device (a may be a column-major view)."""
    num = den = 0.0
    us = u * s
    for r0 in range(0, a.shape[0], chunk):
        blk = a[r0:r0 + chunk]
        num += float(((blk - us[r0:r0 + chunk] @ v.t()) ** 2).sum().item())
        den += float((blk * blk).sum().item())
    return (num / den) ** 0.5


REF_KINDS = {"kn": 0, "rb_kn": 1, "rb_gramian_kn": 2, "rb_wy": 3, "rb_gramian_wy": 4}
REF_FORMERS = {"svd": 0, "gramian": 1, "rb_gramian": 2, "cb_gramian": 3}


def ref_solver(lib, a, omega, k, p, N, integrator, former, maxit, tol, colmajor=False, row_block=True):
    """The reference's own stages (oracle/_ref) set up for repeated whole solves: A and Omega
    loaded and the stages initialized once (the reference drivers' order, src/isvd_dense_rb.cpp:
    118-221); each run() reports the stages' own timers (report/include/stage.hpp pattern)."""
    from oracle import ref_lib
    return ref_lib.Solver(lib, a, omega, k, p, N, REF_KINDS[integrator], REF_FORMERS[former], maxit, tol,
                          colmajor=colmajor, row_block=row_block)


def config1_inputs():
    """Configuration 1: A = U diag(1/j) V' (1000 x 2000, U and V the Q factors of seeded
    Gaussians), Omega 2000 x 320 N(0,1) from seed 0; k = 10, p = 10, N = 16."""
    from mcnla_b200 import synthetic
    return synthetic.config1_numpy(m=1000, n=2000, k=10, p=10, N=16, seed=0)


CONFIG1 = {"workload": "plain iSVD, A = U diag(1/j) V', m=1000 n=2000, k=10 p=10 N=16, Omega N(0,1) seed 0",
           "stages": "Gramian / KolmogorovNagumo (tol 1e-4, maxit 256) / Svd"}


def run_reference_config1(lib, steps, warmup):
    """Configuration 1 in full through the reference's stages: `steps` timed solves, each the
    sum of the stages' own timers (the reference driver's "total computing time")."""
    a, omega = config1_inputs()
    sol = ref_solver(lib, a, omega, 10, 10, 16, "kn", "svd", 256, 1e-4, row_block=False)
    for _ in range(max(1, warmup)):
        sol.run()
    totals, it = [], None
    for _ in range(steps):
        it, t = sol.run()
        totals.append(float(t.sum()))
    s, u, v = sol.result()
    sol.close()
    mean = sum(totals) / len(totals)
    return {**CONFIG1, "value": round(1.0 / mean, 4), "unit": "iSVD/s", "ms_per_step": round(mean * 1e3, 3),
            "steps": steps, "iterations": it, "reconstruction_rel_err": reconstruction_error_np(a, s, u, v),
            "sigma": [float(x) for x in s[:3]]}


def run_reference(args, world, rank):
    """The reference's own CPU stages (oracle/_ref, OpenBLAS on all host threads) on the full
    workload: the same A as this build's arm (its generator and seed; built on the GPU when
    there is one, then copied to host memory) and a seeded N(0,1) Omega.  Each timed step is
    one whole solve on the full matrix.  Warm-up steps run the stages on a 1024-row sample
    (they only warm the BLAS threads and caches).  Timed steps stop early, before a step that
    would end past --ref-budget seconds, and `steps` reports how many ran."""
    if rank != 0:
        return None
    import numpy as np
    from oracle import ref_lib
    from mcnla_b200 import synthetic
    if not ref_lib.available():
        return {"metric": METRIC, "impl": "reference", "unavailable": "oracle/_ref (the reference compiled here) is missing"}
    lib = ref_lib.load()
    cores = os.cpu_count() or 1
    lib.mref_set_threads(cores)
    k, p, N = args.k, args.p, args.N
    L = (k + p) * N
    gpu = False
    try:
        import torch
        gpu = torch.cuda.is_available()
    except Exception:
        pass
    t_setup = time.perf_counter()
    at = workload_matrix(args, 0, device="cuda" if gpu else None)
    a = (at.t() if args.colmajor else at).contiguous().cpu().numpy()
    a = a.T if args.colmajor else a           # column-major A is the transpose of a C-ordered n x m buffer
    del at
    if gpu:
        torch.cuda.empty_cache()
    omega = synthetic.omega_np(args.n, L, seed=5)
    setup_s = time.perf_counter() - t_setup
    t_init = time.perf_counter()
    sol = ref_solver(lib, a, omega, k, p, N, args.integrator, args.former, args.maxit, args.tol,
                     colmajor=args.colmajor)
    init_s = time.perf_counter() - t_init
    for _ in range(args.warmup):
        cpu_sample(args)
    totals, stage_times, iters = [], [], []
    t_begin = time.perf_counter()
    while len(totals) < args.steps:
        if totals and (time.perf_counter() - t_begin) + 1.1 * max(totals) > args.ref_budget:
            break
        it, t = sol.run()
        totals.append(float(t.sum()))
        stage_times.append(t)
        iters.append(it)
    timed_wall = time.perf_counter() - t_begin
    s, u, v = sol.result()
    sol.close()
    mean = sum(totals) / len(totals)
    value = 1.0 / mean
    names = ("sketch_s", "orthogonalize_s", "integrate_s", "form_s")
    detail = {nm: round(float(sum(t[i] for t in stage_times)) / len(stage_times), 4) for i, nm in enumerate(names)}
    c1 = run_reference_config1(lib, args.steps, args.warmup) if not args.quick else None
    return {
        "metric": METRIC, "value": round(value, 6), "unit": "iSVD/s", "n_gpus": world, "steps": len(totals),
        "steps_requested": args.steps, "warmup": args.warmup, "ms_per_step": round(mean * 1e3, 3),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)", "impl": "reference",
        "config": dict(workload(args), parallelism="host CPU"),
        "cpu_baseline": {"value": round(value, 6), "unit": "iSVD/s", "cores": cores, "kind": "reference",
                         "sample": "none: every timed step is one whole solve of the full %d x %d matrix "
                                   "(warm-ups on a 1024-row sample)" % (args.m, args.n)},
        "e2e": {"value": round(value, 6), "unit": "iSVD/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timing": "per step the sum of the four stages' own timers (the reference driver's total computing "
                  "time; A and Omega loaded and the stages initialized once before, as its drivers do)",
        "a_read_gbs": round(2 * args.m * args.n * 8 / mean / 1e9, 3),
        "iterations": iters[-1], "iterations_all": iters, "stage_s": detail, "setup_s": round(setup_s, 1),
        "budget_s": args.ref_budget, "timed_wall_s": round(timed_wall, 1), "init_s": round(init_s, 1),
        "reconstruction_rel_err": reconstruction_error_np(a, s, u, v),
        "config1": c1,
    }


def main():
    args = parse()
    world, rank, local = dist_init(args)
    if args.impl == "reference":
        res = run_reference(args, world, rank)
    elif args.kernel:
        import torch
        torch.cuda.set_device(local)
        res = run_kernel_case(args, torch.device("cuda", local))
    elif args.only_serving:
        import torch
        torch.cuda.set_device(local)
        res = {"metric": METRIC, "serving": run_serving(args, torch.device("cuda", local))}
    else:
        res = run_b200(args, world, rank, local)
        if world == 1 and not args.no_serving:
            import torch
            torch.cuda.empty_cache()
            try:
                res["serving"] = run_serving(args, torch.device("cuda", local))
            except Exception as e:          # the headline line is printed whatever this leg does
                res["serving"] = {"error": "%s: %s" % (type(e).__name__, e)}
                torch.cuda.synchronize()
        if rank == 0 and world == 1 and not args.no_cpu_baseline:
            est, info = cpu_sample(args)
            res["cpu_baseline"] = {"value": round(1.0 / est, 6), "unit": "iSVD/s", "cores": info["cores"],
                                   "kind": info["kind"], "sample": info["sample"], "estimated": True,
                                   "sample_iterations": info["sample_iterations"],
                                   "full_run_iterations": res.get("iterations")}
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
