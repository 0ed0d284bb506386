#!/usr/bin/env python
"""Benchmark of the Nyström operator application on B200.

Workload (the single-GPU configuration the headline metric is quoted on):
3D Helmholtz single layer, k = 10, FP64 complex, matrix-free, on the unit
sphere meshed by 10,368 quadratic triangles with the 6-point VR rule
(N = 62,208 nodes), plus its DIM correction (6 nonzeros per row) applied as a
CSR SpMV fused into the pair kernel's epilogue.  Density: complex Gaussian,
seed 1.  One step = one y = (A + δS) σ over all N² node pairs (the symmetric
kernel of square operators evaluates each unordered pair once for both
products; the metric counts the N² ordered pairs of the product).

value   kernel-pairs/s (G) with σ and y resident in HBM; L2 flushed between
        steps (a 256 MiB write, untimed), each step timed with CUDA events on
        the library's stream.  With N > 1 ranks (torchrun) the target rows of
        the one operator are split over the ranks and y is all-gathered over
        NCCL inside every step (--shard rows, strong scaling; --shard replicas
        runs independent copies instead); time = max over ranks.
e2e     the same metric through the public API (GpuOperator.mul with pinned
        host buffers): host->device copy of σ, the apply, device->host copy
        of y, every step.
gmres   (extra key) time to ||b - Lx|| <= 1e-10 ||b|| for the 3D Laplace
        combined field ½I + D + S on the (1, 0.7, 0.5) ellipsoid, N = 200,934,
        plain FP64 GMRES versus FP32-inner / FP64-outer refinement.

Other workloads (--workload): c2_dl, c2_adl, c2_hs, c3_dl_fp64, c3_dl_fp32c, c3_sl_fp64, c1
(single operators); c4 (batched surfaces x 64 right-hand sides, TF32 tensor
cores and FP64 MMA, --nsurf surfaces); c5 (adjoint); csr (correction SpMV
bandwidth); dim_c2, dim_c3 (GPU construction of the DIM correction).

--impl reference times the reference's CPU algorithm for the same step
(Inti's on-the-fly row sums, restated in C++ as the oracle) on all host
cores, each step a bounded sample of rows scaled to the metric.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "inti.jl_b200"))

import numpy as np  # noqa: E402

METRIC = "G kernel-pairs/s"
UNIT = "Gpairs/s"
# Algorithmic flops per pair (FMA = 2 flops; special functions counted apart)
FLOPS_PER_PAIR = {"helmholtz_sl": 24, "helmholtz_dl": 34, "laplace_sl": 11, "laplace_dl": 18, "laplace2d_dl": 10,
                  # the same count for the adjoint double layer (r.n_x in place of r.n_y) and the
                  # hypersingular kernel: + n_x.n_y, the 1/d^5 term and its complex factor
                  "helmholtz_adl": 34, "helmholtz_hs": 60}
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one pair-kernel
# launch per workload, from the ncu capture of that launch summarised in
# profiles/ (the file named beside each entry); None where no capture exists.
PAIR_TRAFFIC_BYTES = {"c2": (66.74e6, "profiles/pair_symm_helmholtz_sl_fp64_p2sphere62k.md")}
CSR_TRAFFIC_BYTES = (527.0e6, "profiles/csr_bulk_kernel_dim_pattern_c3x20.md")
# Fallback HBM copy bandwidth (GB/s) when MEASURED_PEAKS.json is absent
HBM_FALLBACK_GBS = 6650.0


def hbm_peak() -> tuple[float, str]:
    """The measured HBM copy bandwidth of this pool's B200s
    (MEASURED_PEAKS.json, written by the driver), else the fallback."""
    try:
        with open(ROOT / "MEASURED_PEAKS.json") as f:
            return float(json.load(f)["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs, of measured"
    except (OSError, KeyError, ValueError):
        return HBM_FALLBACK_GBS, "fallback 6.65 TB/s (MEASURED_PEAKS.json absent), of fallback"
# Algorithmic flops per pair of the source-gradient (adjoint) pass
ADJ_FLOPS_PER_PAIR = {"laplace_dl": 40, "laplace_sl": 19}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, device: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(device), f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "50"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        # nvidia-smi takes a while to start: wait (bounded) for its first
        # sample so that short timed regions are covered
        t0 = time.perf_counter()
        while self.p is not None and time.perf_counter() - t0 < 10.0:
            if Path(self.f.name).stat().st_size > 0:
                break
            time.sleep(0.05)

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        for line in Path(self.f.name).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_workload(name: str, ctx):
    """(quadrature, operator, density, flops key, dtype, config) of a named
    workload.  "c2" is the headline; the others exist to time and profile
    the other pair kernels with the same driver."""
    import inti_b200 as inti

    r = np.random.default_rng(1)
    if name == "c2":
        q = inti.p2_sphere_quadrature(36)
        op = inti.Helmholtz(k=10.0, dim=3)
        kern, key, prec, dt = inti.SingleLayerKernel(op), "helmholtz_sl", "fp64", "c128"
        wl = "helmholtz3d_sl_k10_p2sphere_N62208_dim"
    elif name == "c2_dl":
        q = inti.p2_sphere_quadrature(36)
        op = inti.Helmholtz(k=10.0, dim=3)
        kern, key, prec, dt = inti.DoubleLayerKernel(op), "helmholtz_dl", "fp64", "c128"
        wl = "helmholtz3d_dl_k10_p2sphere_N62208_dim"
    elif name in ("c2_adl", "c2_hs"):
        q = inti.p2_sphere_quadrature(36)
        op = inti.Helmholtz(k=10.0, dim=3)
        hs = name == "c2_hs"
        kern = inti.HyperSingularKernel(op) if hs else inti.AdjointDoubleLayerKernel(op)
        key, prec, dt = ("helmholtz_hs" if hs else "helmholtz_adl"), "fp64", "c128"
        wl = f"helmholtz3d_{'hs' if hs else 'adl'}_k10_p2sphere_N62208_dim"
    elif name in ("c3_dl_fp64", "c3_dl_fp32c", "c3_sl_fp64"):
        q = inti.ellipsoid_quadrature(61, 5)
        op = inti.Laplace(dim=3)
        prec = "fp32c" if name.endswith("fp32c") else "fp64"
        sl = name.startswith("c3_sl")
        kern = inti.SingleLayerKernel(op) if sl else inti.DoubleLayerKernel(op)
        key, dt = ("laplace_sl" if sl else "laplace_dl"), ("f32" if prec == "fp32c" else "f64")
        wl = f"laplace3d_{'sl' if sl else 'dl'}_ellipsoid_N200934_dim_{prec}"
    elif name == "c1":
        q = inti.kite_quadrature(200, 9)
        op = inti.Laplace(dim=2)
        kern, key, prec, dt = inti.DoubleLayerKernel(op), "laplace2d_dl", "fp64", "f64"
        wl = "laplace2d_dl_kite_N1000_dim"
    else:
        raise SystemExit(f"unknown workload {name}")
    deriv = isinstance(kern, (inti.AdjointDoubleLayerKernel, inti.HyperSingularKernel))
    t0 = time.perf_counter()
    dS, dD = inti.bdim_correction(op, q, q, derivative=deriv, ctx=ctx)  # derivative: (ADL, HS) corrections
    t_dim = time.perf_counter() - t0
    corr = dS if isinstance(kern, (inti.SingleLayerKernel, inti.AdjointDoubleLayerKernel)) else dD
    A = inti.GpuOperator(kern, q, q, corr, prec, ctx)
    n = len(q)
    if A.is_complex:
        sigma = (r.standard_normal(n) + 1j * r.standard_normal(n)) / np.sqrt(2)
    else:
        sigma = r.standard_normal(n)
    cfg = {"workload": wl, "n": n, "nnz_per_row": q.nq, "precision": prec, "dim_setup_s": t_dim}
    return q, A, sigma, key, dt, cfg


def cpu_sample(q, A, sigma, seconds: float, nthreads: int) -> dict:
    """The oracle's on-the-fly FP64 row sums on a bounded sample of rows (the
    whole product, repeated for the sample time, when one product is short);
    for operators of at most 5,000 nodes also Inti's dense path (assembly once,
    then gemv + CSR per product) as `dense_path`."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O

    n = len(q)
    pde = O.HELMHOLTZ if A.is_complex else O.LAPLACE
    k = float(getattr(A.kernel.op, "k", 0.0))
    args = (pde, A.kernel.kind, k, q.coords, q.normals, q.coords, q.normals, q.weights, sigma)
    t0 = time.perf_counter()
    rows0 = max(8 * nthreads, 32)
    O.apply_rows_block(*args, 0, rows0, nthreads=nthreads)
    dt = time.perf_counter() - t0
    rows = int(min(n, max(rows0, rows0 * seconds / max(dt, 1e-6))))
    if rows < n:
        t0 = time.perf_counter()
        O.apply_rows_block(*args, 0, rows, nthreads=nthreads)
        dt = time.perf_counter() - t0
        return {"value": rows * n / dt / 1e9, "unit": UNIT, "cores": nthreads, "kind": "port",
                "sample": f"{rows} of {n} target rows x {n} sources (C++ FP64 restatement of Inti's "
                          f"on-the-fly row sums), {dt:.1f} s"}
    # the whole product is short: repeat it for the sample time and average
    O.apply_rows_block(*args, 0, n, nthreads=nthreads)
    reps, t0 = 0, time.perf_counter()
    while reps < 3 or time.perf_counter() - t0 < seconds / 2:
        O.apply_rows_block(*args, 0, n, nthreads=nthreads)
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    out = {"value": n * n / dt / 1e9, "unit": UNIT, "cores": nthreads, "kind": "port",
           "sample": f"all {n} target rows x {n} sources (C++ FP64 restatement of Inti's on-the-fly row "
                     f"sums), mean of {reps} products, {dt * reps:.1f} s"}
    if n > 5000:
        return out
    # Inti's own path at this size (compression = :none): the matrix assembled
    # once, column-threaded (src/nystrom.jl:117-124), then one gemv per product
    # plus the correction's sparse product
    t0 = time.perf_counter()
    M = O.assemble(pde, A.kernel.kind, k, q.coords, q.normals, q.coords, q.normals, q.weights, nthreads=nthreads)
    t_asm = time.perf_counter() - t0
    corr = A.correction.arrays() if A.correction is not None else None
    if corr is not None:
        O.csr_apply(*corr, sigma)  # warm-up
    y = M @ sigma
    reps, t0 = 0, time.perf_counter()
    while reps < 3 or time.perf_counter() - t0 < seconds / 4:
        y = M @ sigma
        if corr is not None:
            y = y + O.csr_apply(*corr, sigma)
        reps += 1
    t_mv = (time.perf_counter() - t0) / reps
    out["dense_path"] = {"assemble_s": t_asm, "matvec_ms": t_mv * 1e3, "value": n * n / t_mv / 1e9,
                         "unit": UNIT, "threads": f"assembly {nthreads}, gemv numpy BLAS",
                         "sample": f"one assembly of the {n} x {n} matrix, mean of {reps} gemv + CSR products"}
    return out


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, str(ROOT / "oracle"))
    import inti_b200.geometry as G
    import oracle as O

    q = G.p2_sphere_quadrature(36)
    r = np.random.default_rng(1)
    sigma = (r.standard_normal(len(q)) + 1j * r.standard_normal(len(q))) / np.sqrt(2)
    nt = host_cores()
    n = len(q)
    budget = max(60.0 / max(args.steps + args.warmup, 1), 2.0)  # whole run within a few minutes
    sargs = (O.HELMHOLTZ, O.SL, 10.0, q.coords, q.normals, q.coords, q.normals, q.weights, sigma)
    t0 = time.perf_counter()
    O.apply_rows_block(*sargs, 0, 8 * nt, nthreads=nt)
    rate = 8 * nt / (time.perf_counter() - t0)
    rows = int(min(n, max(8 * nt, rate * budget)))
    for _ in range(args.warmup):
        O.apply_rows_block(*sargs, 0, min(rows, 8 * nt), nthreads=nt)
    times = []
    for s in range(args.steps):
        row0 = (s * rows) % max(n - rows, 1)
        t0 = time.perf_counter()
        O.apply_rows_block(*sargs, row0, rows, nthreads=nt)
        times.append(time.perf_counter() - t0)
    per = statistics.mean(times)
    value = rows * n / per / 1e9
    full_ms = per * (n / rows) * 1e3
    sample = (f"{rows} of {n} target rows x {n} sources per step (the C++ FP64 restatement of Inti's "
              f"on-the-fly row sums): sampled rows, pair sums only (the 6-per-row DIM correction SpMV is not "
              f"timed), rate extrapolated to the full product")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": per * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
        "config": {"workload": "helmholtz3d_sl_k10_p2sphere_N62208_dim", "n": n, "nnz_per_row": 6,
                   "step": "sampled rows, extrapolated, pair sums only", "rows_per_step": rows,
                   "full_product_ms_extrapolated": full_ms},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nt, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def solve_both(inti, make_L, b, restart: int) -> dict:
    """FP64 and MIXED GMRES on L x = b to 1e-10.  `seconds` is the wall time
    of the whole solve call, from the upload of b to x back on the host.
    Each mode starts from freshly created operators (`make_L()`, the DIM
    corrections already built), so its first solve includes the operator
    set-up it triggers: the fused combined field, and for MIXED the FP32C
    twins (`setup_s` is that part).  The same operators are then solved a
    second time, set-up cached, as `seconds_repeat`."""
    out = {}
    for mode in ("fp64", "mixed"):
        L = make_L()
        _, st = inti.gmres(L, b, rtol=1e-10, restart=restart, maxiter=500, mode=mode)
        _, st2 = inti.gmres(L, b, rtol=1e-10, restart=restart, maxiter=500, mode=mode)
        out[mode] = {"seconds": st["seconds"], "setup_s": st["setup_seconds"], "seconds_repeat": st2["seconds"],
                     "iterations": st["iterations"], "outer": st["outer"],
                     "fp64_applies": st["fp64_applies"], "fp32_applies": st["fp32_applies"],
                     "relres_fp64": st["relres"], "converged": bool(st["converged"] and st2["converged"])}
        del L
    if out["fp64"]["converged"] and out["mixed"]["converged"]:
        out["mixed_speedup_vs_fp64"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
        out["mixed_speedup_vs_fp64_repeat"] = out["fp64"]["seconds_repeat"] / out["mixed"]["seconds_repeat"]
    out["timing"] = ("wall time of the whole solve call from the upload of b to x on the host; the first solve "
                     "of each mode on fresh operators (includes the set-up it triggers), the repeat with it cached")
    return out


def gmres_c2_cfie(ctx) -> dict:
    """Sound-soft scattering on the C2 sphere (P2, N = 62,208), k = 10: the
    Brakhage-Werner combined field (1/2 I + D - i k S) sigma = -u_inc
    (docs/src/examples/helmholtz_scattering.jl:485-495) with u_inc a plane
    wave, both layers DIM-corrected.  A single-RHS Helmholtz solve that
    needs more Krylov iterations than the C3 Laplace one."""
    import inti_b200 as inti

    k = 10.0
    q = inti.p2_sphere_quadrature(36)
    op = inti.Helmholtz(k=k, dim=3)
    t0 = time.perf_counter()
    dS, dD = inti.bdim_correction(op, q, q, ctx=ctx)
    t_setup = time.perf_counter() - t0
    d = np.array([0.3, -0.5, 0.81])
    d /= np.linalg.norm(d)
    b = -np.exp(1j * k * (q.coords @ d))

    def make_L():
        S = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, dS, "fp64", ctx)
        D = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, dD, "fp64", ctx)
        return 0.5 * inti.I + D - 1j * k * S

    out = {"workload": "helmholtz3d_cfie(0.5I+D-ikS)_k10_p2sphere_N62208_dim", "n": len(q), "rtol": 1e-10,
           "setup_s": t_setup}
    out.update(solve_both(inti, make_L, b, restart=100))
    return out


def gmres_c1(ctx, S_unused, D, q, cpu: bool) -> dict:
    """The interior Dirichlet problem of the C1 kite, (-I/2 + D) sigma = g with
    g the trace of a point source outside (docs/src/examples/poisson.jl:160-168),
    FP64 GMRES to 1e-10 on the GPU (the small-system Arnoldi form), first solve
    and repeat; beside it the oracle's FP64 GMRES (C++ on-the-fly row sums on
    all host cores) on the same system."""
    import inti_b200 as inti

    xs = np.array([3.0, 2.0])
    b = -np.log(np.linalg.norm(q.coords - xs, axis=1)) / (2 * np.pi)
    L = D - 0.5 * inti.I
    _, st = inti.gmres(L, b, rtol=1e-10, restart=100, maxiter=500)
    reps = [inti.gmres(L, b, rtol=1e-10, restart=100, maxiter=500)[1]["seconds"] for _ in range(5)]
    out = {"workload": "laplace2d_interior_dirichlet(-0.5I+D)_kite_N1000_dim", "rtol": 1e-10,
           "fp64": {"seconds": st["seconds"], "seconds_repeat": statistics.median(reps),
                    "iterations": st["iterations"], "fp64_applies": st["fp64_applies"], "relres_fp64": st["relres"],
                    "converged": bool(st["converged"])},
           "timing": "wall time of the whole solve call (b up, x back); repeat = median of 5"}
    if cpu:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        nt = host_cores()
        dD = D.correction.arrays()
        O.gmres(O.LAPLACE, 0.0, q.coords, q.normals, q.weights, -0.5, [(O.DL, 1.0, dD)], b, rtol=1e-10,
                restart=100, maxiter=500, nthreads=nt)
        t0 = time.perf_counter()
        _, sto = O.gmres(O.LAPLACE, 0.0, q.coords, q.normals, q.weights, -0.5, [(O.DL, 1.0, dD)], b, rtol=1e-10,
                         restart=100, maxiter=500, nthreads=nt)
        out["cpu_fp64"] = {"seconds": time.perf_counter() - t0, "iterations": sto["iterations"], "cores": nt,
                           "kind": "port", "sample": "the whole solve (C++ FP64 restatement, on-the-fly row sums)"}
    return out


def gmres_c3(ctx, cpu_seconds: float | None = None) -> dict:
    """Combined-field Laplace solve on the ellipsoid (N = 200,934).  With
    cpu_seconds, also the CPU estimate of the same FP64 solve: the oracle's
    D and S row sums (the reference's on-the-fly matvec) timed on a sample
    of rows on all host cores, extrapolated to a full product and multiplied
    by the GPU solve's count of operator applications."""
    import inti_b200 as inti

    q = inti.ellipsoid_quadrature(61, 5)
    op = inti.Laplace(dim=3)
    t0 = time.perf_counter()
    dS, dD = inti.bdim_correction(op, q, q, ctx=ctx)
    t_setup = time.perf_counter() - t0
    r = np.random.default_rng(8)
    src = r.uniform(-1, 1, (64, 3))
    src = src[np.sum((src / np.array([0.5, 0.35, 0.25])) ** 2, 1) < 1][:8]  # inside the 0.5-scaled ellipsoid
    c = r.standard_normal(len(src))
    d = np.linalg.norm(q.coords[:, None, :] - src[None, :, :], axis=2)
    b = (c[None, :] / (4 * np.pi * d)).sum(1)
    def make_L():
        S = inti.GpuOperator(inti.SingleLayerKernel(op), q, q, dS, "fp64", ctx)
        D = inti.GpuOperator(inti.DoubleLayerKernel(op), q, q, dD, "fp64", ctx)
        return 0.5 * inti.I + D + S

    out = {"workload": "laplace3d_cfie(0.5I+D+S)_ellipsoid_N200934_dim", "n": len(q), "rtol": 1e-10,
           "setup_s": t_setup}
    out.update(solve_both(inti, make_L, b, restart=100))
    if cpu_seconds:
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        nt, n = host_cores(), len(q)
        rows = max(8 * nt, 32)
        per_row = 0.0
        for kind in (O.DL, O.SL):
            args = (O.LAPLACE, kind, 0.0, q.coords, q.normals, q.coords, q.normals, q.weights, b)
            t0 = time.perf_counter()
            O.apply_rows_block(*args, 0, rows, nthreads=nt)
            dt = time.perf_counter() - t0
            r2 = int(min(n, max(rows, rows * cpu_seconds / 2 / max(dt, 1e-6))))
            t0 = time.perf_counter()
            O.apply_rows_block(*args, 0, r2, nthreads=nt)
            per_row += (time.perf_counter() - t0) / r2
        matvec = per_row * n
        out["cpu_fp64_estimate"] = {
            "seconds": matvec * out["fp64"]["fp64_applies"], "matvec_s": matvec, "cores": nt,
            "kind": "port, extrapolated",
            "sample": "D and S row sums of the C++ FP64 restatement on a sample of rows, scaled to a full "
                      "product and multiplied by the FP64 solve's operator applications"}
    return out


def bench_dim(args, ctx, peaks, torch) -> dict:
    """GPU construction of the on-surface DIM correction (bdim_correction,
    src/bdim.jl:50-196) of the C2 operator (Helmholtz k = 10, P2 sphere,
    N = 62,208, ns = 18) or the C3 operator (Laplace, ellipsoid, N = 200,934,
    ns = 27): traces, the Θ pair product over all node pairs on the FP64 MMA
    path, per-element least squares, CSR assembly.  value = seconds per
    construction (wall clock around the call, synchronised)."""
    import inti_b200 as inti

    if args.workload == "dim_c2":
        q, op, work = inti.p2_sphere_quadrature(36), inti.Helmholtz(k=10.0, dim=3), "helmholtz3d_dim_k10_p2sphere_N62208"
        flops_pair = 24 + 34 + 16 * 18  # S and D values, 2 complex multiply-adds per column
    else:
        q, op, work = inti.ellipsoid_quadrature(61, 5), inti.Laplace(dim=3), "laplace3d_dim_ellipsoid_N200934"
        flops_pair = 11 + 18 + 4 * 27
    n = len(q)
    for _ in range(args.warmup):
        inti.bdim_correction(op, q, q, ctx=ctx)
    ctx.synchronize()
    clocks = Clocks(0)
    launches0 = ctx.launch_count
    ctx.set_profiling(True)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        dS, dD = inti.bdim_correction(op, q, q, ctx=ctx)
    ctx.synchronize()
    wall = (time.perf_counter() - t0) / args.steps
    theta_ms, theta_launches = ctx.profile("dim")
    ctx.set_profiling(False)
    clk = clocks.stop()
    theta_ms /= args.steps
    achieved = float(n) * n * flops_pair / (theta_ms * 1e-3) / 1e12
    fp64 = peaks["fp64_flops"] / 1e12
    return {"metric": "DIM construction time", "value": wall, "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": wall * 1e3, "higher_is_better": False, "scaling": "none",
            "vs_baseline": None, "dtype": "c128" if isinstance(op, inti.Helmholtz) else "f64", "data": "synthetic",
            "config": {"workload": work, "n": n, "nnz_per_row": dS.nnz // n, "l2": "inputs (traces, partials) "
                       "larger than L2 are not flushed: each step rebuilds everything"},
            "roofline": {"bound": "fp64", "kernel": "dim_theta_mma + dim_theta_reduce", "kernel_ms": theta_ms,
                         "achieved": achieved, "peak": fp64, "unit": "TFLOP/s", "frac": achieved / fp64,
                         "flops_per_pair": flops_pair, "traffic": None,
                         "peak_source": "FP64 FMA throughput measured in this run (inti_measure_peaks), of measured"},
            "gpu_launches": (ctx.launch_count - launches0) // args.steps, "clocks": clk}


def build_c4(ctx, nsurf: int = 32, nrhs: int = 64, seed: int = 4):
    """32 seeded star surfaces r = 1 + 0.2*sum a_lm Y_lm (l <= 3), n x n cells
    per cube-sphere patch with n in [6, 27] (N_s = 54 n^2: 1,944 .. 39,366
    nodes), GL3x3; Helmholtz k = 5 combined field D - i k S with per-surface
    DIM corrections; 64 plane waves exp(i k d.x), d uniform on the sphere."""
    import inti_b200 as inti

    r = np.random.default_rng(seed)
    ns = r.integers(6, 28, nsurf)
    quads = [inti.star_quadrature(inti.star_coefficients(r), int(n)) for n in ns]
    k = 5.0
    op = inti.Helmholtz(k=k, dim=3)
    t0 = time.perf_counter()
    corrs = [inti.bdim_correction(op, q, q, ctx=ctx) for q in quads]
    t_dim = time.perf_counter() - t0
    B = inti.BatchOperator(op, quads, "CF", corrs, 1.0, -1j * k, ctx=ctx)
    d = r.standard_normal((nrhs, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    X = np.concatenate([np.exp(1j * k * (q.coords @ d.T)) for q in quads], axis=0)
    pairs = float(sum(len(q) ** 2 for q in quads))
    cfg = {"workload": f"helmholtz3d_cfie_k5_{nsurf}stars_64rhs_dim", "surfaces": nsurf, "n_total": B.n,
           "n_min": int(min(len(q) for q in quads)), "n_max": int(max(len(q) for q in quads)), "nrhs": nrhs,
           "sum_n2": pairs, "dim_setup_s": t_dim}
    return B, X, pairs, cfg, quads


def bench_batch(args, ctx, peaks, torch) -> dict:
    """Batched multi-RHS apply (config 4): value = kernel pairs x right-hand
    sides per second through the TF32 tensor-core path."""
    B, X, pairs, cfg, quads = build_c4(ctx, nsurf=args.nsurf)
    nrhs = X.shape[1]
    dev = torch.device("cuda:0")
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    xs = torch.from_numpy(np.asfortranarray(X).T.copy().view(np.float64)).to(dev)  # column-major: col c at c*n
    ys = torch.zeros_like(xs)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    out = {}
    for prec in ("tf32", "fp64"):
        steps = args.steps if prec == "tf32" else max(3, args.steps // 10)
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                B.apply_device(xs.data_ptr(), ys.data_ptr(), nrhs, prec)
            stream.synchronize()
            clocks = Clocks(0) if prec == "tf32" else None
            launches0 = ctx.launch_count
            ctx.set_profiling(True)
            evs = []
            for _ in range(steps):
                flush.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                B.apply_device(xs.data_ptr(), ys.data_ptr(), nrhs, prec)
                e1.record(stream)
                evs.append((e0, e1))
            stream.synchronize()
            ms = sum(a.elapsed_time(b) for a, b in evs) / steps
            kern = ctx.profile("batch_tc" if prec == "tf32" else "batch")
            pack = ctx.profile("batch_pack")
            ctx.set_profiling(False)
            out[prec] = {"ms": ms, "value": pairs * nrhs / (ms * 1e-3) / 1e9, "kernel_ms": kern[0] / max(kern[1], 1),
                         "pack_ms": pack[0] / max(pack[1], 1) if pack[1] else 0.0,
                         "launches": ctx.launch_count - launches0}
            if clocks:
                out[prec]["clocks"] = clocks.stop()
    # e2e: host (pinned) densities through BatchOperator.apply
    # pinned host buffers in column-major order (torch stores row-major: use the transpose view)
    hx = torch.from_numpy(np.ascontiguousarray(X.T)).pin_memory().numpy().T
    hy = torch.zeros((nrhs, B.n), dtype=torch.complex128).pin_memory().numpy().T
    for _ in range(2):
        B.apply(hx, "tf32", Y=hy)
    t0 = time.perf_counter()
    e2steps = max(3, args.steps // 3)
    for _ in range(e2steps):
        B.apply(hx, "tf32", Y=hy)
    e2e_s = (time.perf_counter() - t0) / e2steps
    tf = out["tf32"]
    # tensor work actually issued: per surface M x K x N = (targets padded to 256) x
    # (2 x sources padded to 32) x 128, two flops per multiply-add
    flops = sum(2.0 * (-(-len(q) // 256) * 256) * (2 * (-(-len(q) // 32) * 32)) * 128 for q in quads)
    tc_peak = peaks["tf32_flops"] / 1e12  # tcgen05 kind::tf32 MMA throughput measured in this run
    achieved = flops / (tf["kernel_ms"] * 1e-3) / 1e12
    line = {
        "metric": METRIC, "value": tf["value"], "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": tf["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "tf32", "data": "synthetic",
        "config": dict(cfg, precision="tf32 tensor cores, fp32 accumulate, fp64 correction", l2="flushed between steps",
                       unit_note="pairs x right-hand sides"),
        "e2e": {"value": pairs * nrhs / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": 16 * B.n * nrhs,
                "d2h_bytes_per_step": 16 * B.n * nrhs, "ms_per_step": e2e_s * 1e3},
        "gpu_launches": tf["launches"],
        "roofline": {"bound": "tensor", "achieved": achieved, "peak": tc_peak, "unit": "TFLOP/s",
                     "frac": achieved / tc_peak, "traffic": None, "kernel": "mrhs_tc_kernel (tcgen05.mma kind::tf32)",
                     "kernel_ms": tf["kernel_ms"],
                     "peak_source": "tcgen05.mma kind::tf32 (M=N=128, K=8) throughput measured in this run "
                                    "(inti_measure_peak_tf32), of measured; half the MEASURED_PEAKS.json bf16 "
                                    "cuBLAS burst would be 828.4",
                     "frac_of_half_bf16": achieved / 828.4},
        "clocks": tf.get("clocks"),
        "fp64_batch": {"value": out["fp64"]["value"], "ms": out["fp64"]["ms"]},
        "peaks_measured": {k: v / 1e12 for k, v in peaks.items()},
    }
    if not args.no_cpu:
        # the reference applies its operator one right-hand side at a time: the
        # oracle's D and S row sums (the combined field needs both passes) on a
        # bounded sample of rows of the largest surface, one RHS, all host cores
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        big = int(np.argmax([len(q) for q in quads]))
        qb, nb = quads[big], len(quads[big])
        off = int(sum(len(q) for q in quads[:big]))
        xcol = np.ascontiguousarray(X[off:off + nb, 0])
        nthreads = host_cores()
        rows = max(8 * nthreads, 64)
        while True:
            t0 = time.perf_counter()
            for kind in (O.DL, O.SL):
                O.apply_rows_block(O.HELMHOLTZ, kind, 5.0, qb.coords, qb.normals, qb.coords, qb.normals, qb.weights,
                                   xcol, 0, rows, nthreads=nthreads)
            dt = time.perf_counter() - t0
            if dt > min(args.cpu_seconds, 10.0) / 2 or rows >= nb:
                break
            rows = min(nb, rows * 2)
        line["cpu_baseline"] = {
            "value": rows * nb / dt / 1e9, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{rows} of {nb} rows of the largest surface x 1 right-hand side, D and S row sums "
                      f"(C++ FP64 restatement of the reference's per-RHS matvec), {dt:.1f} s"}
    if not args.no_gmres:
        # scattering solves (I/2 + D - i k S) sigma = -u_inc for all 32 x 64 systems
        g = {"rtol": 1e-10, "restart": 30, "systems": len(quads) * nrhs,
             "timing": "wall time of the whole solve call: right-hand sides and solutions in page-locked host "
                       "buffers, copied in and out inside the call"}
        # page-locked, column-major host buffers for the right-hand sides and the solutions
        Bh = torch.empty((nrhs, B.n), dtype=torch.complex128, pin_memory=True).numpy().T
        Xh = torch.empty((nrhs, B.n), dtype=torch.complex128, pin_memory=True).numpy().T
        Bh[...] = -X
        for mode in ("mixed", "fp64"):
            _, st = B.gmres(Bh, shift=0.5, rtol=1e-10, restart=30, maxiter=300, mode=mode, out=Xh)
            g[mode] = {"seconds": st["seconds"], "iterations": st["iterations"], "outer": st["outer"],
                       "fp64_applies": st["fp64_applies"], "tf32_applies": st["fp32_applies"],
                       "worst_relres_fp64": st["relres"], "converged": bool(st["converged"])}
        if g["fp64"]["converged"] and g["mixed"]["converged"]:
            g["mixed_speedup_vs_fp64"] = g["fp64"]["seconds"] / g["mixed"]["seconds"]
        line["gmres"] = g
    return line


def build_c5(ctx, ntargets: int = 4096, seed: int = 5):
    """Ellipsoid (1, 0.7, 0.5), n = 31 cells per patch, GL 3x3: N = 51,894
    nodes.  The density comes from a GPU solve of the Laplace combined field
    (½I + D + S) sigma = g, g from 8 seeded interior point sources; 4096
    seeded targets lie on the 1.5x scaled ellipsoid; u* = D[sigma + noise]."""
    import inti_b200 as inti

    q = inti.ellipsoid_quadrature(31, 5)
    op = inti.Laplace(dim=3)
    S, D = inti.single_double_layer(op=op, target=q, source=q, correction={"method": "dim"}, ctx=ctx)
    r = np.random.default_rng(seed)
    src = r.uniform(-1, 1, (64, 3))
    src = src[np.sum((src / np.array([0.5, 0.35, 0.25])) ** 2, 1) < 1][:8]
    c = r.standard_normal(len(src))
    b = (c[None, :] / (4 * np.pi * np.linalg.norm(q.coords[:, None, :] - src[None], axis=2))).sum(1)
    sigma, st = inti.gmres(0.5 * inti.I + D + S, b, rtol=1e-10, restart=100, maxiter=500, mode="mixed")
    dirs = r.standard_normal((ntargets, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    tgt = inti.points(1.5 * dirs * np.array([1.0, 0.7, 0.5]))
    P = inti.GpuOperator(inti.DoubleLayerKernel(op), tgt, q, ctx=ctx)
    ustar = P @ (sigma + 0.05 * np.abs(sigma).mean() * r.standard_normal(len(q)))
    cfg = {"workload": "laplace3d_dl_potential_value_and_gradient_ellipsoid_N51894_4096targets", "n": len(q),
           "targets": ntargets, "density_solve": {"converged": bool(st["converged"]), "relres": st["relres"]},
           "gradients": "dJ/dsigma, dJ/dcoords, dJ/dnormals, dJ/dweights for J = 0.5 |D[sigma] - u*|^2"}
    return q, tgt, P, sigma, ustar, cfg


def bench_adjoint(args, ctx, peaks, torch) -> dict:
    """Value and full source gradient of J = ½‖D[σ] − u*‖² (config 5): one
    step = the forward DL potential (u − u* in its epilogue) plus the adjoint
    pass; value = (forward + adjoint) kernel pairs per second."""
    q, tgt, P, sigma, ustar, cfg = build_c5(ctx)
    n, m = len(q), len(tgt)
    pairs = 2.0 * m * n
    dev = torch.device("cuda:0")
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    f64 = dict(dtype=torch.float64, device=dev)
    sig = torch.from_numpy(sigma).to(dev)
    ust = torch.from_numpy(ustar).to(dev)
    u = torch.zeros(m, **f64)
    ds, dw = torch.zeros(n, **f64), torch.zeros(n, **f64)
    dc, dn = torch.zeros(3 * n, **f64), torch.zeros(3 * n, **f64)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)

    def step():
        u.copy_(ust)
        P.apply_device(sig.data_ptr(), u.data_ptr(), 1, 1.0, -1.0)  # u = D sigma - u*
        P.grad_sources_device(u.data_ptr(), sig.data_ptr(), ds.data_ptr(), dc.data_ptr(), dn.data_ptr(),
                              dw.data_ptr())

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        stream.synchronize()
        clocks = Clocks(0)
        launches0 = ctx.launch_count
        ctx.set_profiling(True)
        evs = []
        for _ in range(args.steps):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            evs.append((e0, e1))
        stream.synchronize()
        ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
        adj_ms, adj_n = ctx.profile("adjoint")
        fwd_ms, fwd_n = ctx.profile("pair")
        ctx.set_profiling(False)
        launches = ctx.launch_count - launches0
        clk = clocks.stop()
    # e2e: the user's calls with host arrays
    for _ in range(2):
        g = P @ sigma - ustar
        P.grad_sources(g, sigma)
    e2steps = max(3, args.steps)
    t0 = time.perf_counter()
    for _ in range(e2steps):
        g = P @ sigma - ustar
        grad = P.grad_sources(g, sigma)
        J = 0.5 * float(g @ g)
    e2e_s = (time.perf_counter() - t0) / e2steps
    adj_kern = adj_ms / max(adj_n, 1)
    achieved = m * n * ADJ_FLOPS_PER_PAIR["laplace_dl"] / (adj_kern * 1e-3) / 1e12
    peak = peaks["fp64_flops"] / 1e12
    line = {
        "metric": METRIC, "value": pairs / (ms * 1e-3) / 1e9, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(cfg, l2="flushed between steps", unit_note="forward + adjoint pairs (2 M N per step)"),
        "e2e": {"value": pairs / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": 8 * (2 * n + m),
                "d2h_bytes_per_step": 8 * (m + 8 * n), "ms_per_step": e2e_s * 1e3, "J": J},
        "gpu_launches": launches,
        "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                     "traffic": None, "kernel": "adjoint_sources (laplace_dl, double)", "kernel_ms": adj_kern,
                     "flops_per_pair": ADJ_FLOPS_PER_PAIR["laplace_dl"],
                     "forward_kernel_ms": fwd_ms / max(fwd_n, 1),
                     "peak_source": "FP64 FMA throughput measured in this run (inti_measure_peaks), of measured"},
        "clocks": clk,
    }
    if not args.no_cpu:
        # The reference has no adjoint; its route to these gradients is forward-mode
        # dual numbers (ForwardDiff), one pass over all pairs per input direction.
        sys.path.insert(0, str(ROOT / "oracle"))
        import oracle as O

        nthreads = host_cores()
        t0 = time.perf_counter()
        reps = 0
        dsx = np.random.default_rng(1).standard_normal(q.coords.shape)
        while True:
            O.dl_potential_jvp(tgt.coords, q.coords, q.normals, q.weights, sigma, dsx, None, None, None, nthreads)
            reps += 1
            if time.perf_counter() - t0 > min(args.cpu_seconds, 10.0):
                break
        t_jvp = (time.perf_counter() - t0) / reps
        line["cpu_baseline"] = {
            "value": m * n / t_jvp / 1e9, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{reps} dual-number (value + one directional derivative) passes over all {m} x {n} pairs",
            "full_gradient_forward_mode_s_estimate": t_jvp * 8 * n,
        }
    return line


def bench_csr(args, ctx, torch) -> dict:
    """Correction SpMV bandwidth (the standalone `inti_csr_apply`) on C3's DIM
    pattern replicated 20 times: 20 x 22,326 elements of 9 nodes, 4,018,680
    rows with their own element's 9 columns (nnz = 36.2M), real (δD) and
    complex (δS) values.  At C3's own size the SpMV is ~25 MB and
    latency-bound; this scaled pattern exceeds L2 several times over."""
    import inti_b200 as inti

    nq, m = 9, 20 * 200_934
    r = np.random.default_rng(3)
    indptr = np.arange(0, m * nq + 1, nq, dtype=np.int64)
    indices = ((np.arange(m, dtype=np.int64) // nq * nq)[:, None] + np.arange(nq)).astype(np.int32).ravel()
    dev = torch.device("cuda:0")
    stream = torch.cuda.ExternalStream(ctx.stream, device=dev)
    out = {}
    for dt in ("f64", "c128"):
        cplx = dt == "c128"
        vals = r.standard_normal(m * nq) + (1j * r.standard_normal(m * nq) if cplx else 0)
        Cm = inti.CorrectionMatrix.from_csr(indptr, indices, vals, (m, m), ctx=ctx)
        del vals
        comps = 2 if cplx else 1
        x = torch.randn(comps * m, dtype=torch.float64, device=dev)
        y = torch.zeros(comps * m, dtype=torch.float64, device=dev)
        torch.cuda.synchronize(dev)
        vb = 16 if cplx else 8
        algo = m * nq * (vb + 4) + (m + 1) * 8 + m * vb + m * vb  # beta = 0: y written once
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                Cm.apply_device(x.data_ptr(), y.data_ptr())
            stream.synchronize()
            launches0 = ctx.launch_count
            evs = []
            for _ in range(args.steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                Cm.apply_device(x.data_ptr(), y.data_ptr())
                e1.record(stream)
                evs.append((e0, e1))
            stream.synchronize()
            ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
        out[dt] = {"ms": ms, "gbs": algo / (ms * 1e-3) / 1e9, "algorithmic_bytes": algo,
                   "launches": ctx.launch_count - launches0}
        # parity on sampled rows against the host product of the same arrays
        rows = r.integers(0, m, 64)
        xh = x.cpu().numpy().view(np.complex128) if cplx else x.cpu().numpy()
        ia, ja, va = Cm.arrays()
        yh = y.cpu().numpy().view(np.complex128) if cplx else y.cpu().numpy()
        ref = np.array([va[ia[i]:ia[i + 1]] @ xh[ja[ia[i]:ia[i + 1]]] for i in rows])
        out[dt]["sampled_rows_max_relerr"] = float(np.max(np.abs(yh[rows] - ref) / np.maximum(np.abs(ref), 1e-300)))
        del Cm
    peak, peak_src = hbm_peak()
    return {"metric": "correction SpMV bandwidth", "value": out["f64"]["gbs"], "unit": "GB/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["f64"]["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "dim_pattern_c3x20_rows4018680_nq9", "nnz": m * nq,
                       "l2": "inputs larger than L2 (>= 470 MB per step)"},
            "roofline": {"bound": "hbm", "achieved": out["f64"]["gbs"], "peak": peak, "unit": "GB/s",
                         "frac": out["f64"]["gbs"] / peak, "traffic": CSR_TRAFFIC_BYTES[0],
                         "traffic_source": f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                                           f"{CSR_TRAFFIC_BYTES[1]}",
                         "kernel": "csr_bulk_kernel<real>", "peak_source": peak_src},
            "complex": out["c128"], "real": out["f64"], "gpu_launches": out["f64"]["launches"]}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-gmres", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--shard", default="items", choices=["items", "rows", "replicas"],
                    help="N > 1: split the symmetric work items of one square operator over the ranks (strong "
                         "scaling, partial y all-reduced every step; operators without the symmetric form fall "
                         "back to rows), split its target rows (y all-gathered every step), or run independent "
                         "replicas (weak scaling)")
    ap.add_argument("--workload", default="c2",
                    choices=["c2", "c2_dl", "c2_adl", "c2_hs", "c3_dl_fp64", "c3_dl_fp32c", "c3_sl_fp64", "c1", "c4", "c5", "csr",
                             "dim_c2", "dim_c3"])
    ap.add_argument("--nsurf", type=int, default=32, help="c4: number of star surfaces (32 = the batched workload)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        run_reference(args)
        return

    import torch

    import inti_b200 as inti

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    ctx = inti.Context(local)
    peaks = ctx.measure_peaks()
    if args.workload in ("c4", "c5", "csr", "dim_c2", "dim_c3"):
        if args.workload == "csr":
            line = bench_csr(args, ctx, torch)
        elif args.workload.startswith("dim"):
            line = bench_dim(args, ctx, peaks, torch)
        else:
            line = (bench_batch if args.workload == "c4" else bench_adjoint)(args, ctx, peaks, torch)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    q, S, sigma, fkey, dtype, cfg = build_workload(args.workload, ctx)
    n = len(q)
    pairs = float(n) * n
    stream = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{local}")
    dev = torch.device(f"cuda:{local}")
    comps = 2 if S.is_complex else 1
    xs = torch.from_numpy(np.ascontiguousarray(sigma).view(np.float64).copy()).to(dev)
    shard = args.shard if world > 1 else "none"
    if shard == "items" and not S.tuning["symmetric"]:
        shard = "rows"
    A, m_loc, yfull = S, n, None
    if shard == "items":
        # every rank holds the whole operator and computes its share of the
        # node pairs as a partial y over all rows; one all-reduce sums them
        S.set_shard(rank, world)
        ys = torch.zeros(comps * n, dtype=torch.float64, device=dev)
    elif shard == "rows":
        # rank r computes target rows [r0, r1) of the one operator (all sources
        # on every rank, correction rows sliced); y is all-gathered each step
        from inti_b200 import shard as SH

        r0, r1 = SH.row_blocks(n, world)[rank]
        prow = SH.padded_rows(n, world)
        corr = None
        if S.correction is not None:
            ip, ix, dv = S.correction.arrays()
            corr = inti.CorrectionMatrix.from_csr(*SH.slice_csr_rows(ip, ix, dv, r0, r1), (r1 - r0, n), ctx=ctx)
        A = inti.GpuOperator(S.kernel, SH.target_block(q, r0, r1), q, corr, cfg["precision"], ctx)
        m_loc = r1 - r0
        ys = torch.zeros(comps * prow, dtype=torch.float64, device=dev)
        yfull = torch.zeros(comps * prow * world, dtype=torch.float64, device=dev)
    else:
        ys = torch.zeros(comps * n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)

    def step():
        A.apply_device(xs.data_ptr(), ys.data_ptr())
        if yfull is not None:
            dist.all_gather_into_tensor(yfull, ys)
        if shard == "items":
            dist.all_reduce(ys)

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step()
        stream.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize(dev)
        clocks = Clocks(local)
        launches0 = ctx.launch_count
        # a single-launch step is one kernel: its own events time it, and the
        # per-kernel events (a few microseconds each) would only inflate it
        single = bool(A.tuning.get("single_launch"))
        ctx.set_profiling(not single)
        evs = []
        for _ in range(args.steps):
            flush.zero_()  # untimed: evicts L2 between steps
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            evs.append((e0, e1))
        stream.synchronize()
        torch.cuda.synchronize(dev)
        step_ms = [a.elapsed_time(b) for a, b in evs]
        if single:
            pair_ms, pair_launches, epi_ms, pack_ms = sum(step_ms), args.steps, 0.0, 0.0
        else:
            pair_ms, pair_launches = ctx.profile("pair")
            epi_ms, _ = ctx.profile("epilogue")
            pack_ms, _ = ctx.profile("pack")
        ctx.set_profiling(False)
        launches = ctx.launch_count - launches0
        clk = clocks.stop()
    ms = sum(step_ms) / len(step_ms)
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    job_pairs = pairs if shard in ("rows", "items") else world * pairs  # whole-job pairs per step
    value = job_pairs / (ms * 1e-3) / 1e9

    # e2e through the public API with pinned host buffers (row shards: each
    # rank uploads sigma and reads back its own row block; item shards: each
    # rank uploads sigma, the partial products are all-reduced on the device
    # and every rank reads back y)
    hx = torch.from_numpy(sigma.copy()).pin_memory().numpy()
    hy = torch.zeros(m_loc, dtype=torch.complex128 if S.is_complex else torch.float64).pin_memory().numpy()
    if shard == "items":
        hx_t = torch.from_numpy(np.ascontiguousarray(sigma).view(np.float64).copy()).pin_memory()
        hy_t = torch.zeros(comps * n, dtype=torch.float64).pin_memory()

        def e2e_step():
            with torch.cuda.stream(stream):
                xs.copy_(hx_t, non_blocking=True)
                A.apply_device(xs.data_ptr(), ys.data_ptr())
                dist.all_reduce(ys)
                hy_t.copy_(ys, non_blocking=True)
            stream.synchronize()
    else:
        def e2e_step():
            A.mul(hy, hx)
    for _ in range(2):
        e2e_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = {"value": job_pairs / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": 8 * comps * n * world,
           "d2h_bytes_per_step": 8 * comps * (n if shard == "rows" else n * world), "ms_per_step": e2e_s * 1e3}

    # roofline of the dominant kernel (the pair kernel)
    kern_ms = pair_ms / max(pair_launches, 1)
    fp32 = cfg["precision"] == "fp32c"
    achieved = float(m_loc) * n * FLOPS_PER_PAIR[fkey] / (kern_ms * 1e-3) / 1e12
    peak = peaks["fp32_flops" if fp32 else "fp64_flops"] / 1e12
    shape = A.tuning
    small = bool(shape.get("single_launch"))
    sym = bool(shape.get("symmetric")) and not small
    if sym:  # diagonal node blocks evaluate every ordered pair, the others each unordered pair once
        bt = 128 * shape["targets_per_thread"]
        nb = -(-n // bt)
        evals = float(nb * (nb + 1) // 2) * bt * bt
    else:
        evals = float(m_loc) * n
    roofline = {"bound": "fp32" if fp32 else "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak,
                "traffic": PAIR_TRAFFIC_BYTES[args.workload][0] if args.workload in PAIR_TRAFFIC_BYTES else None,
                "traffic_source": (f"ncu dram__bytes_read.sum + dram__bytes_write.sum of one launch, "
                                   f"{PAIR_TRAFFIC_BYTES[args.workload][1]}"
                                   if args.workload in PAIR_TRAFFIC_BYTES else "no capture"),
                "kernel": f"{'pair_small_kernel' if small else 'pair_symm' if sym else 'pair_forward'} "
                          f"({fkey}, {'float' if fp32 else 'double'})",
                "kernel_ms": kern_ms,
                "flops_per_pair": FLOPS_PER_PAIR[fkey],
                "form": ("symmetric: one kernel evaluation per unordered pair serves both products; achieved "
                         "counts the metric's M*N ordered pairs" if sym else
                         "single launch: one cluster kernel per product builds the source records, sums the pairs, adds the "
                         "correction rows and applies alpha/beta; kernel_ms is the step's own CUDA-event time "
                         "(the step is that one launch)" if small else
                         "one-sided"),
                "kernel_evaluations_per_step": evals,
                "peak_source": f"{'FP32' if fp32 else 'FP64'} FMA throughput measured in this run "
                               "(inti_measure_peaks), of measured",
                "share_of_step": pair_ms / max(sum(step_ms), 1e-9),
                "other_kernels_ms": {"pack": pack_ms / args.steps, "epilogue": epi_ms / args.steps}}

    roofline["launch_shape"] = dict(A.tuning, picked_by="timing at operator creation (inti_op_tuning)")
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak" if args.shard == "replicas" else "strong",
        "vs_baseline": None, "dtype": dtype, "data": "synthetic",
        "config": dict(cfg, parallelism=(f"replicas{world}" if args.shard == "replicas" else
                                         f"{'rows' if shard in ('rows', 'none') else shard}{world}"),
                       l2="flushed between steps",
                       **({"exchange": "NCCL all_gather of y every step (inside the timed region)"}
                          if shard == "rows" else {}),
                       **({"exchange": "NCCL all_reduce of the partial y every step (inside the timed region)"}
                          if shard == "items" else {})),
        "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "clocks": clk,
        "peaks_measured": {k: v / 1e12 for k, v in peaks.items()},
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_sample(q, S, sigma, args.cpu_seconds, host_cores())
    if not args.no_gmres and world == 1 and args.workload == "c1":
        line["gmres"] = gmres_c1(ctx, None, S, q, not args.no_cpu)
    if not args.no_gmres and world == 1 and args.workload == "c2":
        line["gmres"] = gmres_c3(ctx, None if args.no_cpu else min(args.cpu_seconds, 10.0))
        line["gmres_helmholtz"] = gmres_c2_cfie(ctx)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
