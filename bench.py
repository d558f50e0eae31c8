"""Benchmark: QG 1.5-layer RK3-SSP step (WENO5 + beta + DST Helmholtz), FP32, 2048^2.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n 2048]

One "step" = one rk3_ssp_step of the QG PV tendency on a 2048^2 interior
(2050^2 with the ghost ring), periodic q, DST (Dirichlet) psi with
lambda = 1/Ld^2 (Ld = 40 km), beta = 1.7e-11, Lx = Ly = 5.12e6 m, WENO5,
dt at CFL 0.5 for max|u| = 1 m/s.  Metric: Mcell-steps/s = interior cells x
steps / s / 1e6 (whole job, all ranks).  Inputs: seeded k^-3 Gaussian PV
field (std 1e-5 s^-1), synthetic.

* value: device time (CUDA events on the launching stream) of K steps, each
  replayed from a CUDA graph; L2 flushed (256 MiB write) before every step,
  outside the timed events; max over ranks.
* e2e: the same step through the public API (``QGPipeline``, a stream of
  host-resident states): every step uploads its state from pinned host
  memory, steps it and downloads q_{n+1}, all inside the timed region; the
  upload of state k+1 and the download of state k-1 overlap the step of
  state k on separate streams.
* parity: the GPU step from the bench's initial state against the FP64
  oracle's step (relative max-norm error on q_{n+1}; the FP32 bar is 1e-5).
* roofline: the dominant kernel is the tcgen05 DST GEMM (one of the four
  products per solve); achieved = algorithmic 2*M*N*K flops per launch /
  its device time per launch (per_launch_ms), vs the measured bf16 peak.
* cpu_baseline and --impl reference: the FP64 oracle (NumPy/SciPy
  restatement of the reference's path; finitevolX's JAX stack cannot be
  installed offline) on all host threads (oracle/threaded.py, bit-identical
  to the single-threaded oracle), at the same 2048^2 size.
* extra sections (N = 1): the metric's own configuration (256^2, FP64),
  the stencil throughput sweep, the batched split-precision DST with FP64
  refinement, the masked Helmholtz learned-PCG vs MG-PCG comparison and the
  ensemble of uneven members.

Multi-GPU (--gpus N under torchrun): the single-field step does not shard;
each rank runs an independent replica ("replicas only"), value sums ranks.
The ensemble shards by members (each rank its own members, no collective
in the step) and reports the whole-job rate.
"""

from __future__ import annotations

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

LX = 5.12e6
BETA = 1.7e-11
LD = 4.0e4
METRIC = "QG RK3 Mcell-steps/s"
UNIT = "Mcell-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--n", type=int, default=2048)
    ap.add_argument("--method", default="weno5")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-helmholtz", action="store_true")
    ap.add_argument("--helm-pairs", type=int, default=20000)
    ap.add_argument("--helm-reps", type=int, default=20)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-sweep", action="store_true")
    ap.add_argument("--no-dst", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--dst-rhs", type=int, default=64)
    ap.add_argument("--profile", action="store_true",
                    help="only the warm-up and timed QG steps (for ncu launch lists); no extra sections")
    ap.add_argument("--mg-profile", action="store_true",
                    help="only a few V-cycles, U-Net coarse solves and hybrid preconditioner applications on the "
                         "1024^2 masked basin (untrained network; for ncu launch lists of the Helmholtz path)")
    ap.add_argument("--fp64-profile", action="store_true",
                    help="only three eager FP64 QG steps at 256^2 (the metric's own configuration; for ncu launch "
                         "lists)")
    ap.add_argument("--ens-profile", action="store_true",
                    help="only two eager steps of the 64-member ensemble (for ncu launch lists)")
    ap.add_argument("--train-profile", action="store_true",
                    help="only U-Net training steps at batch 64 on 128^2 (seeded synthetic inputs; for ncu launch "
                         "lists and the per-step time)")
    ap.add_argument("--ens-steps", type=int, default=100)
    ap.add_argument("--stage-tile", default=None, help="fix the stage tile (e.g. 64x32) instead of autotuning")
    return ap.parse_args()


def config(n, method):
    """The workload (identical for both arms); how each arm computes it is
    in the line's dtype and notes."""
    return {"workload": f"qg1.5_rk3ssp_{method}_dst_{n}x{n}", "interior": [n, n], "scheme": method,
            "bc": "periodic q, Dirichlet psi", "lambda": 1.0 / LD ** 2, "beta": BETA, "dt": 0.5 * LX / n,
            "l2": "flushed (256 MiB write) before every step", "parallelism": "replicas"}


def initial_q(n, seed=0):
    import numpy as np
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n, n))
    ky = np.fft.fftfreq(n)[:, None]
    kx = np.fft.rfftfreq(n)[None, :]
    k = np.sqrt(kx ** 2 + ky ** 2)
    k[0, 0] = np.inf
    f = np.fft.irfft2(np.fft.rfft2(w) * k ** -1.5, s=(n, n))
    f = (f - f.mean()) * (1e-5 / f.std())
    q = np.zeros((n + 2, n + 2))
    q[1:-1, 1:-1] = f
    q[0, :], q[-1, :] = q[-2, :], q[1, :]
    q[:, 0], q[:, -1] = q[:, -2], q[:, 1]
    return q


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            t0 = time.time()
            while not self.rows and time.time() - t0 < 5.0:  # sampler running before timing starts
                time.sleep(0.01)
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in self.rows for n, v in zip(names, r[5:9]) if v.strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def _oracle_steps(n, method, steps, q=None):
    """`steps` FP64 oracle steps at n^2 on all host threads; (q_after_first, seconds per step list, cores)."""
    from oracle.threaded import host_threads, qg_step_threaded
    q = initial_q(n) if q is None else q
    dx = LX / n
    cores = host_threads()
    first, times = None, []
    for _ in range(steps):
        t = time.perf_counter()
        q = qg_step_threaded(q, dx, dx, BETA, 1.0 / LD ** 2, 0.5 * dx, method, workers=cores)
        times.append(time.perf_counter() - t)
        if first is None:
            first = q
    return first, times, cores


def cpu_baseline(n, method, steps=3):
    """A bounded sample of the same workload on the host: `steps` FP64 oracle
    steps at the full size on all host threads.  Also returns the oracle's
    first step for the parity check."""
    first, times, cores = _oracle_steps(n, method, steps)
    t = sum(times)
    return {"value": n * n * steps / t / 1e6, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{steps} rk3_ssp_steps at {n}x{n} from the bench's initial state, FP64 NumPy/SciPy oracle "
                      f"(restatement of the reference math; finitevolX's JAX stack is not installable offline), "
                      f"{cores} host threads (row bands + SciPy FFT workers), {t:.1f} s"}, first


def run_reference(args, rank):
    """Reference arm: the oracle port of the reference's CPU path at the
    labelled size, all host threads; every warm-up and timed step is a full
    step.  Under torchrun only rank 0 runs."""
    if rank != 0:
        return
    from oracle.threaded import host_threads, qg_step_threaded
    n = args.n
    q = initial_q(n)
    dx = LX / n
    cores = host_threads()
    times = []
    for k in range(args.warmup + args.steps):
        t = time.perf_counter()
        q = qg_step_threaded(q, dx, dx, BETA, 1.0 / LD ** 2, 0.5 * dx, args.method, workers=cores)
        t = time.perf_counter() - t
        if k >= args.warmup:
            times.append(t)
    tot = sum(times)
    val = n * n * len(times) / tot / 1e6
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": val, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config(n, args.method),
        "cpu_baseline": {"value": val, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"per step: 1 rk3_ssp_step at {n}x{n} (FP64 NumPy/SciPy oracle port of the "
                                   f"reference path, oracle/threaded.py: row bands on {cores} threads, SciPy FFT "
                                   f"workers = {cores})"},
        "e2e": {"value": val, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def per_launch_ms(launch, flush, reps: int = 20, rounds: int = 5) -> float:
    """Device time of one launch with L2 flushed before it: `reps` (flush,
    launch) pairs between two events on the launching stream, minus `reps`
    flushes alone, divided by reps (the median of `rounds`).  The flushes keep
    the GPU busy while the host queues the next launch, so no host launch
    gap enters the window."""
    import torch

    est = []
    for _ in range(rounds):
        ts = []
        for with_launch in (True, False):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            flush.fill_(0.0)
            e0.record()
            for k in range(reps):
                flush.fill_(float(k))
                if with_launch:
                    launch()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        est.append((ts[0] - ts[1]) / reps)
    return statistics.median(est)


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def _graph_steps(model, qa, qb, dt, steps, warmup, flush):
    """Device ms of `steps` graph-replayed steps (L2 flushed before each),
    launches per step."""
    import torch
    for _ in range(max(warmup, 3)):
        model.step(qa, dt, out=qb)
        qa.copy_(qb)
    model.step(qa, dt, out=qb)
    torch.cuda.synchronize()
    graphs = []
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for src, dst in ((qb, qa), (qa, qb)):
            g = torch.cuda.CUDAGraph()
            l0 = model.kernel_launches
            with torch.cuda.graph(g, stream=s):
                model.step(src, dt, out=dst, presplit=model.dtype == torch.float32)
            per_step = model.kernel_launches - l0
            graphs.append(g)
    torch.cuda.current_stream().wait_stream(s)
    for g in graphs:
        g.replay()
    torch.cuda.synchronize()
    return graphs, per_step


def _time_graphs(graphs, steps, flush):
    import torch
    total = 0.0
    for k in range(steps):
        flush.fill_(float(k))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        graphs[k % 2].replay()
        e1.record()
        e1.synchronize()
        total += e0.elapsed_time(e1)
    return total


def fp64_metric_section(method, steps, flush, n=256):
    """The metric's own configuration: 256^2 interior, FP64 state, DST by the
    FP64 chain; K graph-replayed steps (L2 flushed before each), parity vs
    the FP64 oracle after one step (bar 1e-12), and the oracle on the host
    at the same size."""
    import numpy as np
    import torch

    import finitevolx_b200 as fvx
    from finitevolx_b200.qg import QGModel
    grid = fvx.ArakawaCGrid2D.from_interior(n, n, LX, LX)
    dt = 0.5 * grid.dx
    model = QGModel(grid, BETA, 1.0 / LD ** 2, method=method, dtype=torch.float64)
    q0 = initial_q(n, seed=7)
    qd = torch.as_tensor(q0, device="cuda")
    got = model.step(qd, dt).cpu().numpy()
    from finitevolx_b200 import autotune
    tile = autotune.tune_qg_stage(model, qd, dt)["tile"]  # the FP64 stage tile, as the FP32 line's
    ref, times, cores = _oracle_steps(n, method, 3, q=q0)
    err = float(np.abs(got - ref).max() / np.abs(ref).max())
    qa, qb = qd.clone(), torch.empty_like(qd)
    graphs, per_step = _graph_steps(model, qa, qb, dt, steps, 3, flush)
    ms = _time_graphs(graphs, steps, flush)
    return {"workload": f"qg1.5_rk3ssp_{method}_dst_{n}x{n}", "dtype": "f64", "steps": steps,
            "ms_per_step": ms / steps, "value": n * n * steps / (ms * 1e-3) / 1e6, "unit": UNIT,
            "launches_per_step": per_step, "dst": "FP64 SIMT transform-matrix chain", "stage_tile": tile,
            "parity": {"rel_err_vs_fp64_oracle": err, "bar": 1e-12},
            "cpu_oracle": {"value": n * n * len(times) / sum(times) / 1e6, "unit": UNIT, "cores": cores}}


def _kminus3_torch(ny, nx, gen, count=1, dtype=None):
    """Seeded k^-3 Gaussian fields on the device (unit std), [count, ny, nx]."""
    import torch
    w = torch.randn((count, ny, nx), generator=gen, device="cuda", dtype=torch.float64)
    ky = torch.fft.fftfreq(ny, device="cuda", dtype=torch.float64)[:, None]
    kx = torch.fft.rfftfreq(nx, device="cuda", dtype=torch.float64)[None, :]
    k = torch.sqrt(kx ** 2 + ky ** 2)
    k[0, 0] = float("inf")
    f = torch.fft.irfft2(torch.fft.rfft2(w) * k ** -1.5, s=(ny, nx))
    f = f - f.mean(dim=(-2, -1), keepdim=True)
    f = f / f.std(dim=(-2, -1), keepdim=True)
    return f if dtype is None else f.to(dtype)


def stencil_sweep_section(flush, sizes=(512, 2048, 4096)):
    """Config 1: single-field stencil throughput, FP32 and FP64, periodic
    ghost ring, seeded k^-3 tracer and divergence-free C-grid (u, v) from a
    random streamfunction.  Per operator: the library's fused kernel and the
    unfused form (the reference's sequence of array passes: face fluxes then
    their divergence; two Laplacian passes then the scale), device time per
    launch with L2 flushed, algorithmic bytes (each array once at full size)
    per second against the measured HBM copy bandwidth."""
    import torch

    from finitevolx_b200 import boundary as B
    from finitevolx_b200._lib import D, I, P, SCHEMES, check, fn, sfx, stream_ptr
    from finitevolx_b200 import operators as O
    from finitevolx_b200.timestepping import lincomb

    hbm = _peaks().get("hbm_gbs")
    out = {"workload": "config 1: 2-D stencils, periodic, seeded k^-3 tracer, u/v from a random streamfunction",
           "bytes_per_cell": {"advection": "h,u,v read + out written (16 B FP32, 32 B FP64)",
                              "jacobian": "f,g read + J written (12 / 24 B)",
                              "biharmonic": "h read + out written (8 / 16 B)"},
           "peak_gbs": hbm, "peak_source": "measured HBM copy (MEASURED_PEAKS.json)", "rows": []}
    gen = torch.Generator(device="cuda").manual_seed(5)
    for n in sizes:
        for dt in (torch.float32, torch.float64):
            es = 4 if dt == torch.float32 else 8
            N = n + 2
            dx = LX / n
            h = torch.zeros((N, N), dtype=dt, device="cuda")
            h[1:-1, 1:-1] = _kminus3_torch(n, n, gen, dtype=dt)[0]
            h = B.enforce_periodic(h)
            psi = torch.zeros_like(h)
            psi[1:-1, 1:-1] = _kminus3_torch(n, n, gen, dtype=dt)[0] * (dx / 10.0)
            px = O.cgrid_op("T_to_X", psi)
            u = lincomb(-1.0, O.cgrid_op("diff_y_X_to_U", px, dx=dx, dy=dx))
            v = O.cgrid_op("diff_x_X_to_V", px, dx=dx, dy=dx)
            o = torch.empty_like(h)
            fe, fnn, lap = torch.empty_like(h), torch.empty_like(h), torch.empty_like(h)
            jo = torch.empty((N - 2, N - 2), dtype=dt, device="cuda")
            s = sfx(h)
            st = stream_ptr()
            adv = fn(f"fvx_advect2d_{s}")
            ff = fn(f"fvx_face_flux2d_{s}")
            fd = fn(f"fvx_flux_divergence2d_{s}")
            cg = fn(f"fvx_cgrid_op2d_{s}")
            cells = N * N
            for op in ("weno5", "weno7", "van_leer", "jacobian", "biharmonic"):
                if op in ("weno5", "weno7", "van_leer"):
                    m = I(SCHEMES[op])
                    fused = lambda m=m: check(adv(P(h), P(u), P(v), P(o), I(N), I(N), D(dx), D(dx), m, None, None,  # noqa: E731
                                                  st), "advect")

                    def unfused(m=m):
                        check(ff(P(h), P(u), P(v), P(fe), P(fnn), I(N), I(N), m, None, st), "face flux")
                        check(fd(P(fe), P(fnn), P(o), I(N), I(N), D(dx), D(dx), None, st), "divergence")
                    nbytes = 4 * es * cells
                    form = "face fluxes (fe, fn to HBM) + flux divergence"
                elif op == "jacobian":
                    jac = fn(f"fvx_arakawa_jacobian_{s}")
                    fused = lambda: check(jac(P(h), P(psi), P(jo), I(1), I(N), I(N), D(dx), D(dx), st), "J")  # noqa: E731
                    unfused = None
                    nbytes = 3 * es * cells
                    form = None
                else:
                    bh = fn(f"fvx_biharmonic2d_{s}")
                    fused = lambda: check(bh(P(h), D(1e9), P(o), I(N), I(N), D(dx), D(dx), None, st), "biharm")  # noqa: E731

                    def unfused():
                        check(cg(I(8), P(h), None, P(lap), None, I(N), I(N), D(dx), D(dx), None, None, st), "lap")
                        check(cg(I(8), P(lap), None, P(o), None, I(N), I(N), D(dx), D(dx), None, None, st), "lap")
                        o.mul_(-1e9)
                    nbytes = 2 * es * cells
                    form = "laplacian -> HBM, laplacian, scale"
                for _ in range(3):
                    fused()
                    if unfused:
                        unfused()
                t_f = per_launch_ms(fused, flush, reps=10, rounds=3)
                row = {"n": n, "dtype": "f32" if es == 4 else "f64", "op": op, "fused_ms": t_f,
                       "gbs": nbytes / (t_f * 1e-3) / 1e9}
                row["frac"] = row["gbs"] / hbm if hbm else None
                if unfused:
                    t_u = per_launch_ms(unfused, flush, reps=10, rounds=3)
                    row.update(unfused_ms=t_u, fused_speedup=t_u / t_f, unfused_form=form)
                out["rows"].append(row)
            del h, psi, px, u, v, o, fe, fnn, lap, jo
            torch.cuda.empty_cache()
    return out


def dst_batch_section(n_rhs, sizes=(1024, 2048)):
    """Config 3: Dirichlet box (Lx = 5.12e6 m), lambda in {0, 1/(4e4)^2,
    1/(1e4)^2}, n_rhs seeded k^-3 right-hand sides per size.  FP32: the
    3xBF16 tensor-core chain; FP64: the same chain plus FP64 iterative
    refinement on the 5-point residual to a 1e-12 normwise backward error.
    Times per right-hand side (CUDA events, whole batch), the refinement's
    passes and backward error, and every result's max-norm error against
    the FP64 DST oracle (SciPy, all host threads)."""
    import numpy as np
    import scipy.fft
    import torch

    from finitevolx_b200.solvers import DSTHelmholtzPlan
    from oracle.threaded import host_threads

    peak = _peaks().get("bf16_tflops") or 1590.0
    cores = host_threads()
    out = {"workload": f"config 3: DST Helmholtz, Dirichlet box, {n_rhs} seeded k^-3 RHS per size", "cases": []}
    gen = torch.Generator(device="cuda").manual_seed(11)
    for n in sizes:
        dx = LX / n
        f64 = _kminus3_torch(n, n, gen, count=n_rhs) * 1e-5
        f32 = f64.float()
        fh = f64.cpu().numpy()
        with scipy.fft.set_workers(cores):
            fhat = scipy.fft.dstn(fh, type=1, axes=(-2, -1))
        k = np.arange(n)
        ev = -4.0 / dx ** 2 * np.sin(np.pi * (k + 1) / (2 * (n + 1))) ** 2
        for lam in (0.0, 1.0 / 4e4 ** 2, 1.0 / 1e4 ** 2):
            plan = DSTHelmholtzPlan(n, n, dx, dx, (lam,), batch_max=n_rhs)
            with scipy.fft.set_workers(cores):
                ref = scipy.fft.idstn(fhat / (ev[:, None] + ev[None, :] - lam), type=1, axes=(-2, -1))
            refmax = np.abs(ref).reshape(n_rhs, -1).max(axis=1)
            o32 = torch.empty_like(f32)
            o64 = torch.empty_like(f64)
            plan.solve(f32, out=o32)
            plan.solve_refined(f64, tol=1e-12, out=o64)
            torch.cuda.synchronize()
            res = {}
            for name, call in (("fp32_split", lambda: plan.solve(f32, out=o32)),
                               ("fp64_refined", lambda: plan.solve_refined(f64, tol=1e-12, out=o64)[1])):
                ts, info = [], None
                for _ in range(3):
                    torch.cuda.synchronize()
                    e0 = torch.cuda.Event(enable_timing=True)
                    e1 = torch.cuda.Event(enable_timing=True)
                    e0.record()
                    info = call()
                    e1.record()
                    e1.synchronize()
                    ts.append(e0.elapsed_time(e1))
                ms = statistics.median(ts)
                res[name] = {"ms_batch": ms, "us_per_rhs": 1e3 * ms / n_rhs}
                if isinstance(info, dict):
                    res[name].update(passes=info["passes"], backward_error=info["backward_error"],
                                     converged=info["converged"])
            plan.check_device()
            for name, o in (("fp32_split", o32), ("fp64_refined", o64)):
                got = o.double().cpu().numpy()
                e = np.abs(got - ref).reshape(n_rhs, -1).max(axis=1) / refmax
                res[name].update(err_max=float(e.max()), err_median=float(np.median(e)),
                                 errors=[float(f"{x:.3g}") for x in e])
            flops = 4 * 2.0 * n ** 3 * n_rhs  # 4 dense products of 2 N^3 per RHS
            res["fp32_split"]["tflops_algorithmic"] = flops / (res["fp32_split"]["ms_batch"] * 1e-3) / 1e12
            res["fp32_split"]["frac_of_bf16_peak"] = res["fp32_split"]["tflops_algorithmic"] / peak
            out["cases"].append({"n": n, "lambda": lam, **res})
            del plan, o32, o64, ref
            torch.cuda.empty_cache()
        del f64, f32, fh, fhat
    out["error"] = "max|psi - psi_oracle| / max|psi_oracle| per right-hand side; oracle = SciPy FP64 DST-I"
    return out


def masked_basin(n, seed=0):
    """Masked-Helmholtz workload: Gaussian-filtered (sigma = 20 cells) seeded
    field thresholded at 30% land, largest connected ocean kept, closed
    boundary ring; c = exp(0.5 g) with g a second smooth field (unit std);
    white-noise right-hand side on the ocean."""
    import numpy as np
    from scipy import ndimage
    rng = np.random.default_rng(seed)
    g = ndimage.gaussian_filter(rng.standard_normal((n, n)), sigma=20, mode="wrap")
    m = g > np.quantile(g, 0.3)
    lab, k = ndimage.label(m)
    if k > 1:
        sizes = ndimage.sum(m, lab, range(1, k + 1))
        m = lab == (1 + int(np.argmax(sizes)))
    m[0, :] = m[-1, :] = m[:, 0] = m[:, -1] = False
    g2 = ndimage.gaussian_filter(rng.standard_normal((n, n)), sigma=20, mode="wrap")
    c = np.exp(0.5 * g2 / g2.std())
    f = rng.standard_normal((n, n)) * m
    return m.astype(np.float64), c, f


def helmholtz_case(n, ld, pairs, reps):
    """Masked variable-coefficient Helmholtz, time to 1e-8 relative residual
    (FP64-checked): MG-PCG (one V-cycle per iteration, the reference's
    6/6/50 sweeps) against flexible PCG with the learned coarse solver
    (U-Net at the first level at or below 128^2, the same fine sweeps,
    energy-scaled correction; MG-PCG as its fallback when a calibration
    solve on another right-hand side finds MG-PCG faster) and the same
    cycle without the network.  Each solve is timed with CUDA events around
    the whole call (set-up, iterations, final FP64 check); median, min, max
    over ``reps``; the network is trained and calibrated once beforehand
    (not timed)."""
    import torch

    import finitevolx_b200 as fvx
    from finitevolx_b200.learned import LearnedPreconditioner, generate_pairs

    m, c, f = masked_basin(n, 1)
    dx = LX / n
    mg = fvx.build_multigrid_solver(m, dx, dx, lambda_=1.0 / ld ** 2, coeff=c, dtype=torch.float32)
    pcg = fvx.MaskedHelmholtzPCG(mg)
    b = torch.from_numpy(f).float().cuda()

    def timed(kw):
        pcg.solve(b, rtol=1e-8, **kw)
        ts, info = [], None
        for _ in range(reps):
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            x, info = pcg.solve(b, rtol=1e-8, **kw)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return {"ms": statistics.median(ts), "ms_min": min(ts), "ms_max": max(ts), "reps": reps,
                "iterations": info["iterations"], "rel_residual_fp64": info["rel_residual"],
                "converged": info["converged"]}

    out = {"workload": f"masked Helmholtz {n}^2, Ld {ld / 1e3:.0f} km, variable c, FP32 work vectors, "
                       "FP64 iterate/dots/residual, rtol 1e-8", "levels": mg.n_levels}
    out["mg_pcg"] = timed(dict(precond="mg", graph=True))
    t0 = time.time()
    pc = LearnedPreconditioner(mg, n_pre=6, n_post=6, batch_max=64, seed=0)
    F, E = generate_pairs(mg, pc.lvl, pairs, pc.n_pre, seed=1)
    torch.cuda.synchronize()
    t_gen = time.time() - t0
    t0 = time.time()
    hist = pc.train(F, E, epochs=6, batch=64, lr=2e-3, seed=1)
    torch.cuda.synchronize()
    out["training"] = {"pairs": pairs, "epochs": 6, "batch": 64, "gen_s": t_gen, "train_s": time.time() - t0,
                       "loss_first_epoch": hist[0], "loss_last_epoch": hist[-1], "level": pc.lvl}
    del F, E
    # calibration on another right-hand side of the same operator (not the
    # timed one): the learned preconditioner keeps MG-PCG as its fallback
    # when MG-PCG is the faster method there
    rng = torch.Generator(device="cuda").manual_seed(7)
    b_cal = torch.randn(b.shape, generator=rng, device="cuda") * torch.from_numpy(m).float().cuda()
    out["calibration"] = pc.calibrate(pcg, b_cal, rtol=1e-8)
    out["learned_pcg"] = timed(dict(precond=pc, flexible=True, graph=True, max_iter=500))
    out["learned_pcg"]["method"] = "MG-PCG (fallback)" if pc.use_fallback else "flexible PCG, learned coarse solve"
    fb = pc.use_fallback
    pc.use_fallback = False
    out["network_without_fallback"] = timed(dict(precond=pc, flexible=True, graph=True, max_iter=500))
    pc.use_fallback = fb
    pc0 = LearnedPreconditioner(mg, n_pre=6, n_post=6, batch_max=1, coarse=False, scale=False)
    out["same_cycle_without_network"] = timed(dict(precond=pc0, flexible=True, graph=True, max_iter=500))
    out["speedup_learned_vs_mg"] = out["mg_pcg"]["ms"] / out["learned_pcg"]["ms"]
    return out


def helmholtz_section(pairs, reps):
    return {"cases": [helmholtz_case(n, ld, pairs, reps) for n, ld in ((1024, LD), (512, LD), (1024, 4.0e5))]}


def ensemble_members(count=64, seed=0):
    """Config-2 ensemble: sizes drawn (seeded) from {128, 256, 512, 1024}^2,
    1-3 layers (H = 400/1100/2600 m)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    sizes = rng.choice([128, 256, 512, 1024], size=count)
    nls = rng.integers(1, 4, size=count)
    return list(zip(sizes.tolist(), nls.tolist()))


def ensemble_section(members, n_steps):
    """All members advanced n_steps RK3-SSP steps by one CUDA graph per rank
    (per RK stage: one batched DST chain per grid size, one persistent
    work-queue launch of the fused stage over every tile of every layer).
    With N ranks each rank runs the members ``shard_members`` gives it.
    Metric: interior layer-cells x steps / s over all ranks."""
    import torch

    import finitevolx_b200 as fvx
    from finitevolx_b200 import autotune
    from finitevolx_b200.replicas import sharded_ensemble_run

    tuned = {}

    def factory(sub, idx):
        ens = fvx.QGEnsemble(sub)
        for m, ((n, nl), gi) in enumerate(zip(sub, idx)):
            g = torch.Generator(device="cuda").manual_seed(1000 + gi)
            for k in range(nl):
                q = torch.zeros((n + 2, n + 2), device="cuda")
                q[1:-1, 1:-1] = torch.randn((n, n), device="cuda", generator=g) * 1e-5
                ens.set_layer(m, k, q)
        tuned.update(autotune.tune_ensemble(ens))
        return ens

    r = sharded_ensemble_run(members, n_steps, factory)
    ms = r["t_max_ms"]
    return {"workload": f"{len(members)} multi-layer QG members, sizes {{128,256,512,1024}}^2, 1-3 layers, "
                        f"WENO5, FP32, {n_steps} RK3 steps in one CUDA graph per rank",
            "members": len(members), "layer_cells_per_step": r["cells_per_step"], "steps": n_steps, "ms": ms,
            "ms_per_step": ms / n_steps, "value": r["value"], "unit": "Mcell-steps/s",
            "ranks": r["world"], "members_per_rank": r["members_per_rank"],
            "launches_per_step": r["launches_per_step"], "autotuned_blocks_per_sm": tuned.get("blocks_per_sm")}


def fp64_profile_run(method, n=256, steps=3):
    """The FP64 step's kernels (the metric's own configuration) in a short
    run for ncu launch lists: one warm-up step and ``steps`` eager steps."""
    import torch

    import finitevolx_b200 as fvx
    from finitevolx_b200.qg import QGModel
    grid = fvx.ArakawaCGrid2D.from_interior(n, n, LX, LX)
    dt = 0.5 * grid.dx
    model = QGModel(grid, BETA, 1.0 / LD ** 2, method=method, dtype=torch.float64)
    qa = torch.as_tensor(initial_q(n, seed=7), device="cuda")
    qb = torch.empty_like(qa)
    model.step(qa, dt, out=qb)
    torch.cuda.synchronize()
    for _ in range(steps):
        model.step(qb, dt, out=qa)
        qa, qb = qb, qa
    torch.cuda.synchronize()
    print(json.dumps({"fp64_profile_run": True, "n": n, "steps": steps}))


def ens_profile_run(steps=2):
    """The ensemble's kernels in a short run for ncu launch lists: the bench's
    64 members (seeded states), ``steps`` eager RK3 steps after one warm-up
    step, default persistent-grid occupancy."""
    import torch

    import finitevolx_b200 as fvx

    members = ensemble_members()
    ens = fvx.QGEnsemble(members)
    for m, (n, nl) in enumerate(members):
        g = torch.Generator(device="cuda").manual_seed(1000 + m)
        for k in range(nl):
            q = torch.zeros((n + 2, n + 2), device="cuda")
            q[1:-1, 1:-1] = torch.randn((n, n), device="cuda", generator=g) * 1e-5
            ens.set_layer(m, k, q)
    ens.step(1)
    torch.cuda.synchronize()
    ens.step(steps)
    torch.cuda.synchronize()
    print(json.dumps({"ens_profile_run": True, "members": len(members), "steps": steps,
                      "launches_per_step": ens.launches_per_step}))


def train_profile_run(steps=20, batch=64, n=128):
    """U-Net training steps (forward, backward, Adam) at the bench's training
    batch on a 128^2 level, seeded synthetic inputs and targets (channel 1 a
    0/1 mask): three warm-up steps, then ``steps`` steps timed with CUDA
    events on the current stream; prints the milliseconds per step."""
    import torch

    from finitevolx_b200.learned import UNet
    net = UNet(n, n, batch_max=batch, seed=0)
    g = torch.Generator(device="cuda").manual_seed(0)
    x = torch.randn((batch, 3, n, n), generator=g, device="cuda")
    x[:, 1] = (torch.rand((batch, n, n), generator=g, device="cuda") > 0.3).float()
    t = torch.randn((batch, 1, n, n), generator=g, device="cuda")
    loss = torch.zeros(1, dtype=torch.float64, device="cuda")
    for _ in range(3):
        net.train_step(x, t, lr=1e-3, loss_out=loss)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        net.train_step(x, t, lr=1e-3, loss_out=loss)
    e1.record()
    torch.cuda.synchronize()
    print(json.dumps({"train_profile_run": True, "batch": batch, "n": n, "steps": steps,
                      "ms_per_step": e0.elapsed_time(e1) / steps}))


def mg_profile_run(n=1024, reps=3):
    """The Helmholtz path's kernels in a short run for ncu launch lists:
    ``reps`` MG V-cycles, U-Net coarse solves (per-layer chain) and hybrid
    preconditioner applications on the masked basin, Ld 40 km (the network
    untrained: its launches are what is profiled, not its answer)."""
    import torch

    import finitevolx_b200 as fvx
    from finitevolx_b200.learned import LearnedPreconditioner

    m, c, f = masked_basin(n, 1)
    dx = LX / n
    mg = fvx.build_multigrid_solver(m, dx, dx, lambda_=1.0 / LD ** 2, coeff=c, dtype=torch.float32)
    b = torch.from_numpy(f).float().cuda()
    pc = LearnedPreconditioner(mg, n_pre=6, n_post=6, batch_max=1, seed=0)
    pc.activate()
    fl = torch.randn(pc.m_lvl.shape, device="cuda")
    for _ in range(reps):
        mg.v_cycle(None, b)
        pc.coarse_solve(fl)
        pc(b)
    torch.cuda.synchronize()
    print(json.dumps({"mg_profile_run": True, "n": n, "reps": reps, "levels": mg.n_levels, "unet_level": pc.lvl}))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.mg_profile:
        mg_profile_run(reps=3)
        return
    if args.ens_profile:
        ens_profile_run(steps=2)
        return
    if args.fp64_profile:
        fp64_profile_run(args.method)
        return
    if args.train_profile:
        train_profile_run(steps=args.steps)
        return
    import numpy as np
    import torch
    import torch.distributed as dist

    import finitevolx_b200 as fvx
    from finitevolx_b200 import _lib as L
    from finitevolx_b200.qg import QGModel
    from finitevolx_b200.replicas import max_over_ranks, whole_job_rate

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120))
    n = args.n
    grid = fvx.ArakawaCGrid2D.from_interior(n, n, LX, LX)
    dt = 0.5 * grid.dx / 1.0
    model = QGModel(grid, BETA, 1.0 / LD ** 2, method=args.method, dtype=torch.float32)
    q0_host = initial_q(n, seed=rank)
    q0 = torch.as_tensor(q0_host, dtype=torch.float32, device="cuda")
    qa, qb = q0.clone(), torch.empty_like(q0)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    # the GPU step from the bench's initial state, for the parity check
    q1_gpu = model.step(q0, dt).double().cpu().numpy()

    # autotuned launch choices (stage tile shape; fused or separate DST split)
    from finitevolx_b200 import autotune
    tuned = {}
    if args.stage_tile:
        autotune.set_stage_tile(args.method, torch.float32, autotune._TILES.index(args.stage_tile))
        tuned["stage_tile"] = args.stage_tile
    if not args.profile:
        tuned = {"stage_tile": tuned.get("stage_tile") or autotune.tune_qg_stage(model, qa, dt)["tile"],
                 "fused_split": autotune.tune_qg_split(model, qa, dt)["fused"],
                 "dst_kernel": autotune.tune_dst_kernel(model, qa, dt)["kernel"]}
    qa.copy_(q0)

    graphs, per_step_launches = _graph_steps(model, qa, qb, dt, args.steps, args.warmup, flush)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        total_ms = _time_graphs(graphs, args.steps, flush)
    torch.cuda.synchronize()
    t_max = max_over_ranks(total_ms, device="cuda")
    if world > 1:
        dist.barrier()
    cells = n * n
    value = whole_job_rate(cells, args.steps, t_max, world)
    if args.profile:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": UNIT, "steps": args.steps,
                              "ms_per_step": t_max / args.steps, "profile_run": True}))
        if world > 1:
            dist.barrier()
            del graphs
            dist.destroy_process_group()
        return

    # e2e through the public API (QGPipeline): every step uploads its input
    # state from pinned host memory and downloads its result; the pipeline
    # overlaps the upload of state k+1 and the download of state k-1 with
    # the step of state k.  L2 flushed before every step on the step stream.
    from finitevolx_b200.qg import QGPipeline
    pipe = QGPipeline(model, dt)
    n_host = 4
    host_in = torch.empty((n_host,) + tuple(q0.shape), dtype=torch.float32, pin_memory=True)
    for h in range(n_host):
        host_in[h].copy_(q0.cpu())
    host_out = torch.empty_like(host_in, pin_memory=True)
    flush_fn = lambda: flush.fill_(1.0)  # noqa: E731
    pipe.run(host_in, host_out, n=max(args.warmup, 3), between_steps=flush_fn)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    pipe.run(host_in, host_out, n=args.steps, between_steps=flush_fn)
    e1.record()
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    # the pipeline's output is the step of q0: the same q_{n+1} as above
    e2e_diff = float(np.abs(host_out[(args.steps - 1) % n_host].double().numpy() - q1_gpu).max()
                     / np.abs(q1_gpu).max())
    if not e2e_diff <= 1e-6:
        raise RuntimeError(f"e2e pipeline result differs from QGModel.step ({e2e_diff:.3e})")
    e2e_ms = max_over_ranks(e2e_ms, device="cuda")
    e2e = whole_job_rate(cells, args.steps, e2e_ms, world)
    nbytes = host_in[0].numel() * host_in.element_size()

    # fused vs unfused: the same step as the reference's operator sequence,
    # one kernel (or torch copy) per operator, through the same library
    for _ in range(3):
        model.step_unfused(qa, dt)
    torch.cuda.synchronize()
    unf_ms = 0.0
    n_unf = max(5, min(20, args.steps))
    for k in range(n_unf):
        flush.fill_(float(k))
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        model.step_unfused(qa, dt)
        e1.record()
        e1.synchronize()
        unf_ms += e0.elapsed_time(e1)
    unf_ms /= n_unf

    # the fused stage kernel alone (HBM roofline): stage 2's form (reads
    # q_stage, q_n, psi; writes q_next and the split DST operand)
    stage_ms = per_launch_ms(lambda: model._stage(qa, qb, qb, 0.75, 0.25, 0.25 * dt, True, False), flush)
    # algorithmic bytes: q_stage, q_n, psi read, q_next written (FP32, one
    # pass each) = 16 B/cell, plus the DST operand written as bf16 hi/lo
    # (4 B/cell)
    stage_bytes = 20.0 * n * n
    peaks = _peaks()
    hbm_peak = peaks.get("hbm_gbs")

    # dominant kernel: one tcgen05 DST GEMM (2048 x 2048 x 2048, 3xBF16)
    from finitevolx_b200._lib import I, fn, stream_ptr
    h = model.plan.handle
    sym = fn("fvx_dst_operand_layout")(h) == 1
    gemm = fn("fvx_dst_gemm_step")
    for _ in range(5):
        gemm(h, I(0), I(1), stream_ptr())
    gemm_ms = per_launch_ms(lambda: L.check(gemm(h, I(0), I(1), stream_ptr()), "gemm"), flush)
    flops = 2.0 * n * n * n
    peak = peaks.get("bf16_tflops")
    peak_src = "measured burst bf16 (MEASURED_PEAKS.json)" if peak else "fallback 1590"
    peak = peak or 1590.0
    achieved = flops / (gemm_ms * 1e-3) / 1e12
    # DRAM traffic of this kernel per launch, from the ncu capture of the
    # 2048^2 step committed under profiles/ (dram__bytes_read.sum +
    # dram__bytes_write.sum of the first product of a solve)
    traffic = None
    try:
        with open(os.path.join(ROOT, "profiles", "dst_product_traffic.json")) as f:
            tr = json.load(f)
        if tr.get("n") == n and tr.get("kernel") == ("gemm_sym_bf16_kernel" if sym else "gemm_split_bf16_kernel"):
            traffic = tr.get("dram_bytes_per_launch")
    except Exception:
        pass

    res = {}
    if rank == 0:
        res = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(config(n, args.method), autotuned=tuned,
                           helmholtz="DST-I as tensor-core transform-matrix products, 3xBF16 split, FP32 accumulate"),
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
                    "ms_per_step": e2e_ms / args.steps,
                    "form": "QGPipeline: upload of state k+1, step k (CUDA graph), download of k-1 on three "
                            "streams; L2 flushed before every step"},
            "gpu_launches": per_step_launches * args.steps,
            "roofline": {"bound": "tensor",
                         "kernel": ("gemm_sym_bf16_kernel (even/odd DST-I product, 3xBF16)" if sym
                                    else "gemm_split_bf16_kernel (DST product, 3xBF16)"),
                         "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                         "peak_source": peak_src,
                         "traffic": traffic, "traffic_unit": "bytes",
                         "traffic_source": "profiles/dst_product_traffic.json (ncu capture of this kernel)"
                                           if traffic else None,
                         "per_launch_ms": gemm_ms, "algorithmic_flops_per_launch": flops,
                         "executed_tensor_flops_per_launch": (3.0 if sym else 6.0) * n ** 3,
                         "executed_frac": (3.0 if sym else 6.0) * n ** 3 / (gemm_ms * 1e-3) / 1e12 / peak},
            "stage_kernel": {"bound": "hbm", "kernel": f"qg stage_kernel<float, {args.method.upper()}>",
                             "per_launch_ms": stage_ms, "algorithmic_bytes_per_launch": stage_bytes,
                             "achieved": stage_bytes / (stage_ms * 1e-3) / 1e9, "unit": "GB/s",
                             "peak": hbm_peak,
                             "frac": (stage_bytes / (stage_ms * 1e-3) / 1e9 / hbm_peak) if hbm_peak else None},
            "fused_vs_unfused": {"fused_ms_per_step": t_max / args.steps, "unfused_ms_per_step": unf_ms,
                                 "speedup": unf_ms / (t_max / args.steps),
                                 "unfused": "the reference operator sequence, one library kernel or torch copy per "
                                            "operator (QGModel.step_unfused)"},
            "clocks": clk.summary(),
        }
        if world == 1 and not args.no_cpu_baseline:
            cb, q1_ref = cpu_baseline(n, args.method)
            res["cpu_baseline"] = cb
            if rank == 0 and np.array_equal(q0_host, initial_q(n)):
                err = float(np.abs(q1_gpu - q1_ref).max() / np.abs(q1_ref).max())
                res["parity"] = {"rel_err_vs_fp64_oracle": err, "bar": 1e-5, "passed": err < 1e-5,
                                 "what": "max|q1_gpu - q1_oracle| / max|q1_oracle| after one step from the bench's "
                                         "initial state (FP64 oracle)"}
        if world == 1 and not args.no_fp64:
            res["fp64_metric_config"] = fp64_metric_section(args.method, args.steps, flush)
        if world == 1 and not args.no_sweep:
            res["stencil_sweep"] = stencil_sweep_section(flush)
        if world == 1 and not args.no_dst:
            res["dst_batched"] = dst_batch_section(args.dst_rhs)
        if world == 1 and not args.no_helmholtz:
            # each section is its own workload: the earlier sections' cached
            # device memory (batched DST, 4096^2 sweep fields) is released
            # first (the learned path measured ~1-2 % slower on top of it)
            torch.cuda.empty_cache()
            res["helmholtz"] = helmholtz_section(args.helm_pairs, args.helm_reps)
    if not args.no_ensemble:
        torch.cuda.empty_cache()
        ens = ensemble_section(ensemble_members(), args.ens_steps)  # every rank: its own members
        if rank == 0:
            res["ensemble"] = ens
    if rank == 0:
        print(json.dumps(res))
    if world > 1:
        dist.barrier()
        del graphs
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
