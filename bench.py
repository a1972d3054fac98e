"""Benchmark: T_eff of the 3D Maxwell visco-elastic PT iteration at 511^3 (FP64) on B200.

A step is one check block of the reference's PT loop: `nout` PT iterations
(compute_Pt_τ! + compute_V! + the free-slip copies) followed by one convergence check
(compute_Res! + norms), for the Stokes3D_ve_perf.jl problem (spherical inclusion,
pure shear) at nx = ny = nz = 511. T_eff = A_eff / t_it with the reference's
A_eff = 29 * nx*ny*nz * 8 bytes per PT iteration (Stokes3D_ve_perf.jl:229).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs an independent replica (the path is single-GPU; there is
no data-path collective): value = sum over ranks of the work / max-over-ranks time.
"""
import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "pseudotransientstokes.jl_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

METRIC = "T_eff GB/s & time-to-tol 1e-8, 3D VE 511³: FP32+FP64 refine vs plain FP64, 1 B200"
A_EFF_ARRAYS = 29  # Stokes3D_ve_perf.jl:229: (10*2 + 6*1 + 3) arrays per PT iteration


def a_eff(n, itemsize=8):
    return A_EFF_ARRAYS * n * n * n * itemsize


def hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        med = sm[len(sm) // 2] if sm else None
        return {"sm_mhz": med, "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch
        import torch.distributed as dist

        # one process per GPU over NCCL; on a host without GPUs (the reference arm, tests) gloo
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(x, pg):
    if pg is None:
        return x
    import torch

    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


# ------------------------------------------------------------------------------ CPU arm
def cpu_sample(n, iters):
    """The oracle's OpenMP FP64 restatement of Stokes3D_ve_perf.jl on the host cores."""
    from oracle import scripts as S
    from oracle.binding import lib

    nthreads = lib().ora_num_threads()
    c = S.make("3d_ve_perf", n, n, n)
    c.assign_tau()
    c.iteration()  # warm the pages
    t0 = time.perf_counter()
    for _ in range(iters):
        c.iteration()
    dt = time.perf_counter() - t0
    return a_eff(n) * iters / dt / 1e9, nthreads, dt


def cpu_sample_2d(n, iters):
    """The oracle's OpenMP FP64 restatement of Stokes2D_ve_perf.jl on the host cores:
    T_eff with the script's A_eff = 18*nx*ny*8 bytes per PT iteration."""
    from oracle import scripts as S
    from oracle.binding import lib

    c = S.make("2d_ve_perf", n, n)
    c.assign_tau()
    c.iteration()
    t0 = time.perf_counter()
    for _ in range(iters):
        c.iteration()
    dt = time.perf_counter() - t0
    return 18 * n * n * 8 * iters / dt / 1e9, lib().ora_num_threads(), dt


def small_2d_case():
    """The reference's CPU-runnable case: 2D viscous Stokes (Stokes2D.jl), 127^2, a check every
    100 iterations, to 1e-8 -- on the host (the oracle, all threads) and on the GPU."""
    import torch

    import ptstokes
    from oracle import scripts as S
    from oracle.binding import lib

    o = S.make("2d_v", 127, 127, nout=100)
    t0 = time.perf_counter()
    o.run()
    cpu_s = time.perf_counter() - t0
    g = ptstokes.Solver("2d_v", 127, 127, nout=100)
    g.setup_inclusion()
    g.sync()
    st = torch.cuda.ExternalStream(g.stream_handle())
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(st)
    r = g.run()
    b.record(st)
    b.synchronize()
    out = {"workload": "2D viscous Stokes2D.jl 127^2, check every 100 iterations, tol 1e-8",
           "cpu_oracle": {"seconds": round(cpu_s, 4), "iters": o.iters, "threads": lib().ora_num_threads()},
           "gpu": {"seconds": round(a.elapsed_time(b) / 1e3, 4), "iters": r["iters"]}}
    g.close()
    return out


DATA_3D = "synthetic (the reference's own inclusion problem: spherical inclusion r=1 mu=1e-3, pure shear, G=1, dt=1)"


def workload_config(n, precision):
    """The `config` of the default line: the workload alone, the same for both arms (the
    reference arm times bounded samples of it; its cpu_baseline.sample says how many PT
    iterations a step holds)."""
    px = (n + 1 + 15) // 16 * 16  # the padded x-extent of every field (128-byte rows)
    field_gb = px * (n + 1) * (n + 1) * 8 / 1e9
    return {"workload": f"3D VE Stokes (Stokes3D_ve_perf.jl kernels), {precision.upper()}, {n}^3, box 10^3, "
                        "spherical inclusion r=1 mu=1e-3",
            "nx": n, "ny": n, "nz": n,
            "l2": f"inputs larger than L2 ({field_gb:.2f} GB per field)" if field_gb > 0.126 else
                  f"inputs of {field_gb:.3f} GB per field: not larger than L2"}


def run_reference(args, ws, rank, pg):
    if rank != 0:
        return
    n = args.cpu_n
    vals = []
    for s in range(args.warmup + args.steps):
        v, thr, dt = cpu_sample(n, args.cpu_iters)
        if s >= args.warmup:
            vals.append(v)
    val = sum(vals) / len(vals)
    sample = f"Stokes3D_ve_perf.jl kernels at {n}^3, {args.cpu_iters} PT iterations per step (OpenMP FP64 restatement)"
    line = {
        "impl": "reference", "metric": METRIC, "value": round(val, 3), "unit": "GB/s", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": DATA_3D,
        "config": workload_config(args.n, "fp64"),
        "cpu_baseline": {"value": round(val, 3), "unit": "GB/s", "cores": thr, "kind": "port",
                         "sample": sample},
        "e2e": {"value": round(val, 3), "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference's own CPU path (Julia ParallelStencil Threads) cannot run here: no Julia runtime; "
                "timed instead: the oracle port of the same kernels",
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------ GPU arm
def block_kernel_means(blocks, nout):
    """Mean duration (ms) of the first kernel, the second kernel and the rest of a block (the
    check; in mixed precision the FP64 fold and the sources/check) over check blocks whose
    per-kernel times (pts_kernel_times: compute_Pt_τ!, compute_V! + bc, ..., the rest) were
    read after each block."""
    a = b = c = 0.0
    for t in blocks:
        a += sum(t[2 * q] for q in range(nout))
        b += sum(t[2 * q + 1] for q in range(nout))
        c += sum(t[2 * nout:])
    k = max(len(blocks), 1)
    return a / (k * nout), b / (k * nout), c / k


def run_ours(args, ws, rank, local, pg):
    import numpy as np
    import torch

    import ptstokes

    torch.cuda.set_device(local)
    n = args.n
    nout = args.iters_per_step
    variant = args.variant
    s = ptstokes.Solver(variant, n, n, n, nout=nout, eps=1e-300, iter_max=nout - 1,
                        single_pass=args.single_pass, precision=args.precision, stencil=args.stencil,
                        stencil_tile=args.stencil_tile, stencil_vtile=args.stencil_vtile, stencil_kz=args.stencil_kz)
    s.setup_inclusion()
    s.assign_tau()
    stream = torch.cuda.ExternalStream(s.stream_handle())
    # A step is one graph launch: nout PT iterations + check. On the FP64 two-kernel path the
    # graph also records a CUDA event after each kernel (pts_set_kernel_timing), read back
    # after each step, so the roofline's per-kernel durations come from the timed region.
    per_kernel = not args.single_pass
    blocks = []
    if per_kernel:
        s.set_kernel_timing(True)

    def step():
        s.solve()
        if per_kernel:
            blocks.append(s.kernel_times())

    for _ in range(args.warmup):
        step()
    s.sync()
    blocks.clear()
    torch.cuda.synchronize()
    barrier(pg)
    clk = ClockSampler(local)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    barrier(pg)
    clocks = clk.stop()
    t_ms = max_over_ranks(e0.elapsed_time(e1), pg)
    iters = args.steps * nout
    t_it = t_ms / 1e3 / iters
    value = ws * a_eff(n) / t_it / 1e9

    # the dominant kernel compute_Pt_τ! (25 arrays/launch) and compute_V!+bc (14): their mean
    # durations over the timed region (per_kernel), else timed alternating right after it, in
    # the state the timed steps left, each launch bracketed by CUDA events on the context's stream
    mixed = args.precision == "mixed"

    def time_pair(reps=20):
        # the mixed path's FP32 sweep kernels on its corrections, else the FP64 kernels
        fa = (lambda: s._ck(s.lib.pts_sweep32_kernel(s.ctx, 0))) if mixed else s.compute_Pt_tau
        fb = (lambda: s._ck(s.lib.pts_sweep32_kernel(s.ctx, 1))) if mixed else s.compute_V_bc
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * reps + 1)]
        ev[0].record(stream)
        for q in range(reps):
            fa()
            ev[2 * q + 1].record(stream)
            fb()
            ev[2 * q + 2].record(stream)
        ev[-1].synchronize()
        ta = sum(ev[2 * q].elapsed_time(ev[2 * q + 1]) for q in range(reps)) / reps
        tb = sum(ev[2 * q + 1].elapsed_time(ev[2 * q + 2]) for q in range(reps)) / reps
        return ta, tb

    if per_kernel:
        ms_A, ms_B, ms_check = block_kernel_means(blocks, nout)
    else:
        (ms_A, ms_B), ms_check = time_pair(), None
    peak, peak_kind = hbm_peak()
    # algorithmic bytes: FP64 compute_Pt_τ! 25 arrays x 8 B, compute_V! + bc 14 x 8 B; the
    # FP32 sweep's δ-form kernels 20 x 4 B and 17 x 4 B
    bytes_A = (20 * 4 if mixed else 25 * 8) * n ** 3
    bytes_B = (17 * 4 if mixed else 14 * 8) * n ** 3
    achieved = bytes_A / (ms_A / 1e3) / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "dram_traffic_per_cell.txt")  # from the committed ncu capture
    if os.path.exists(tp):
        try:
            tj = None if mixed else json.load(open(tp)).get("k3_Pt_tau_zs" if args.stencil == 0 else "k3_Pt_tau")
            if tj:
                traffic = tj["bytes_per_cell"] * n ** 3
        except Exception:
            traffic = None

    # e2e through the public API with host buffers: per step upload the initial fields
    # (Mus, Vx, Vy, Vz) from pinned host memory, set up, iterate, read Pt back.
    e2e = None
    if not args.no_e2e:
        host = {}
        # ICs exactly as the script builds them (Stokes3D_ve_perf.jl:164-172), in pinned memory
        shapes = {"Vx": (n + 1, n, n), "Vy": (n, n + 1, n), "Vz": (n, n, n + 1), "Mus": (n, n, n)}
        dx = 10.0 / n
        for name, shp in shapes.items():
            t = torch.empty(int(np.prod(shp)), dtype=torch.float64, pin_memory=True)
            host[name] = t.numpy().reshape(shp, order="F")
        ix = np.arange(n + 1, dtype=np.float64)
        host["Vx"][...] = (-1.0 * (ix * dx - 0.5 * 10.0))[:, None, None]
        host["Vy"][...] = 0.0
        host["Vz"][...] = (1.0 * (ix * dx - 0.5 * 10.0))[None, None, :]
        X = (ix[:n] * dx + 0.5 * dx) - 0.5 * 10.0
        rad2 = (X[:, None, None] ** 2 + X[None, :, None] ** 2) + X[None, None, :] ** 2
        host["Mus"][...] = np.where(rad2 < 1.0, 1e-3, 1.0)
        h2d = sum(a.nbytes for a in host.values())
        d2h = n * n * n * 8
        # `--e2e-contexts` contexts in flight, one host thread each (the C calls release the
        # GIL): the copies and set-up of one overlap the PT iterations of another
        nctx = max(1, min(args.e2e_contexts, args.steps))
        ctxs = [s] + [ptstokes.Solver(variant, n, n, n, nout=nout, eps=1e-300, iter_max=nout - 1,
                                      single_pass=args.single_pass, precision=args.precision, stencil=args.stencil,
                        stencil_tile=args.stencil_tile, stencil_vtile=args.stencil_vtile, stencil_kz=args.stencil_kz)
                      for _ in range(nctx - 1)]
        outs = [torch.empty(n * n * n, dtype=torch.float64, pin_memory=True).numpy().reshape((n, n, n), order="F")
                for _ in ctxs]

        def e2e_step(c, out, before_solve=None):
            for name, a in host.items():
                c._ck(c.lib.pts_set_field(c.ctx, ptstokes._abi.FIELD_ID[name], a.ctypes.data, a.size))
            c.smooth(10, 1.0)
            c.compute_maxloc()
            c.compute_iter_params()
            c.assign_tau()
            if before_solve:
                before_solve()
            c.solve()
            c._ck(c.lib.pts_get_field(c.ctx, ptstokes._abi.FIELD_ID["Pt"], out.ctypes.data, out.size))

        for c, o in zip(ctxs, outs):
            e2e_step(c, o)
            c.sync()
        share = [args.steps // nctx + (1 if q < args.steps % nctx else 0) for q in range(nctx)]
        torch.cuda.synchronize()
        barrier(pg)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        a.synchronize()
        failures = []
        # staggered start: context q begins its first step once context q-1 has launched its
        # first solve, so one context's copies and set-up run while another iterates (started
        # together, the contexts would copy at the same time and iterate at the same time)
        solving = [threading.Event() for _ in ctxs]

        def worker(q, c, o, k):
            try:
                if q > 0 and not solving[q - 1].wait(timeout=600):
                    raise RuntimeError("the previous context did not start")
                for step in range(k):
                    e2e_step(c, o, solving[q].set if step == 0 else None)
            except Exception as exc:  # re-raised below: a failed step must not yield a number
                failures.append(exc)
            finally:
                solving[q].set()

        threads = [threading.Thread(target=worker, args=(q, c, o, k))
                   for q, (c, o, k) in enumerate(zip(ctxs, outs, share))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        if failures:
            raise failures[0]
        for c in ctxs:
            c.sync()
        b.record(stream)
        b.synchronize()
        t_e2e = max_over_ranks(a.elapsed_time(b), pg)
        for c in ctxs[1:]:
            c.close()
        e2e = {"value": round(ws * a_eff(n) * nout * args.steps / (t_e2e / 1e3) / 1e9, 3), "unit": "GB/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": round(t_e2e / args.steps, 3), "contexts": nctx,
               "includes": "per step: pinned H2D of Mus,Vx,Vy,Vz; set-up kernels; nout PT iterations + check; "
                           "D2H of Pt; with several contexts, started staggered, the copies of one overlap the "
                           "iterations of another"}

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v, thr, dt = cpu_sample(args.cpu_n, args.cpu_iters)
        cpu = {"value": round(v, 3), "unit": "GB/s", "cores": thr, "kind": "port",
               "sample": f"oracle (C++/OpenMP FP64 restatement of Stokes3D_ve_perf.jl) at {args.cpu_n}^3, "
                         f"{args.cpu_iters} PT iterations, {dt:.1f} s",
               "time_to_tol_2d_127": small_2d_case()}

    # per step: 2 kernels per iteration and the check (k3_check, k_check_finalize); mixed:
    # the sweeps' 2 per iteration, the fold, the sources/check (3) and, in pts_solve's
    # preparation, the FP32 coefficient copy and the sources again (4)
    launches = args.steps * (2 * nout + 2) if args.precision == "fp64" else args.steps * (2 * nout + 8)
    s.close()
    ttt = ttt2 = incl = None
    if args.ttt_n > 0:
        ttt = time_to_tol(args, args.ttt_n, stream_cls=torch.cuda.ExternalStream)
    if args.ttt_n2 > 0:
        ttt2 = time_to_tol(args, args.ttt_n2, stream_cls=torch.cuda.ExternalStream)
    if args.incl_default_n > 0:
        incl = inclusions_block(args.incl_default_n, args.log10_range, rank, clocks_too=False)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "GB/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(t_ms / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32 sweeps, f64 correction",
            "data": DATA_3D,
            "config": workload_config(n, args.precision),
            "run": {"iters_per_step": nout, "t_it_ms": round(t_it * 1e3, 4),
                    "path": "CUDA graph per check block (2 kernels per PT iteration" +
                            (", a CUDA event-record node after each)" if per_kernel else ")"),
                    "parallelism": f"replicas x{ws}"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "traffic": traffic,
                         "kernel": ("k3_corrA_zs" if mixed else "k3_Pt_tau_zs") if args.stencil == 0 else
                                   ("k3_corrA" if mixed else "k3_Pt_tau"),
                         "peak_kind": peak_kind, "kernel_ms": round(ms_A, 4), "algorithmic_bytes": bytes_A,
                         "kernel_ms_from": "mean over the timed region's launches" if per_kernel else
                                           "20 alternating launches after the timed region",
                         "check_ms_per_block": None if ms_check is None else round(ms_check, 4),
                         "other_kernel": {"name": ("k3_V_bc_zs<float>" if mixed else "k3_V_bc_zs") if args.stencil == 0
                                          else ("k3_corrB" if mixed else "k3_V_bc"), "ms": round(ms_B, 4),
                                          "achieved": round(bytes_B / (ms_B / 1e3) / 1e9, 1)}},
            "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clocks,
            "time_to_tol": ttt, "time_to_tol_small": ttt2, "inclusions_20": incl,
        }
        print(json.dumps(line), flush=True)


def run_2d(args, ws, rank, local, pg):
    """The 2D visco-elastic perf script (Stokes2D_ve_perf.jl) at `--n2`^2: T_eff = A_eff/t_it
    with the script's A_eff = 18*nx*ny*8 bytes (Stokes2D_ve_perf.jl:173), a step being one
    check block of `--iters-per-step` PT iterations (two kernels each) + one check."""
    import torch

    import ptstokes

    torch.cuda.set_device(local)
    n, nout = args.n2, args.iters_per_step
    s = ptstokes.Solver("2d_ve_perf", n, n, nout=nout, eps=1e-300, iter_max=nout - 1, stencil=args.stencil,
                        stencil_tile=args.stencil_tile, stencil_kz=args.stencil_kz)
    s.setup_inclusion()
    s.assign_tau()
    stream = torch.cuda.ExternalStream(s.stream_handle())
    s.set_kernel_timing(True)  # a CUDA event after each kernel of the check block's graph
    blocks = []
    for _ in range(args.warmup):
        s.solve()
    s.sync()
    barrier(pg)
    clk = ClockSampler(local)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.solve()
        blocks.append(s.kernel_times())
    e1.record(stream)
    e1.synchronize()
    barrier(pg)
    clocks = clk.stop()
    t_ms = max_over_ranks(e0.elapsed_time(e1), pg)
    t_it = t_ms / 1e3 / (args.steps * nout)
    aeff = 18 * n * n * 8

    ms_A, ms_B, ms_check = block_kernel_means(blocks, nout)
    peak, peak_kind = hbm_peak()
    bytes_A = 15 * n * n * 8  # Vx Vy Gdτ Mus Pt τ(3) τ_o(3) read, Pt τ(3) written
    traffic = None
    tp = os.path.join(ROOT, "profiles", "dram_traffic_per_cell.txt")  # from the committed ncu capture
    if args.stencil == 0 and os.path.exists(tp):
        try:
            tj = json.load(open(tp)).get("k2_Pt_tau_ys")
            traffic = tj["bytes_per_cell"] * n * n if tj else None
        except Exception:
            traffic = None
    s.close()
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        v, thr, dt = cpu_sample_2d(args.cpu_n2, args.cpu_iters2)
        cpu = {"value": round(v, 3), "unit": "GB/s", "cores": thr, "kind": "port",
               "sample": f"oracle (C++/OpenMP FP64 restatement of Stokes2D_ve_perf.jl) at {args.cpu_n2}^2, "
                         f"{args.cpu_iters2} PT iterations, {dt:.1f} s"}
    if rank == 0:
        line = {
            "metric": "T_eff GB/s, 2D VE perf (Stokes2D_ve_perf.jl), FP64, 1 B200", "value": round(ws * aeff / t_it / 1e9, 3),
            "unit": "GB/s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(t_ms / args.steps, 3), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (the script's circular inclusion r=1 mu=1e-3, pure shear, G=1, dt=1)",
            "config": {"workload": f"2D VE Stokes (Stokes2D_ve_perf.jl kernels), FP64, {n}^2, box 10^2", "nx": n,
                       "ny": n, "iters_per_step": nout, "t_it_ms": round(t_it * 1e3, 5),
                       "A_eff": "18 arrays x 8 B per cell (Stokes2D_ve_perf.jl:173)",
                       "path": "CUDA graph per check block (2 kernels per PT iteration, a CUDA event-record "
                               "node after each)",
                       "l2": f"inputs larger than L2 ({n * n * 8 / 1e6:.0f} MB per field)"},
            "reference_published": {"value": 932.8, "unit": "GB/s", "hardware": "A100 SXM4",
                                    "source": "output/out_Stokes2D_ve_perf_ampere.txt:45 (8191^2)"},
            "roofline": {"bound": "hbm", "achieved": round(bytes_A / (ms_A / 1e3) / 1e9, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(bytes_A / (ms_A / 1e3) / 1e9 / peak, 4), "traffic": traffic,
                         "kernel": "k2_Pt_tau_ys" if args.stencil == 0 else "k2_Pt_tau",
                         "peak_kind": peak_kind, "kernel_ms": round(ms_A, 4), "algorithmic_bytes": bytes_A,
                         "kernel_ms_from": "mean over the timed region's launches",
                         "check_ms_per_block": round(ms_check, 4),
                         "other_kernel": {"name": "k2_V_bc", "ms": round(ms_B, 4),
                                          "achieved": round(9 * n * n * 8 / (ms_B / 1e3) / 1e9, 1)}},
            "cpu_baseline": cpu, "gpu_launches": args.steps * (2 * nout + 2), "clocks": clocks,
        }
        print(json.dumps(line), flush=True)


def run_batch(args, ws, rank, local):
    """The batched 2D viscous sweep: `--batch-n` seeded instances (nx in {63,127,255,511},
    lx/ly ~ U[1,4], log10 contrast ~ U[-6,-1], buoyancy or pure shear), each to err <= 1e-8
    or its iterMax = 100max(nx,ny) (Stokes2D_param.jl:146), in one persistent launch.
    Work = Σ instances cells x PT iterations."""
    import torch

    from ptstokes.batch import Batch, TILE_SHAPES, autotune, sweep_instances

    torch.cuda.set_device(local)
    inst = sweep_instances(args.batch_n, seed=1855 + rank)
    b = Batch(inst, nout=200, eps=1e-8, iter_max=args.batch_iter_max).setup()
    tune = autotune(b)
    b.setup()
    st = torch.cuda.ExternalStream(b.stream_handle())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    res = b.solve()
    e1.record(st)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    cell_it = sum(d["nx"] * d["ny"] * it for d, it in zip(inst, res["iters"]))
    its = sorted(res["iters"])
    line = {
        "metric": "batched 2D viscous sweep to 1e-8: cell-iterations/s (one persistent launch)",
        "value": round(cell_it / sec, 1), "unit": "cell-iterations/s", "n_gpus": ws, "higher_is_better": True,
        "scaling": "weak", "dtype": "f64", "data": "synthetic seeded sweep (seed 1855)",
        "config": {"workload": f"Stokes2D_param.jl numerics, {len(inst)} uneven 2D instances", "instances": len(inst),
                   "nx_set": sorted({d["nx"] for d in inst}), "total_cells": sum(d["nx"] * d["ny"] for d in inst),
                   "tile": TILE_SHAPES[b.tile], "autotune_ms": tune.get("ms"), "graph": res["used_graph"]},
        "seconds": round(sec, 3), "converged": sum(res["converged"]),
        "iters": {"min": its[0], "median": its[len(its) // 2], "max": its[-1]},
        "T_eff_GBs": round(6 * 8 * cell_it / sec / 1e9, 1),
        "T_eff_convention": "A_eff = 6 arrays x 8 B per cell and PT iteration (Stokes2D_param.jl:212)",
        "algorithmic_GBs": round(14 * 8 * cell_it / sec / 1e9, 1),
        "algorithmic_convention": "8 arrays read (Vx Vy Pt txx tyy txy Mus rhog) + 6 written, 8 B each",
    }
    # roofline of the one launch: the operands of its two phases per cell-iteration (compute_P!
    # + compute_τ! reads 7 arrays and writes 4, compute_V! + bc reads 7 and writes 2: 20 x 8 B),
    # against the measured copy peak; DRAM traffic per cell-iteration from the committed capture
    peak, peak_kind = hbm_peak()
    alg = 20 * 8 * cell_it
    line["roofline"] = {"bound": "hbm", "achieved": round(alg / sec / 1e9, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(alg / sec / 1e9 / peak, 4), "traffic": round(167.3 * cell_it),
                        "traffic_from": "profiles/k2_batch_sweep_64inst.md (167.3 B per cell-iteration)",
                        "kernel": "k2_batch", "peak_kind": peak_kind, "kernel_ms": round(sec * 1e3, 3),
                        "algorithmic_bytes": alg}
    b.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_batch_ve(args, ws, rank, local):
    """The visco-elastic aspect-ratio sweep: Stokes2D_ve_param.jl for every FACT x NSUB of
    runme_Stokes2D_aspect_ratio.jl at RESOL = `--ve-ny` (5 Maxwell steps each, eps = 1e-6,
    nout = nx, iterMax = 100nx), all instances in one persistent launch; beside it the same
    instances as separate contexts (`--ve-contexts` in flight on their own streams). Work =
    Σ instances cells x PT iterations; iteration totals checked against the published rows of
    output/out_Stokes2D_ve_aspect_ratio_param.txt (a committed fixture)."""
    import time

    import torch

    from ptstokes.batch import TILE_SHAPES, BatchVE, aspect_ratio_instances, autotune
    from ptstokes.scripts import aspect_ratio_sweep

    torch.cuda.set_device(local)
    nsubs = tuple(args.ve_nsub)
    inst = aspect_ratio_instances(nsubs=nsubs, resols=(args.ve_ny,))
    b = BatchVE(inst, tile=max(args.ve_tile, 0))
    b.setup()
    tune = autotune(b) if args.ve_tile < 0 else {}
    st = torch.cuda.ExternalStream(b.stream_handle())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    res = b.solve()
    e1.record(st)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    cell_it = sum(d["nx"] * d["ny"] * it for d, it in zip(b.instances, res["ittot"]))
    golden = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden", "reference_output_lines.json")
    rows = json.load(open(golden))["out_Stokes2D_ve_aspect_ratio_param.txt"]
    pub = {tuple(r.split()[:4]): int(r.split()[4]) for r in rows}
    keyed = [tuple(ln.split()[:4]) for ln in res["lines"]]
    have = [q for q, k in enumerate(keyed) if k in pub]
    match = [q for q in have if res["ittot"][q] == pub[keyed[q]]]
    line = {
        "metric": "batched 2D VE aspect-ratio sweep (Stokes2D_ve_param.jl x FACT x NSUB), one persistent launch: "
                  "cell-iterations/s",
        "value": round(cell_it / sec, 1), "unit": "cell-iterations/s", "n_gpus": ws, "higher_is_better": True,
        "scaling": "weak", "dtype": "f64", "data": "the reference's own sweep problem (no random input)",
        "config": {"workload": f"{len(inst)} instances: RESOL {args.ve_ny}, NSUB {list(nsubs)}, FACT 1.0..0.1, "
                               f"5 Maxwell steps each, eps 1e-6", "instances": len(inst),
                   "total_cells": sum(d["nx"] * d["ny"] for d in b.instances), "tile": TILE_SHAPES[b.tile],
                   "autotune_ms": tune.get("ms"), "graph": res["used_graph"]},
        "seconds": round(sec, 3), "ittot": {"min": min(res["ittot"]), "max": max(res["ittot"])},
        "converged_last_step": sum(res["converged"]),
        "published_rows_matched": f"{len(match)} of {len(have)} (iteration totals equal)",
    }
    peak, peak_kind = hbm_peak()
    alg = 24 * 8 * cell_it  # phase A reads 11 arrays and writes 4, phase B reads 7 and writes 2
    line["roofline"] = {"bound": "hbm", "achieved": round(alg / sec / 1e9, 1), "peak": peak, "unit": "GB/s",
                        "frac": round(alg / sec / 1e9 / peak, 4), "traffic": None, "kernel": "k2_batch_ve",
                        "peak_kind": peak_kind, "kernel_ms": round(sec * 1e3, 3), "algorithmic_bytes": alg}
    b.close()
    if args.ve_contexts > 0:
        t0 = time.perf_counter()
        out = aspect_ratio_sweep(facts=tuple(sorted({d["fact"] for d in inst}, reverse=True)), nsubs=nsubs,
                                 resols=(args.ve_ny,), in_flight=args.ve_contexts)
        sec_ctx = time.perf_counter() - t0
        by_key = {(r["fact"], r["nsub"], r["ny"]): r["ittot"] for r in out}
        same = all(by_key[(d["fact"], d["nsub"], d["ny"])] == t for d, t in zip(b.instances, res["ittot"]))
        line["contexts"] = {"seconds": round(sec_ctx, 3), "in_flight": args.ve_contexts,
                            "same_iteration_totals": same, "speedup_of_one_launch": round(sec_ctx / sec, 2)}
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_adjoint(args, ws, rank, local):
    """Adjoint gradient of the 3D viscous solve at `--adj-n`³: viscosity = matrix 1 plus 20
    seeded spherical inclusions (radii U[0.3,0.8], log10 μ U[-L,L], L = `--log10-range`),
    smoothed 10x; Vobs =
    Vz on the top interior plane from a forward solve on that field times a log-normal
    perturbation (σ = 0.5 in log10 μ, Gaussian correlation of 8 cells); J = ½‖Vz − Vobs‖².
    Timed: forward solve + transposed (adjoint) solve + ∂J/∂log μ, each solve to 1e-8.
    Checked: a directional derivative of J along a smooth random direction by central
    differences (two more forward solves)."""
    import numpy as np
    import torch

    from ptstokes.adjoint import ViscousAdjoint, inclusion_set, lognormal_factor, viscosity_field

    torch.cuda.set_device(local)
    n = args.adj_n
    L = args.log10_range
    incl = inclusion_set(seed=1855 + rank, log10_mu=(-L, L))
    pert = lognormal_factor((n, n, n), sigma=0.5, corr=8.0, seed=1856 + rank)
    p = ViscousAdjoint(n, n, n, eps=1e-8, nout=200, iter_max=2e5)
    # the synthetic observations: the inclusion field times the log-normal perturbation
    p.set_viscosity(viscosity_field(n, n, n, incl) * pert)
    obs = p.forward()
    vobs = p.top_vz()
    # the field whose gradient is taken is built on the device (pts_init_inclusions + smooth!)
    p.set_inclusions(incl)
    mus = viscosity_field(n, n, n, incl)
    st = torch.cuda.ExternalStream(p.fwd.stream_handle())
    clk = ClockSampler(local)
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    J, g, fo, ao = p.misfit_gradient(vobs)
    e1.record(st)
    e1.synchronize()
    clocks = clk.stop()
    sec = e0.elapsed_time(e1) / 1e3
    # directional derivative along a smooth direction δ (unit standard deviation in log μ)
    delta = np.log(lognormal_factor((n, n, n), sigma=1.0, corr=8.0, seed=1857 + rank)) / np.log(10.0)
    dd_adj = float(np.sum(g * delta))
    mus0 = p.mus.copy()
    h = 1e-3
    Js = []
    for sgn in (1, -1):
        p.mus = mus0 * np.exp(sgn * h * delta)
        p.forward()
        r = p.top_vz() - vobs
        Js.append(0.5 * float(np.sum(r * r)))
    p.mus = mus0
    dd_fd = (Js[0] - Js[1]) / (2 * h)
    its = fo["iters"] + ao["iters"]
    bytes_it = 23 * n ** 3 * 8  # 3D viscous: the A_eff convention without the 6 τ_o arrays
    line = {
        "metric": f"adjoint gradient dJ/dlog(mu), 3D viscous {n}^3: forward + adjoint solve + gradient",
        "value": round(sec, 3), "unit": "s", "n_gpus": ws, "higher_is_better": False, "scaling": "weak",
        "dtype": "f64", "data": "synthetic seeded 20-inclusion field and log-normal perturbation",
        "config": {"workload": f"3D viscous Stokes {n}^3, J = 1/2 |Vz(top) - Vobs|^2", "eps": 1e-8, "nout": 200,
                   "inclusions": 20, "log10_mu_range": [-L, L], "perturbation": "sigma 0.5 log10, 8-cell Gaussian"},
        "forward": {"iters": fo["iters"], "converged": fo["converged"], "err": fo["last"]["err"]},
        "adjoint": {"iters": ao["iters"], "converged": ao["converged"], "err": ao["last"]["err"]},
        "observation_solve_iters": obs["iters"], "J": J,
        "T_eff_GBs": round(bytes_it * its / sec / 1e9, 1),
        "T_eff_convention": "23 arrays x 8 B per cell and PT iteration (3D viscous)",
        "directional_check": {"adjoint": dd_adj, "central_difference": dd_fd, "h": h,
                              "rel_err": abs(dd_adj - dd_fd) / max(abs(dd_fd), 1e-300)},
        "clocks": clocks,
    }
    p.close()
    if args.adj_ve_steps > 0:
        line["visco_elastic"] = adjoint_ve(args, n, mus, incl, pert, delta, rank)
    if rank == 0:
        print(json.dumps(line), flush=True)


def adjoint_ve(args, n, mus, incl, pert, delta, rank):
    """The visco-elastic variant: `--adj-ve-steps` Maxwell steps (G = 1, dt = 1), each to 1e-8,
    per-step stress checkpoints, the backward adjoint time loop; J on the last step."""
    import numpy as np
    import torch

    from ptstokes.adjoint import ViscoElasticAdjoint

    nt = args.adj_ve_steps
    p = ViscoElasticAdjoint(n, n, n, nt=nt, eps=1e-8, nout=200, iter_max=2e5)
    p.set_viscosity(mus * pert)
    p.forward()
    vobs = p.top_vz()
    p.set_inclusions(incl)
    st = torch.cuda.ExternalStream(p.fwd.stream_handle())
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(st)
    J, g, fo, ao = p.misfit_gradient(vobs)
    e1.record(st)
    e1.synchronize()
    sec = e0.elapsed_time(e1) / 1e3
    dd_adj = float(np.sum(g * delta))
    mus0, h, Js = p.mus.copy(), 1e-3, []
    for sgn in (1, -1):
        p.mus = mus0 * np.exp(sgn * h * delta)
        p.forward()
        r = p.top_vz() - vobs
        Js.append(0.5 * float(np.sum(r * r)))
    dd_fd = (Js[0] - Js[1]) / (2 * h)
    p.close()
    return {"steps": nt, "seconds": round(sec, 3), "forward_iters": [r["iters"] for r in fo],
            "adjoint_iters": [r["iters"] for r in ao], "converged": all(r["converged"] for r in fo + ao),
            "checkpoint_bytes": 6 * nt * n ** 3 * 8, "J": J,
            "directional_check": {"adjoint": dd_adj, "central_difference": dd_fd, "h": h,
                                  "rel_err": abs(dd_adj - dd_fd) / max(abs(dd_fd), 1e-300)}}


def inclusions_block(n, L, rank, clocks_too=True):
    """Mixed precision on the 20-inclusion 3D viscous problem at n^3 (viscosity = matrix 1
    plus 20 seeded spheres, radii U[0.3,0.8], log10 μ U[-L,L], built on the device by
    pts_init_inclusions and smoothed 10x there): time to err <= 1e-8 in plain FP64 and with
    FP32 inner sweeps + FP64 defect correction, same problem and check; per-field L2 and max
    errors of the mixed solution against the FP64 one."""
    import torch

    import ptstokes
    from ptstokes.adjoint import inclusion_array, inclusion_set

    rows = inclusion_array(inclusion_set(seed=1855 + rank, log10_mu=(-L, L)))
    out, fields = {}, {}
    clk = ClockSampler(torch.cuda.current_device())
    clk.start()
    for prec in ("fp64", "mixed"):
        s = ptstokes.Solver("3d_v", n, n, n, precision=prec, eps=1e-8, nout=200, iter_max=4e5)
        s.init_inclusions(rows, mus0=1.0, ebg=1.0)  # the 20-sphere field, built on the device
        s.smooth(10, 1.0)
        s.compute_maxloc()
        s.compute_iter_params()
        s.sync()
        st = torch.cuda.ExternalStream(s.stream_handle())
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st)
        r = s.solve()
        b.record(st)
        b.synchronize()
        sec = a.elapsed_time(b) / 1e3
        out[prec] = {"seconds": round(sec, 3), "iters": r["iters"], "converged": r["converged"], "err": r["last"]["err"],
                     "T_eff_GBs": round(23 * n ** 3 * 8 * r["iters"] / sec / 1e9, 1)}
        fields[prec] = device_fields(s)
        s.close()
    clocks = clk.stop()
    blk = {"grid": n, "workload": f"3D viscous Stokes {n}^3, 20 seeded inclusions (set-up on the device)",
           "inclusions": 20, "log10_mu_range": [-L, L], "eps": 1e-8, "nout": 200,
           "fp64": out["fp64"], "mixed": out["mixed"],
           "speedup_mixed_vs_fp64": round(out["fp64"]["seconds"] / out["mixed"]["seconds"], 3),
           "mixed_error_vs_fp64": field_errors(fields["mixed"], fields["fp64"]),
           "T_eff_convention": "23 arrays x 8 B per cell and PT iteration (3D viscous, FP64 bytes for both)",
           "deviation": "log10 mu in [-2, 2], not [-4, 4]: with the reference's 3D numerics the +-4 field "
                        "diverges or stalls in plain FP64 too" if L < 4 else None}
    if clocks_too:
        blk["clocks"] = clocks
    return blk


def run_inclusions(args, ws, rank, local):
    """The 20-inclusion mixed-vs-FP64 comparison (``inclusions_block``) as its own JSON line."""
    import torch

    torch.cuda.set_device(local)
    n, L = args.incl_n, args.log10_range
    blk = inclusions_block(n, L, rank)
    line = {
        "metric": f"time to err <= 1e-8, 3D viscous {n}^3 with 20 inclusions: FP32 inner sweeps + FP64 correction vs FP64",
        "value": blk["speedup_mixed_vs_fp64"], "unit": "speed-up (x)", "n_gpus": ws,
        "higher_is_better": True, "scaling": "weak", "dtype": "f32 sweeps, f64 correction",
        "data": "synthetic seeded 20-inclusion field",
        "config": {"workload": blk["workload"], "inclusions": 20, "log10_mu_range": [-L, L], "eps": 1e-8,
                   "nout": 200},
        "fp64": blk["fp64"], "mixed": blk["mixed"], "mixed_error_vs_fp64": blk["mixed_error_vs_fp64"],
        "T_eff_GBs": {p: blk[p]["T_eff_GBs"] for p in ("fp64", "mixed")},
        "T_eff_convention": blk["T_eff_convention"], "deviation": blk["deviation"], "clocks": blk["clocks"],
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_damped(args, ws, rank, local):
    """The damped ("accel. 1") scheme of scripts/previous_damp against the current one, on
    the reference's own problems: PT iterations and device time to err <= 1e-8 for 2D
    Maxwell VE (Stokes2D_ve0.jl vs Stokes2D_ve.jl, 5 physical steps) at each of
    `--damp-n2`, and for 3D viscous (Stokes3D0_multixpu.jl on one rank vs the 3D viscous
    variant) at each of `--damp-n3`. The reference's published 2D VE totals of both schemes
    (its output/ files, kept in tests/golden) are listed beside ours."""
    import torch

    import ptstokes

    torch.cuda.set_device(local)
    pub = {}
    try:
        with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "tests", "golden",
                               "reference_output_lines.json")) as fh:
            lines = json.load(fh)
        for key, name in (("2d_ve", "out_Stokes2D_ve.txt"), ("2d_ve_damp", "out_Stokes2D_ve0.txt")):
            pub[key] = {int(r.split()[0]): int(r.split()[2]) for r in lines.get(name, [])}
    except OSError:
        pass

    def solve(variant, dims):
        s = ptstokes.Solver(variant, *dims)
        s.setup_inclusion()
        s.sync()
        st = torch.cuda.ExternalStream(s.stream_handle())
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st)
        res = s.run()
        b.record(st)
        b.synchronize()
        s.close()
        return {"ittot": res["ittot"], "iters": res["iters"], "converged": res["converged"],
                "seconds": round(a.elapsed_time(b) / 1e3, 4)}

    clk = ClockSampler(local)
    clk.start()
    rows = []
    for n in args.damp_n2:
        row = {"problem": f"2D Maxwell VE {n}^2, 5 steps"}
        for v in ("2d_ve", "2d_ve_damp"):
            row[v] = solve(v, (n, n))
            if n in pub.get(v, {}):
                row[v]["published_ittot"] = pub[v][n]
        rows.append(row)
    for n in args.damp_n3:
        row = {"problem": f"3D viscous {n}^3, one solve"}
        for v in ("3d_v", "3d_v_damp"):
            row[v] = solve(v, (n, n, n))
        rows.append(row)
    clocks = clk.stop()
    big = [r for r in rows if "2d_ve" in r][-1]
    line = {
        "metric": "PT iterations to err <= 1e-8: damped scheme (scripts/previous_damp) / current scheme, 2D VE",
        "value": round(big["2d_ve_damp"]["ittot"] / big["2d_ve"]["ittot"], 3), "unit": "iteration ratio",
        "n_gpus": ws, "higher_is_better": False, "scaling": "weak", "dtype": "f64",
        "data": "the reference's inclusion problem (synthetic, deterministic)",
        "config": {"workload": big["problem"], "eps": 1e-8, "nout": "the scripts' (200 VE, 500 viscous)"},
        "rows": rows, "clocks": clocks,
        "note": ("published_ittot: the reference's output files; its Stokes2D_ve0 totals do not match what "
                 "the committed Stokes2D_ve0.jl computes (the oracle's restatement agrees with the GPU)"),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def time_to_tol(args, n, stream_cls):
    """Time to tolerance of the converged problem of the metric: `nt` physical steps of
    3D VE, each PT loop run to err <= 1e-8 with a check every 200 iterations
    (Stokes3D_ve_multixpu.jl:128-134 numerics on the Stokes3D_ve_perf.jl kernels), plain
    FP64 vs FP32 sweeps + FP64 defect correction, same problem, same check."""
    import torch

    import ptstokes

    out = {"grid": n, "nt": args.ttt_nt, "eps": 1e-8, "nout": 200}
    fields = {}
    for prec in ("fp64", "mixed"):
        s = ptstokes.Solver("3d_ve_perf", n, n, n, precision=prec, nt=args.ttt_nt, nout=200, iter_max=2e5, eps=1e-8)
        s.setup_inclusion()
        s.sync()
        st = stream_cls(s.stream_handle())
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(st)
        res = s.run()
        b.record(st)
        b.synchronize()
        sec = a.elapsed_time(b) / 1e3
        out[prec] = {"seconds": round(sec, 3), "iters": res["iters"], "ittot": res["ittot"],
                     "converged": res["converged"], "err": res["last"]["err"],
                     "T_eff_GBs": round(a_eff(n) * res["ittot"] / sec / 1e9, 1)}
        fields[prec] = device_fields(s)
        s.close()
    out["speedup_mixed_vs_fp64"] = round(out["fp64"]["seconds"] / out["mixed"]["seconds"], 3)
    out["T_eff_convention"] = ("the FP64 A_eff (29 arrays x 8 B) per PT iteration for both paths: for the mixed "
                               "path an FP64-equivalent rate; its FP32 sweeps move 43 arrays x 4 B per iteration")
    out["mixed_error_vs_fp64"] = field_errors(fields["mixed"], fields["fp64"])
    return out


ITERATED = ("Pt", "Vx", "Vy", "Vz", "txx", "tyy", "tzz", "txy", "txz", "tyz")


def device_fields(s):
    """The ten iterated fields of a context, copied into dense device tensors."""
    import numpy as np
    import torch

    out = {}
    for k in ITERATED:
        t = torch.empty(int(np.prod(s.shape(k))), dtype=torch.float64, device="cuda")
        s.get_device(k, t.data_ptr(), t.numel())
        out[k] = t
    torch.cuda.synchronize()
    return out


def field_errors(got, ref):
    """Per field: ||got-ref||_2/||ref||_2 and max|got-ref|/max|ref| (computed on the device)."""
    out = {}
    for k, r in ref.items():
        d = got[k] - r
        out[k] = {"l2_rel": float(d.norm() / max(float(r.norm()), 1e-300)),
                  "max_rel": float(d.abs().max() / max(float(r.abs().max()), 1e-300))}
    return out


def resolve_block_defaults(args, ws):
    """The time-to-tolerance (511^3, 255^3) and 20-inclusion (255^3) blocks take minutes per
    replica: they belong to the one-GPU line, and a replica run (ws > 1) measures the
    throughput alone unless a grid is given for them."""
    if args.ttt_n is None:
        args.ttt_n = 511 if ws == 1 else 0
    if args.ttt_n2 is None:
        args.ttt_n2 = 255 if ws == 1 else 0
    if args.incl_default_n is None:
        args.incl_default_n = 255 if ws == 1 else 0
    return args


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=511)
    ap.add_argument("--variant", default="3d_ve_perf", choices=["3d_ve_perf", "3d_ve", "3d_v", "2d_ve_perf"],
                    help="2d_ve_perf: the 2D perf script at --n2 (its own JSON line)")
    ap.add_argument("--n2", type=int, default=8191)
    ap.add_argument("--cpu-n2", type=int, default=2047)
    ap.add_argument("--cpu-iters2", type=int, default=101)
    ap.add_argument("--single-pass", type=int, nargs="?", const=1, default=0, choices=[0, 1, 2],
                    help="one launch per PT iteration: 1 staged kernel, 2 direct-load kernel")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--stencil", type=int, default=0, choices=[0, 1],
                    help="0: z-marching TMA-staged kernels, 1: one thread per point")
    ap.add_argument("--stencil-tile", type=int, default=0, help="tile configuration of the TMA-staged compute_Pt_τ!")
    ap.add_argument("--stencil-vtile", type=int, default=0, help="tile configuration of the TMA-staged compute_V!")
    ap.add_argument("--stencil-kz", type=int, default=0, help="z-planes (2D: rows) per block of the TMA-staged kernels")
    ap.add_argument("--ttt-n", type=int, default=None,
                    help="grid of the time-to-tolerance comparison (0: skip; default 511 on one GPU, skipped on more)")
    ap.add_argument("--ttt-n2", type=int, default=None,
                    help="a second, smaller time-to-tolerance grid (0: skip; default 255 on one GPU, skipped on more)")
    ap.add_argument("--incl-default-n", type=int, default=None,
                    help="grid of the 20-inclusion mixed-vs-FP64 block of the default line "
                         "(0: skip; default 255 on one GPU, skipped on more)")
    ap.add_argument("--ttt-nt", type=int, default=5, help="physical steps of the time-to-tolerance comparison")
    ap.add_argument("--batch", action="store_true", help="run the batched 2D sweep instead")
    ap.add_argument("--batch-n", type=int, default=256)
    ap.add_argument("--batch-ve", action="store_true",
                    help="run the batched visco-elastic aspect-ratio sweep (Stokes2D_ve_param.jl) instead")
    ap.add_argument("--ve-ny", type=int, default=127, help="RESOL of the aspect-ratio sweep")
    ap.add_argument("--ve-nsub", type=int, nargs="*", default=[1, 2, 4], help="NSUB values of the aspect-ratio sweep")
    ap.add_argument("--ve-tile", type=int, default=-1,
                    help="tile shape of the aspect-ratio sweep (0..3; -1: the autotuner's choice)")
    ap.add_argument("--ve-contexts", type=int, default=4,
                    help="contexts in flight for the per-instance comparison run (0: skip)")
    ap.add_argument("--adjoint", action="store_true", help="run the adjoint-gradient configuration instead")
    ap.add_argument("--adj-n", type=int, default=255)
    ap.add_argument("--adj-ve-steps", type=int, default=5, help="visco-elastic adjoint steps (0: skip)")
    ap.add_argument("--inclusions", action="store_true", help="run the 20-inclusion mixed-precision comparison")
    ap.add_argument("--incl-n", type=int, default=255)
    ap.add_argument("--log10-range", type=float, default=2.0,
                    help="inclusion log10 viscosity drawn from U[-L, L] (adjoint and inclusion modes)")
    ap.add_argument("--batch-iter-max", type=float, default=0,
                    help="common iterMax of the sweep (0: 100*max(nx,ny) per instance)")
    ap.add_argument("--damped", action="store_true",
                    help="compare iterations to tolerance of the damped scheme (scripts/previous_damp)")
    ap.add_argument("--damp-n2", type=int, nargs="*", default=[63, 127, 255, 511])
    ap.add_argument("--damp-n3", type=int, nargs="*", default=[63, 127])
    ap.add_argument("--iters-per-step", type=int, default=200)
    ap.add_argument("--cpu-n", type=int, default=511)
    ap.add_argument("--cpu-iters", type=int, default=25)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--e2e-contexts", type=int, default=2, help="contexts in flight in the end-to-end measurement")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    ws, rank, local, pg = dist_setup()
    resolve_block_defaults(args, ws)
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank, pg)
        elif args.batch:
            run_batch(args, ws, rank, local)
        elif args.batch_ve:
            run_batch_ve(args, ws, rank, local)
        elif args.adjoint:
            run_adjoint(args, ws, rank, local)
        elif args.inclusions:
            run_inclusions(args, ws, rank, local)
        elif args.damped:
            run_damped(args, ws, rank, local)
        elif args.variant == "2d_ve_perf":
            run_2d(args, ws, rank, local, pg)
        else:
            run_ours(args, ws, rank, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
