"""Benchmark of the B200 Trotter-Suzuki evolution.

Workload (the configuration the headline metric is quoted on): 2D GPE
imaginary-time ground state in FP64 on a 2048 x 2048 lattice over length 24,
closed boundaries, harmonic trap omega_x = 1, omega_y = 1.5, g = 100,
Omega = 0; initial state a normalised Gaussian (sigma 2) times
(1 + 0.01 u), u seeded uniform in [-1, 1); dt = 1e-4, renormalised every step.
One bench step = one evolve() of 2000 Trotter steps, so the default 10 timed
steps are the configuration's 20000-step run.  Synthetic inputs of the
configuration's shape; nothing is read from disk.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (torchrun, one process per GPU) every rank evolves its own copy
(replicas: a single lattice is not split across GPUs), times are the max over
ranks and the value is the total site-steps of all ranks per second.

`--impl reference` times the reference's own CPU implementation (the
reference arm's value) and, on the same GPU, the reference's own CUDA kernel
(`reference_gpu_kernel`).

The JSON line reports: value (device-resident, CUDA events on the kernel's
stream), e2e (through the C ABI from pinned host buffers, state copied in and
out every step), the roofline of the step kernel against the measured HBM
peak, the FP32-storage form on the same workload, the reference's own CPU
implementation timed on this host (cpu_baseline), clocks sampled during the
timed region and the number of kernel launches.
"""
import argparse
import ctypes as C
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "trotter-suzuki-mpi_b200"))

import numpy as np  # noqa: E402

N_SIDE = 2048
LENGTH = 24.0
OMEGA_X, OMEGA_Y = 1.0, 1.5
G = 100.0
DT = 1e-4
TROTTER_PER_STEP = 2000
BYTES_PER_SITE_STEP = {"fp64": 40, "fp32": 20}  # imaginary time: psi in + psi out + real table
SEED = 20240601
WORKLOAD = "gpe_imaginary_time_2048"


def initial_state(grid_info):
    """Normalised Gaussian (sigma 2) x (1 + 0.01 u) over the tile (host numpy)."""
    W, H = grid_info["dim_x"], grid_info["dim_y"]
    dx, dy = grid_info["delta_x"], grid_info["delta_y"]
    x = (np.arange(W) + 0.5) * dx - W * dx * 0.5
    y = (np.arange(H) + 0.5) * dy - H * dy * 0.5
    X, Y = np.meshgrid(x, y)
    w = 1.0 / 4.0  # omega = 1 / sigma^2
    psi = np.sqrt(w / math.pi) * np.exp(-(w * X * X + w * Y * Y) * 0.5)
    rng = np.random.Generator(np.random.PCG64(SEED))
    psi = psi * (1.0 + 0.01 * rng.uniform(-1.0, 1.0, psi.shape))
    psi = psi / math.sqrt(np.sum(psi * psi) * dx * dy)
    return psi.astype(np.complex128)


def measured_peak():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


_PINNED = []


def pinned_array(shape):
    """A float64 numpy array in page-locked host memory (the host buffers of
    the end-to-end legs); the tensor that owns it is kept for the process."""
    import torch
    t = torch.empty(shape, dtype=torch.float64, pin_memory=True)
    _PINNED.append(t)
    return t.numpy()


def committed_traffic(summary="step_kernel_gpe_imag_2048.md"):
    """DRAM bytes (read + write) per step-kernel launch on a workload, from
    its committed ncu summary (a line `dram_bytes_per_launch: <int>`), if any."""
    import re
    path = os.path.join(REPO, "profiles", summary)
    try:
        with open(path) as f:
            m = re.search(r"^dram_bytes_per_launch:\s*(\d+)", f.read(), re.M)
        return int(m.group(1)) if m else None
    except OSError:
        return None


def committed_traffic_per_site(summary, sites):
    """DRAM bytes per launch scaled to `sites` from a committed capture of a
    smaller case of the same kernel (lines `dram_bytes_per_launch: <int>` and
    `sites_per_launch: <int>`), if any."""
    import re
    t = committed_traffic(summary)
    try:
        with open(os.path.join(REPO, "profiles", summary)) as f:
            m = re.search(r"^sites_per_launch:\s*(\d+)", f.read(), re.M)
    except OSError:
        return None
    if t is None or not m:
        return None
    return int(t * sites / int(m.group(1)))


def rotating_frame_traffic():
    """DRAM bytes per FP64 rotating-frame step launch at the current vortex
    side: the committed capture on 4096^2 (the 8192^2 workload is too large
    to capture within a few GB) scaled by the lattice sites (the traffic grows
    with the cells: every strip and segment has the same shape)."""
    t = committed_traffic("step_kernel_rotating_frame_4096.md")
    return None if t is None else int(t * (VORTEX_N / 4096.0) ** 2)


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.tmp = None

    def __enter__(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.tmp, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.tmp:
            return None
        try:
            rows = [r.split(",") for r in open(self.tmp.name).read().strip().splitlines()]
            os.unlink(self.tmp.name)
        except Exception:
            return None
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[0]))
                mx.append(float(r[1]))
                for n, v in zip(names, r[4:8]):
                    if v.strip().lower() == "active":
                        reasons.add(n)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import torch.distributed as dist
        import datetime
        dist.init_process_group("nccl" if args.impl == "b200" else "gloo",
                                timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, world, local, pg


def max_over_ranks(value, pg, device=None):
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# --------------------------------------------------------------- CPU legs
def cpu_reference_rate(psi0, budget_s=12.0, threads=None):
    """The reference's own CPU implementation (oracle/_ref, compiled from the
    reference sources; its -Ofast build when present) on the bench workload."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import tsref
    flavour = "fast" if tsref.available("fast") else ("parity" if tsref.available() else None)
    threads = threads or os.cpu_count() or 1

    def run(steps):
        cfg = tsref.make_config(N_SIDE, LENGTH, harmonic=(OMEGA_X, OMEGA_Y, 1.0, 0.0, 0.0),
                                coupling=G, delta_t=DT, segments=((1, True), (steps, True)),
                                omp_threads=threads)
        _, res = tsref.run(cfg, psi0, None, flavour=flavour)
        return res.seg_seconds[1]

    if flavour is not None:
        t = run(4)
        steps = int(max(4, min(2000, budget_s / max(t / 4, 1e-6))))
        secs = run(steps)
        kind = "reference"
        sample = (f"{N_SIDE}x{N_SIDE} GPE imaginary time, {steps} Trotter steps after 1 warm-up "
                  f"step, reference CPUBlock ({'-Ofast' if flavour == 'fast' else '-O2'} "
                  f"build), {threads} OpenMP threads")
        return N_SIDE * N_SIDE * steps / secs, threads, kind, sample, steps
    # the oracle restatement, single thread
    import oracle as O
    lat = O.Lattice(N_SIDE, LENGTH)
    V = lat.harmonic(OMEGA_X, OMEGA_Y)
    n0 = O.expectations(lat, psi0)["norm2"]
    p = lat.params(DT, True, 1.0, G, 0.0, 0.0, norm0=n0)
    tr, ti = O.exp_table(V, DT, True)
    t0 = time.perf_counter()
    O.evolve(p, psi0, tr, ti, 2)
    t = time.perf_counter() - t0
    steps = int(max(2, min(500, budget_s / max(t / 2, 1e-6))))
    t0 = time.perf_counter()
    O.evolve(p, psi0, tr, ti, steps)
    secs = time.perf_counter() - t0
    sample = f"{N_SIDE}x{N_SIDE} GPE imaginary time, {steps} Trotter steps, C restatement, 1 thread"
    return N_SIDE * N_SIDE * steps / secs, 1, "port", sample, steps


def reference_gpu_kernel_rate(psi0, steps=TROTTER_PER_STEP):
    """The reference's own CUDA kernel (CC2Kernel, src/gpukernel.cu and
    src/gpucartesian.cu, kernel_type "gpu"; compiled for sm_100a into
    oracle/_ref/libtsref_gpu.so) on the bench workload, on this box's GPU.
    Its per-step device synchronisation and cuBLAS renormalisation are part of
    what is timed, as in the reference.  None when the library or a GPU is
    missing."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import tsref
    try:
        import torch
        if not torch.cuda.is_available() or not tsref.available("gpu"):
            return None
    except ImportError:
        return None
    cfg = tsref.make_config(N_SIDE, LENGTH, harmonic=(OMEGA_X, OMEGA_Y, 1.0, 0.0, 0.0),
                            coupling=G, delta_t=DT, segments=((1, True), (steps, True)),
                            omp_threads=os.cpu_count() or 1, kernel_gpu=True)
    _, res = tsref.run(cfg, psi0, None, flavour="gpu")
    secs = res.seg_seconds[1]
    return {"value": N_SIDE * N_SIDE * steps / secs, "unit": "site-steps/s",
            "sample": f"{N_SIDE}x{N_SIDE} GPE imaginary time, {steps} Trotter steps after 1 "
                      f"warm-up step, one evolve() call, wall time",
            "kernel": "reference CC2Kernel (src/gpukernel.cu, src/gpucartesian.cu) built for "
                      "sm_100a, same GPU",
            "energy_after": res.total_energy}


def run_reference_arm(args, rank, world, pg):
    if rank != 0:
        return
    grid_info = {"dim_x": N_SIDE, "dim_y": N_SIDE, "delta_x": LENGTH / N_SIDE,
                 "delta_y": LENGTH / N_SIDE}
    psi0 = initial_state(grid_info)
    for _ in range(args.warmup):
        cpu_reference_rate(psi0, budget_s=2.0)
    rates = []
    last = None
    for _ in range(args.steps):
        last = cpu_reference_rate(psi0, budget_s=args.ref_budget)
        rates.append(last[0])
    rate = statistics.mean(rates)
    _, cores, kind, sample, steps = last
    ref_gpu = None if args.no_ref_gpu else reference_gpu_kernel_rate(psi0)
    line = {
        "impl": "reference", "metric": "site-steps/s", "value": rate, "unit": "site-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": N_SIDE * N_SIDE * steps / rate * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "lattice": f"{N_SIDE}x{N_SIDE}", "length": LENGTH,
                   "trotter_steps_per_step": steps, "dt": DT, "g": G,
                   "omega_xy": [OMEGA_X, OMEGA_Y], "boundary": "closed", "imag_time": True},
        "cpu_baseline": {"value": rate, "unit": "site-steps/s", "cores": cores, "kind": kind,
                         "sample": sample},
        "e2e": {"value": rate, "unit": "site-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_gpu_kernel": ref_gpu,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- GPU leg
def build_solver(kernel_type):
    import trottersuzuki_b200 as ts
    grid = ts.Lattice2D(N_SIDE, LENGTH)
    state = ts.State(grid)
    info = {"dim_x": grid.dim_x, "dim_y": grid.dim_y, "delta_x": grid.delta_x,
            "delta_y": grid.delta_y}
    psi0 = initial_state(info)
    state.init_state_matrix(psi0.real, psi0.imag)
    pot = ts.HarmonicPotential(grid, OMEGA_X, OMEGA_Y)
    ham = ts.Hamiltonian(grid, pot, 1.0, G)
    solver = ts.Solver(grid, state, ham, DT, kernel_type=kernel_type)
    return ts, grid, state, pot, ham, solver, psi0


def time_device(solver, handle, stream, steps):
    """K bench steps with the state resident in HBM: evolve(-T) keeps the tile
    on the device (no copy back), events on the kernel's stream."""
    import torch
    from trottersuzuki_b200 import launch_count
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    l0 = launch_count()
    e0.record(stream)
    for _ in range(steps):
        solver.evolve(-TROTTER_PER_STEP, True)
    e1.record(stream)
    e1.synchronize()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), launch_count() - l0


def run_b200_arm(args, rank, world, local, pg):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    from trottersuzuki_b200 import _capi
    L = _capi.lib()

    # ---- FP64, device resident (value)
    ts, grid, state, pot, ham, solver, psi0 = build_solver("gpu")
    stream = torch.cuda.Stream(device=device)
    solver.evolve(-1, True)  # builds the kernel (table, norm0, upload)
    handle = solver.kernel_handle()
    _capi.check(L.ts_b200_set_stream(handle, C.c_void_p(stream.cuda_stream)), handle)
    for _ in range(args.warmup):
        solver.evolve(-TROTTER_PER_STEP, True)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    with Clocks(local) as clocks:
        ms, launches = time_device(solver, handle, stream, args.steps)
    if pg:
        pg.barrier()
    ms = max_over_ranks(ms, pg, device)
    site_steps = float(N_SIDE) * N_SIDE * TROTTER_PER_STEP * args.steps
    value = world * site_steps / (ms * 1e-3)
    shape = _capi.LaunchShape()
    L.ts_b200_launch_info(handle, C.byref(shape))

    # energies and tile of the final FP64 state (for the FP32 comparison)
    solver.evolve(0, True)  # copies the tile back (get_sample)
    e64 = solver.get_total_energy()
    n64 = solver.get_squared_norm()
    psi64 = state.get_state()

    # ---- e2e: through the C ABI with pinned host buffers, every step copies
    # the state in (H2D) and the result out (D2H)
    W, H = grid.dim_x, grid.dim_y
    nbytes = W * H * 8
    bufs = []
    for _ in range(4):
        p = C.c_void_p()
        _capi.check(L.ts_b200_host_alloc(C.byref(p), nbytes))
        bufs.append(p)
    re_in = np.ctypeslib.as_array(C.cast(bufs[0], C.POINTER(C.c_double)), shape=(H, W))
    im_in = np.ctypeslib.as_array(C.cast(bufs[1], C.POINTER(C.c_double)), shape=(H, W))
    re_in[...] = psi0.real
    im_in[...] = psi0.imag
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)

    def e2e_step():
        _capi.check(L.ts_b200_set_state(handle, bufs[0], bufs[1], W), handle)
        _capi.check(L.ts_b200_evolve(handle, TROTTER_PER_STEP), handle)
        _capi.check(L.ts_b200_get_sample(handle, W, 0, 0, W, H, bufs[2], bufs[3]), handle)

    for _ in range(args.warmup):
        e2e_step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), pg, device)
    e2e_value = world * site_steps / (e2e_ms * 1e-3)
    for p in bufs:
        L.ts_b200_host_free(p)
    del solver, ham, pot, state, grid

    # ---- FP32 storage on the same workload
    fp32 = None
    if not args.no_fp32:
        ts, grid, state, pot, ham, solver32, _ = build_solver("gpu_fp32")
        solver32.evolve(-1, True)
        h32 = solver32.kernel_handle()
        _capi.check(L.ts_b200_set_stream(h32, C.c_void_p(stream.cuda_stream)), h32)
        for _ in range(args.warmup):
            solver32.evolve(-TROTTER_PER_STEP, True)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        ms32, _ = time_device(solver32, h32, stream, args.steps)
        ms32 = max_over_ranks(ms32, pg, device)
        solver32.evolve(0, True)
        e32 = solver32.get_total_energy()
        n32 = solver32.get_squared_norm()
        d = state.get_state() - psi64
        v32 = world * site_steps / (ms32 * 1e-3)
        fp32 = {"value": v32, "unit": "site-steps/s", "speedup_vs_fp64": v32 / value,
                "rel_energy_err_vs_fp64": abs(e32 - e64) / abs(e64),
                "rel_norm_err_vs_fp64": abs(n32 - n64) / abs(n64),
                "rel_psi_l2_err_vs_fp64": float(np.linalg.norm(d) / np.linalg.norm(psi64)),
                "max_abs_psi_err_vs_fp64": float(np.abs(d).max()),
                "trotter_steps_compared": (args.warmup + args.steps) * TROTTER_PER_STEP + 1,
                "bytes_per_site_step": BYTES_PER_SITE_STEP["fp32"]}
        peak32, peak32_kind = measured_peak()
        ach32 = BYTES_PER_SITE_STEP["fp32"] * v32 / world / 1e9
        fp32["roofline"] = {"bound": "hbm", "achieved": ach32, "peak": peak32, "unit": "GB/s",
                            "frac": ach32 / peak32, "peak_kind": peak32_kind,
                            "traffic": committed_traffic("step_kernel_gpe_imag_2048_fp32.md"),
                            "kernel": "tsb::step2_kernel<float, C=2, imaginary, GPE, 2 rows per "
                                      "iteration> (look-ahead walk)"}
        del solver32

    # ---- the metric's other two parts, on their own configurations: FP64
    # against FP32 storage on the precision configuration (8192^2 periodic
    # rotating-frame GPE, 5000 steps) and the adjoint/forward cost with its
    # finite-difference check (512^2 real time, 3000 steps)
    precision = adjoint = slab = None
    if not args.no_configs:
        torch.cuda.empty_cache()
        vres, vclk, _ = vortex_leg(args, local, pg, device, stream, conditioning=False)
        precision = {
            "config": vortex_config(),
            "fp64": {k: vres["fp64"][k] for k in ("value", "us_per_launch", "roofline", "energy",
                                                   "norm", "launch")},
            "fp32_store": dict({k: vres["fp32"][k] for k in ("value", "us_per_launch",
                                                             "roofline", "energy", "norm",
                                                             "launch")},
                               speedup_vs_fp64=vres["fp32"]["value"] / vres["fp64"]["value"]),
            "fp32_vs_fp64_errors": vres["errors_fp32"],
            "clocks": vclk,
        }
        torch.cuda.empty_cache()
        aout, aclk, _ = adjoint_leg(args, local, device, stream)
        adjoint = {
            "config": {"workload": "adjoint512", "lattice": f"{ADJ_N}x{ADJ_N}",
                       "length": ADJ_LENGTH, "dt": ADJ_DT, "trotter_steps": ADJ_STEPS,
                       "boundary": "closed", "loss": "sum_{x>0} |psi(T)|^2 dx dy"},
            "runs": {k: {kk: v[kk] for kk in ("adjoint_over_forward", "forward_ms", "adjoint_ms",
                                              "fd_rel_err", "fd_sites", "checkpoint_every", "g",
                                              "imag_time")}
                     for k, v in aout.items()},
            "clocks": aclk,
        }
        # the precision configuration's lattice as one lattice in slabs of
        # rows over the ranks (strong scaling; at N = 1 one slab that is its
        # own neighbour across the periodic wrap)
        torch.cuda.empty_cache()
        sres, sclk, _ = slab_leg(args, rank, world, local, pg, device)
        slab = dict(sres, config=slab_config(), clocks=sclk)

    if rank != 0:
        return

    # ---- roofline of the step kernel
    peak, peak_kind = measured_peak()
    per_launch_ms = ms / launches if launches else None  # this rank's launches; ms is the max
    bytes_per_launch = BYTES_PER_SITE_STEP["fp64"] * N_SIDE * N_SIDE
    achieved = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms else None
    traffic = committed_traffic()
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak if achieved else None, "peak_kind": peak_kind,
                "traffic": traffic,
                "algorithmic_bytes_per_launch": bytes_per_launch,
                "kernel": "tsb::step2_kernel<double, C=2, imaginary, GPE, 2 rows per iteration> "
                          "(look-ahead walk)"}

    cpu = None
    if not args.no_cpu_baseline:
        rate, cores, kind, sample, _ = cpu_reference_rate(psi0, budget_s=args.ref_budget)
        cpu = {"value": rate, "unit": "site-steps/s", "cores": cores, "kind": kind,
               "sample": sample}
        if cores > 1:
            # the same reference path on one thread (a bounded ~4 s sample)
            r1, _, _, s1, _ = cpu_reference_rate(psi0, budget_s=4.0, threads=1)
            cpu["single_thread"] = {"value": r1, "unit": "site-steps/s", "sample": s1}

    clk = clocks.summary()
    line = {
        "metric": "site-steps/s", "value": value, "unit": "site-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "lattice": f"{N_SIDE}x{N_SIDE}", "length": LENGTH,
                   "trotter_steps_per_step": TROTTER_PER_STEP, "dt": DT, "g": G,
                   "omega_xy": [OMEGA_X, OMEGA_Y], "boundary": "closed", "imag_time": True,
                   "precision": "fp64", "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2: 160 MiB read+written per Trotter step > 126 MiB",
                   "launch": {k: getattr(shape, k) for k, _ in _capi.LaunchShape._fields_}},
        "e2e": {"value": e2e_value, "unit": "site-steps/s", "h2d_bytes_per_step": 2 * nbytes,
                "d2h_bytes_per_step": 2 * nbytes,
                "path": "C ABI ts_b200_set_state / ts_b200_evolve / ts_b200_get_sample, "
                        "pinned host buffers"},
        "roofline": roofline,
        "fp32_store": fp32,
        "precision_config": precision,
        "adjoint_config": adjoint,
        "slab_config": slab,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------- batched workload
# 512 independent real-time GPE instances of uneven sizes in one persistent
# launch per Trotter step.  Sides uniform in {128, 192, ..., 1024}; per
# instance omega ~ U[0.5, 2], g ~ U[0, 200], Gaussian centre ~ U[-2, 2]^2,
# width ~ U[0.5, 2]; length 20 per side (the configuration leaves it open),
# closed boundaries, dt = 1e-4.  One bench step = 200 Trotter steps, so 10
# bench steps are the configuration's 2000-step run.
BATCH_N = 512
BATCH_SIDES = tuple(range(128, 1025, 64))
BATCH_LENGTH = 20.0
BATCH_DT = 1e-4
BATCH_TROTTER_PER_STEP = 200
BATCH_SEED = 20240602
BATCH_BYTES = {"fp64": 48, "fp32": 24}  # real time: psi in + psi out + complex table


def batch_config(n=BATCH_N, seed=BATCH_SEED):
    rng = np.random.Generator(np.random.PCG64(seed))
    sides = rng.choice(np.array(BATCH_SIDES), n)
    omega = rng.uniform(0.5, 2.0, n)
    g = rng.uniform(0.0, 200.0, n)
    centre = rng.uniform(-2.0, 2.0, (n, 2))
    width = rng.uniform(0.5, 2.0, n)
    return [dict(side=int(sides[i]), omega=float(omega[i]), g=float(g[i]),
                 cx=float(centre[i, 0]), cy=float(centre[i, 1]), width=float(width[i]))
            for i in range(n)]


def batch_solvers(ts, cfgs, kernel_type):
    out = []
    for c in cfgs:
        grid = ts.Lattice2D(c["side"], BATCH_LENGTH)
        w = 1.0 / c["width"] ** 2
        state = ts.GaussianState(grid, w, w, c["cx"], c["cy"])
        pot = ts.HarmonicPotential(grid, c["omega"], c["omega"])
        ham = ts.Hamiltonian(grid, pot, 1.0, c["g"])
        out.append((ts.Solver(grid, state, ham, BATCH_DT, kernel_type=kernel_type),
                    (grid, state, pot, ham)))
    return out


def batch_cpu_rate(cfgs, budget_s=10.0):
    """The reference's CPUBlock (oracle/_ref) on the first instances of the batch."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import tsref
    flavour = "fast" if tsref.available("fast") else ("parity" if tsref.available() else None)
    if flavour is None:
        return None
    threads = os.cpu_count() or 1
    sites = 0.0
    secs = 0.0
    used = 0
    for c in cfgs:
        w = 1.0 / c["width"] ** 2
        cfg = tsref.make_config(c["side"], BATCH_LENGTH, gaussian=(w, w, c["cx"], c["cy"], 1.0, 0.0),
                                harmonic=(c["omega"], c["omega"], 1.0, 0.0, 0.0), coupling=c["g"],
                                delta_t=BATCH_DT, segments=((1, False), (20, False)),
                                omp_threads=threads)
        _, res = tsref.run(cfg, None, None, flavour=flavour)
        sites += c["side"] ** 2 * 20
        secs += res.seg_seconds[1]
        used += 1
        if secs > budget_s:
            break
    return {"value": sites / secs, "unit": "site-steps/s", "cores": threads, "kind": "reference",
            "sample": f"first {used} instances of the batch, 20 real-time Trotter steps each, "
                      f"reference CPUBlock ({'-Ofast' if flavour == 'fast' else '-O2'} build), "
                      f"{threads} OpenMP threads"}


def run_batch_workload(args, rank, world, local, pg):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import trottersuzuki_b200 as ts
    from trottersuzuki_b200 import _capi, launch_count
    L = _capi.lib()
    cfgs = batch_config(args.batch_instances)
    total_sites = float(sum(c["side"] ** 2 for c in cfgs))
    T = BATCH_TROTTER_PER_STEP
    stream = torch.cuda.Stream(device=device)
    res = {}
    clk = None
    e2e = None
    launches = 0
    for kernel_type, prec in (("gpu", "fp64"), ("gpu_fp32", "fp32")):
        solvers = batch_solvers(ts, cfgs, kernel_type)
        sb = ts.SolverBatch([s for s, _ in solvers])
        sb.batch.set_stream(stream.cuda_stream)
        handles = [s.kernel_handle() for s, _ in solvers]
        for h in handles:
            _capi.check(L.ts_b200_set_stream(C.c_void_p(h), C.c_void_p(stream.cuda_stream)))
        t0 = time.perf_counter()
        shape = sb.autotune(trial_steps=3, use_cache=False)
        tune_s = time.perf_counter() - t0
        for _ in range(args.warmup):
            sb.batch.evolve(T)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        l0 = launch_count()
        with Clocks(local) as clocks:
            e0.record(stream)
            for _ in range(args.steps):
                sb.batch.evolve(T)
            e1.record(stream)
            e1.synchronize()
        if prec == "fp64":
            clk = clocks.summary()
            launches = launch_count() - l0
        ms = max_over_ranks(e0.elapsed_time(e1), pg, device)
        value = world * total_sites * T * args.steps / (ms * 1e-3)
        # per-instance launch loop on the same stream (each tile's own
        # graph-replayed evolve, one tile after the other)
        loop_steps = max(1, args.steps // 5)
        for h in handles:
            _capi.check(L.ts_b200_evolve(C.c_void_p(h), T))
        torch.cuda.synchronize()
        e0.record(stream)
        for _ in range(loop_steps):
            for h in handles:
                _capi.check(L.ts_b200_evolve(C.c_void_p(h), T))
        e1.record(stream)
        e1.synchronize()
        ms_loop = max_over_ranks(e0.elapsed_time(e1), pg, device)
        loop_value = world * total_sites * T * loop_steps / (ms_loop * 1e-3)
        res[prec] = {"value": value, "ms_per_step": ms / args.steps, "loop_value": loop_value,
                     "speedup_vs_loop": value / loop_value, "autotune_s": tune_s,
                     "shape": {k: shape[k] for k in ("segment_rows", "warps_per_block", "blocks")}}
        if prec == "fp64":
            # e2e: every bench step uploads all initial states from host
            # arrays, evolves the batch and reads every state back
            init = []
            for c in cfgs:
                n_side = c["side"]
                dx = BATCH_LENGTH / n_side
                x = (np.arange(n_side) + 0.5) * dx - BATCH_LENGTH * 0.5
                X, Y = np.meshgrid(x, x)
                w = 1.0 / c["width"] ** 2
                g0 = np.sqrt(w / math.pi) * np.exp(-0.5 * w * ((X - c["cx"]) ** 2 + (Y - c["cy"]) ** 2))
                re0 = pinned_array(g0.shape)
                re0[...] = g0
                im0 = pinned_array(g0.shape)
                im0[...] = 0.0
                init.append((re0, im0))
            outs = [(pinned_array(a.shape), pinned_array(a.shape)) for a, _ in init]
            h2d = sum(a.nbytes + b.nbytes for a, b in init)

            def e2e_step():
                for h, (a, b), c in zip(handles, init, cfgs):
                    _capi.check(L.ts_b200_set_state(C.c_void_p(h), a.ctypes.data, b.ctypes.data,
                                                    c["side"]))
                sb.batch.evolve(T)
                for h, (a, b), c in zip(handles, outs, cfgs):
                    n_side = c["side"]
                    _capi.check(L.ts_b200_get_sample(C.c_void_p(h), n_side, 0, 0, n_side, n_side,
                                                     a.ctypes.data, b.ctypes.data))
            e2e_step()
            torch.cuda.synchronize()
            e0.record(stream)
            for _ in range(args.steps):
                e2e_step()
            e1.record(stream)
            e1.synchronize()
            e2e_ms = max_over_ranks(e0.elapsed_time(e1), pg, device)
            e2e = {"value": world * total_sites * T * args.steps / (e2e_ms * 1e-3),
                   "unit": "site-steps/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": h2d,
                   "path": "ts_b200_set_state x512, ts_b200_batch_evolve, ts_b200_get_sample x512, "
                           "pinned host buffers"}
        sb.close()
        del solvers, sb
        torch.cuda.synchronize()
    if rank != 0:
        return
    peak, peak_kind = measured_peak()
    bytes_step = BATCH_BYTES["fp64"] * total_sites
    achieved = bytes_step / (res["fp64"]["ms_per_step"] * 1e-3 / T) / 1e9
    cpu = None if args.no_cpu_baseline else batch_cpu_rate(cfgs)
    line = {
        "metric": "site-steps/s", "value": res["fp64"]["value"], "unit": "site-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["fp64"]["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batch512_real_time", "instances": len(cfgs),
                   "sides": list(BATCH_SIDES), "total_sites": total_sites, "length": BATCH_LENGTH,
                   "dt": BATCH_DT, "trotter_steps_per_step": T, "boundary": "closed",
                   "imag_time": False, "seed": BATCH_SEED, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2: %.1f GB moved per Trotter step" % (bytes_step / 1e9)},
        "per_instance_loop": {"value": res["fp64"]["loop_value"], "unit": "site-steps/s",
                              "speedup_batch_vs_loop": res["fp64"]["speedup_vs_loop"]},
        "autotune": {"fp64": res["fp64"]["shape"], "fp32": res["fp32"]["shape"],
                     "seconds_fp64": res["fp64"]["autotune_s"]},
        "fp32_store": {"value": res["fp32"]["value"], "unit": "site-steps/s",
                       "speedup_vs_fp64": res["fp32"]["value"] / res["fp64"]["value"],
                       "loop_value": res["fp32"]["loop_value"],
                       "speedup_batch_vs_loop": res["fp32"]["speedup_vs_loop"],
                       "roofline": {"bound": "hbm", "unit": "GB/s", "peak": peak,
                                    "achieved": BATCH_BYTES["fp32"] * res["fp32"]["value"]
                                    / world / 1e9,
                                    "frac": BATCH_BYTES["fp32"] * res["fp32"]["value"]
                                    / world / 1e9 / peak,
                                    "peak_kind": peak_kind,
                                    "bytes_per_site_step": BATCH_BYTES["fp32"]}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": committed_traffic_per_site("batch_step_batch512.md", total_sites),
                     "algorithmic_bytes_per_launch": bytes_step,
                     "kernel": "tsb::batch2_kernel<double, C=2, real, no rotation, GPE, "
                               "2 rows per iteration> (look-ahead walk)"},
        "e2e": e2e,
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------- differentiation workload
# 512 x 512 over length 20, real time, FP64, closed boundaries; V = harmonic
# (omega 1) + 16 Gaussians (amplitude U[-0.5, 0.5], width U[1, 3], centres
# uniform over the box); psi0 = normalised Gaussian (sigma 1) at (-3, 0) times
# exp(2 i x); dt = 1e-4, 3000 steps; L = sum_{x > 0} |psi(T)|^2 dx dy.  Run
# linear (inverse steps) and with g = 50 (checkpoints every 100 steps).
ADJ_N = 512
ADJ_LENGTH = 20.0
ADJ_DT = 1e-4
ADJ_STEPS = 3000
ADJ_SEED = 20240603
ADJ_SITES = 64


def adjoint_setup(n=ADJ_N, seed=ADJ_SEED):
    rng = np.random.Generator(np.random.PCG64(seed))
    dx = ADJ_LENGTH / n
    x = (np.arange(n) + 0.5) * dx - ADJ_LENGTH * 0.5
    X, Y = np.meshgrid(x, x)
    V = 0.5 * (X * X + Y * Y)
    amp = rng.uniform(-0.5, 0.5, 16)
    wid = rng.uniform(1.0, 3.0, 16)
    cen = rng.uniform(-ADJ_LENGTH * 0.5, ADJ_LENGTH * 0.5, (16, 2))
    for a, w, (cx, cy) in zip(amp, wid, cen):
        V += a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * w * w))
    psi0 = np.exp(-0.5 * ((X + 3.0) ** 2 + Y ** 2)) * np.exp(2j * X)
    psi0 /= math.sqrt((np.abs(psi0) ** 2).sum() * dx * dx)
    mask = (X > 0).astype(np.float64)
    # FD sites where the wave packet travels (|x|, |y| < 6)
    sites = [(int(a), int(b)) for a, b in
             zip(rng.integers(int(n * 0.2), int(n * 0.8), ADJ_SITES),
                 rng.integers(int(n * 0.2), int(n * 0.8), ADJ_SITES))]
    return V, psi0.astype(np.complex128), mask, dx, sites


# (label, g, checkpoint interval, imaginary time)
ADJ_CASES = (("linear_inverse_steps", 0.0, 0, False), ("gpe_g50_checkpoint100", 50.0, 100, False),
             ("imag_gpe_g50_checkpoint100", 50.0, 100, True))


def adjoint_leg(args, local, device, stream, cases=ADJ_CASES, n_sites=ADJ_SITES):
    """Forward and adjoint runs of the differentiation configuration, timed on
    the device, with central finite differences of the B200 forward pass at
    `n_sites` seeded sites."""
    import torch
    import trottersuzuki_b200 as ts
    from trottersuzuki_b200 import launch_count
    from trottersuzuki_b200.adjoint import AdjointEngine
    V, psi0, mask, dx, sites = adjoint_setup()
    sites = sites[:n_sites]
    dA = dx * dx
    m = torch.tensor(mask, device=device)
    out = {}
    clk = None
    launches = 0
    for label, g, every, imag in cases:
        grid = ts.Lattice2D(ADJ_N, ADJ_LENGTH)
        ham = ts.Hamiltonian(grid, None, 1.0, g)
        desc = ts.make_desc(grid, ham, ADJ_DT, imag_time=imag, norm=1.0 if imag else 0.0)
        eng = AdjointEngine(desc, ADJ_DT, ADJ_STEPS, every)
        with torch.cuda.stream(stream):
            Vt = torch.tensor(V, dtype=torch.float64, device=device)
            p0 = torch.tensor(psi0, dtype=torch.complex128, device=device)

            def loss_of(psi_t):
                return float(((psi_t.abs() ** 2) * m).sum().item() * dA)

            fwd_ms, bwd_ms = [], []
            for it in range(args.warmup + args.steps):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e2 = torch.cuda.Event(enable_timing=True)
                l0 = launch_count()
                timed = it >= args.warmup
                clocks = Clocks(local) if (timed and label == "linear_inverse_steps" and
                                            it == args.warmup) else None
                if clocks:
                    clocks.__enter__()
                e0.record(stream)
                psi_t = eng.forward(Vt, p0)
                e1.record(stream)
                grad_t = (2.0 * dA) * m * psi_t
                gv, gp = eng.backward(grad_t)
                e2.record(stream)
                e2.synchronize()
                if clocks:
                    clocks.__exit__(None, None, None)
                    clk = clocks.summary()
                if timed:
                    fwd_ms.append(e0.elapsed_time(e1))
                    bwd_ms.append(e1.elapsed_time(e2))
                    if label == "linear_inverse_steps":
                        launches = launch_count() - l0
            L0 = loss_of(psi_t)
            gv = gv.cpu().numpy()
            gp = gp.cpu().numpy()
            # central differences of the B200 forward pass at the seeded sites
            hv, hp = 1e-4, 1e-5
            fd_v, fd_r, fd_i = [], [], []
            for (y, x) in sites:
                e = torch.zeros_like(Vt)
                e[y, x] = hv
                fd_v.append((loss_of(eng.forward(Vt + e, p0)) - loss_of(eng.forward(Vt - e, p0)))
                            / (2 * hv))
                ec = torch.zeros_like(p0)
                ec[y, x] = hp
                fd_r.append((loss_of(eng.forward(Vt, p0 + ec)) - loss_of(eng.forward(Vt, p0 - ec)))
                            / (2 * hp))
                fd_i.append((loss_of(eng.forward(Vt, p0 + 1j * ec))
                             - loss_of(eng.forward(Vt, p0 - 1j * ec))) / (2 * hp))
        ys, xs = zip(*sites)

        def rel(a, b):
            b = np.asarray(b)
            return float(np.abs(np.asarray(a) - b).max() / np.abs(b).max())

        f = statistics.median(fwd_ms)
        b = statistics.median(bwd_ms)
        out[label] = {
            "loss": L0, "forward_ms": f, "adjoint_ms": b, "adjoint_over_forward": b / f,
            "forward_site_steps_per_s": ADJ_N * ADJ_N * ADJ_STEPS / (f * 1e-3),
            "fd_rel_err": {"dL_dV": rel(gv[ys, xs], fd_v), "dL_dre_psi0": rel(gp.real[ys, xs], fd_r),
                           "dL_dim_psi0": rel(gp.imag[ys, xs], fd_i)},
            "fd_sites": len(sites), "fd_step": {"V": hv, "psi0": hp},
            "checkpoint_every": every, "g": g, "imag_time": imag}
        eng.close()
    return out, clk, launches


def run_adjoint_workload(args, rank, world, local, pg):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=device)
    out, clk, launches = adjoint_leg(args, local, device, stream)
    if rank != 0:
        return
    lin = out["linear_inverse_steps"]
    peak, peak_kind = measured_peak()
    # adjoint step: psi, lambda in and out, table, dL/dV in and out
    bytes_step = 96.0 * ADJ_N * ADJ_N
    achieved = bytes_step * ADJ_STEPS / (lin["adjoint_ms"] * 1e-3) / 1e9
    line = {
        "metric": "adjoint/forward cost", "value": lin["adjoint_over_forward"], "unit": "ratio",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": lin["forward_ms"] + lin["adjoint_ms"], "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "adjoint512_real_time", "lattice": f"{ADJ_N}x{ADJ_N}",
                   "length": ADJ_LENGTH, "dt": ADJ_DT, "trotter_steps": ADJ_STEPS,
                   "boundary": "closed", "seed": ADJ_SEED, "loss": "sum_{x>0} |psi(T)|^2 dx dy",
                   "parallelism": f"replicas{world}",
                   "l2": "state 4 MiB is L2-resident: a latency-bound size"},
        "runs": out,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                     "algorithmic_bytes_per_launch": bytes_step,
                     "kernel": "tsb::adjoint_kernel<inverse steps>"},
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------- precision workload
# 8192 x 8192 periodic lattice over length 40, real-time GPE in the rotating
# frame: harmonic trap omega = 1, g = 500, Omega = 0.7, dt = 5e-5, 5000 steps.
# psi0 = Thomas-Fermi profile sqrt(max(0, mu - V) / g) (norm 1: mu = sqrt(g / pi)
# for this trap) times exp(i theta_k) windings around 8 seeded centres uniform
# in the disk of radius 10.  The FP32-storage path runs against the FP64 path
# (the oracle here: the reference refuses periodic boundaries with a rotating
# frame, src/model.cpp:936-940).
VORTEX_N = 8192
VORTEX_LENGTH = 40.0
VORTEX_G = 500.0
VORTEX_OMEGA = 0.7
VORTEX_DT = 5e-5
VORTEX_STEPS = 5000
VORTEX_SEED = 20240604
VORTEX_BYTES = {"fp64": 48, "fp32": 24}


def vortex_initial(grid):
    """Thomas-Fermi profile times 8 windings, evaluated with torch in FP64 on
    the current device (the 8192^2 tile is 1 GiB; numpy would take ~20 s)."""
    import torch
    from trottersuzuki_b200.api import _coordinate_grid
    X, Y = _coordinate_grid(grid)
    dev = torch.device("cuda", torch.cuda.current_device())
    x = torch.tensor(np.ascontiguousarray(X[0, :]), dtype=torch.float64, device=dev)[None, :]
    y = torch.tensor(np.ascontiguousarray(Y[:, 0]), dtype=torch.float64, device=dev)[:, None]
    rng = np.random.Generator(np.random.PCG64(VORTEX_SEED))
    r = 10.0 * np.sqrt(rng.uniform(0.0, 1.0, 8))
    phi = rng.uniform(0.0, 2.0 * math.pi, 8)
    centres = np.stack([r * np.cos(phi), r * np.sin(phi)], axis=1)
    mu = math.sqrt(VORTEX_G / math.pi)
    dens = torch.clamp((mu - 0.5 * (x * x + y * y)) / VORTEX_G, min=0.0)
    theta = torch.zeros_like(dens)
    for cx, cy in centres:
        theta += torch.atan2(y - float(cy), x - float(cx))
    amp = torch.sqrt(dens)
    re = (amp * torch.cos(theta)).cpu().numpy()
    im = (amp * torch.sin(theta)).cpu().numpy()
    del x, y, dens, theta, amp
    return re, im, centres


def vortex_leg(args, local, pg, device, stream, conditioning=True, steps=VORTEX_STEPS):
    """The precision configuration: FP64 and FP32-storage runs of `steps`
    Trotter steps from the same psi0 (and, with `conditioning`, FP64 from psi0
    rounded to float), timed on the device; errors of FP32 against FP64."""
    import torch
    import trottersuzuki_b200 as ts
    from trottersuzuki_b200 import _capi, launch_count
    L = _capi.lib()
    res = {}
    clk = None
    launches = 0
    psi64 = None
    inner = None
    runs = [("gpu", "fp64"), ("gpu_fp32", "fp32")]
    if conditioning:
        runs.append(("gpu", "fp64_from_fp32_psi0"))
    for kernel_type, prec in runs:
        grid = ts.Lattice2D(VORTEX_N, VORTEX_LENGTH, periodic_x_axis=True, periodic_y_axis=True,
                            angular_velocity=VORTEX_OMEGA)
        state = ts.State(grid)
        re0, im0, centres = vortex_initial(grid)
        if prec == "fp64_from_fp32_psi0":
            re0 = re0.astype(np.float32).astype(np.float64)
            im0 = im0.astype(np.float32).astype(np.float64)
        state.init_state_matrix(re0, im0)
        pot = ts.HarmonicPotential(grid, 1.0, 1.0)
        ham = ts.Hamiltonian(grid, pot, 1.0, VORTEX_G, 0.0, VORTEX_OMEGA)
        solver = ts.Solver(grid, state, ham, VORTEX_DT, kernel_type=kernel_type)
        e0_energy = solver.get_total_energy()
        # warm-up steps, then the state is reset and the kernel rebuilt from it
        solver.evolve(-args.warmup)
        torch.cuda.synchronize()
        state.init_state_matrix(re0, im0)
        del re0, im0
        solver.update_parameters()
        solver.evolve(0)
        h = solver.kernel_handle()
        _capi.check(L.ts_b200_set_stream(C.c_void_p(h), C.c_void_p(stream.cuda_stream)))
        torch.cuda.synchronize()
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        l0 = launch_count()
        with Clocks(local) as clocks:
            ev0.record(stream)
            solver.evolve(-steps)
            ev1.record(stream)
            ev1.synchronize()
        ms = max_over_ranks(ev0.elapsed_time(ev1), pg, device)
        if prec == "fp64":
            clk = clocks.summary()
            launches = launch_count() - l0
        shape = _capi.LaunchShape()
        L.ts_b200_launch_info(C.c_void_p(h), C.byref(shape))
        solver.evolve(0)  # copies the tile back
        psi = np.array(state.p_real) + 1j * np.array(state.p_imag)
        sh = VORTEX_N * VORTEX_N
        peak, peak_kind = measured_peak()
        bpl = VORTEX_BYTES["fp32" if prec == "fp32" else "fp64"] * sh
        ach = bpl / (ms / steps * 1e-3) / 1e9
        res[prec] = {"value": pg_world(pg) * sh * steps / (ms * 1e-3), "ms": ms,
                     "us_per_launch": ms / steps * 1e3,
                     "energy": solver.get_total_energy(), "norm": solver.get_squared_norm(),
                     "initial_energy": e0_energy,
                     "roofline": {"achieved": ach, "peak": peak, "unit": "GB/s",
                                  "frac": ach / peak, "peak_kind": peak_kind,
                                  "algorithmic_bytes_per_launch": bpl},
                     "launch": {k: getattr(shape, k) for k, _ in _capi.LaunchShape._fields_},
                     "clocks": clocks.summary()}
        if prec == "fp64":
            psi64 = psi
            inner = (slice(grid.inner_start_y - grid.start_y, grid.inner_end_y - grid.start_y),
                     slice(grid.inner_start_x - grid.start_x, grid.inner_end_x - grid.start_x))
        else:
            d = psi[inner] - psi64[inner]
            res["errors_" + prec] = {
                "psi_rel_l2": float(np.linalg.norm(d) / np.linalg.norm(psi64[inner])),
                "psi_max_abs": float(np.abs(d).max()),
                "psi_max_abs_over_max": float(np.abs(d).max() / np.abs(psi64[inner]).max()),
                "norm_rel": abs(res[prec]["norm"] - res["fp64"]["norm"]) / abs(res["fp64"]["norm"]),
                "energy_rel": abs(res[prec]["energy"] - res["fp64"]["energy"]) /
                              abs(res["fp64"]["energy"])}
        del solver, ham, pot, state, grid, psi
        torch.cuda.synchronize()
    return res, clk, launches


def pg_world(pg):
    import torch.distributed as dist
    return dist.get_world_size() if pg else 1


def vortex_config(steps=VORTEX_STEPS):
    return {"workload": f"vortex{VORTEX_N}_precision", "lattice": f"{VORTEX_N}x{VORTEX_N}",
            "length": VORTEX_LENGTH, "boundary": "periodic", "g": VORTEX_G,
            "omega_rot": VORTEX_OMEGA, "dt": VORTEX_DT, "trotter_steps": steps,
            "initial": "Thomas-Fermi x 8 windings (radius 10)", "seed": VORTEX_SEED}


# ------------------------------------------------------------- slab workload
# The precision workload's lattice (8192^2, periodic, rotating frame, FP64
# real time) as ONE lattice split into slabs of rows: one slab per rank over
# NCCL (strong scaling: the whole job does the same work at every N), or
# several slabs on the one GPU of a process (--slabs-per-gpu), exchanged by
# device copies.  Each slab steps as its edge bands and its interior on two
# streams; the halo rows move while the interior runs.
SLAB_STEPS = 200      # Trotter steps per bench step
SLAB_BYTES = 48       # FP64 real time, rotating frame: psi in + out + complex table


def slab_tiles(rank, world, per_gpu, precision):
    """This rank's slab kernels of the 8192^2 vortex lattice (state and
    potential table from the same psi0 and trap as the precision workload)."""
    import torch
    import trottersuzuki_b200 as ts
    from trottersuzuki_b200 import Kernel
    from trottersuzuki_b200.api import _coordinate_grid
    from trottersuzuki_b200.slab import SlabLayout
    grid = ts.Lattice2D(VORTEX_N, VORTEX_LENGTH, periodic_x_axis=True, periodic_y_axis=True,
                        angular_velocity=VORTEX_OMEGA)
    pot = ts.HarmonicPotential(grid, 1.0, 1.0)
    ham = ts.Hamiltonian(grid, pot, 1.0, VORTEX_G, 0.0, VORTEX_OMEGA)
    whole = ts.make_desc(grid, ham, VORTEX_DT, False, 0.0, precision)
    re0, im0, _ = vortex_initial(grid)
    X, Y = _coordinate_grid(grid)
    dev = torch.device("cuda", torch.cuda.current_device())
    x = torch.tensor(np.ascontiguousarray(X[0, :]), dtype=torch.float64, device=dev)[None, :]
    ys = np.ascontiguousarray(Y[:, 0])
    n_slabs = world * per_gpu
    kernels, layouts = [], []
    for j in range(per_gpu):
        r = rank * per_gpu + j
        lay = SlabLayout(VORTEX_N, whole.halo_y, True, r, n_slabs)
        d = type(whole).from_buffer_copy(whole)
        d.dim_y = lay.rows
        d.inner_y0, d.inner_y1 = lay.inner_rows()
        d.periodic_y = 0
        d.rot_offset_y = whole.rot_offset_y + lay.start + whole.halo_y
        rows = slice(lay.start + whole.halo_y, lay.end + whole.halo_y)
        k = Kernel(d)
        k.set_state(re0[rows] + 1j * im0[rows])
        y = torch.tensor(ys[rows], dtype=torch.float64, device=dev)[:, None]
        V = (0.5 * (x * x + y * y)).contiguous()
        torch.cuda.synchronize()
        k.set_potential_device(V.data_ptr(), V.shape[1], VORTEX_DT)
        k.synchronize()
        del V, y
        kernels.append(k)
        layouts.append(lay)
    del re0, im0, X, Y
    return kernels, layouts


def slab_leg(args, rank, world, local, pg, device, per_gpu=1, split=True, steps=SLAB_STEPS):
    """Strong scaling of one lattice: value = lattice site-steps per second of
    the whole job (the slowest rank's device time)."""
    import torch
    from trottersuzuki_b200 import _capi, launch_count
    from trottersuzuki_b200.slab import NativeSlabs
    if world > 1 and per_gpu != 1:
        raise ValueError("several slabs per GPU only in a one-process run")
    kernels, layouts = slab_tiles(rank, world, per_gpu, _capi.FP64)
    stream = torch.cuda.Stream(device=device)
    for k in kernels:
        k.set_stream(stream.cuda_stream)
    if per_gpu > 1:
        slabs = NativeSlabs.local(kernels, layouts)
        transport = f"{per_gpu} slabs on one GPU, device copies"
    else:
        import torch.distributed as dist
        slabs = NativeSlabs.nccl(kernels[0], layouts[0], dist if pg else None)
        transport = "NCCL send/recv between ranks" if world > 1 else \
            "NCCL send/recv of the one slab with itself across the periodic wrap"
    slabs.set_split(split)
    edge, inner, is_split, per_step = slabs.plan(0)
    for _ in range(args.warmup):
        slabs.evolve(20)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    l0 = launch_count()
    with Clocks(local) as clocks:
        e0.record(stream)
        for _ in range(args.steps):
            slabs.evolve(steps)
        e1.record(stream)
        e1.synchronize()
    launches = launch_count() - l0
    ms = max_over_ranks(e0.elapsed_time(e1), pg, device)
    norm = sum(k.squared_norm() for k in kernels)
    if pg:
        t = torch.tensor([norm], dtype=torch.float64, device=device)
        pg.all_reduce(t)
        norm = float(t.item())
    total = VORTEX_N * VORTEX_N * steps * args.steps
    rows_here = sum(lay.inner_end - lay.inner_start for lay in layouts)
    per_gpu_bytes = SLAB_BYTES * VORTEX_N * rows_here * steps * args.steps
    peak, peak_kind = measured_peak()
    ach = per_gpu_bytes / (ms * 1e-3) / 1e9
    slabs.close()
    for k in kernels:
        k.close()
    return {"value": total / (ms * 1e-3), "unit": "site-steps/s", "ms": ms,
            "us_per_trotter_step": ms / (steps * args.steps) * 1e3,
            "slabs": world * per_gpu, "slabs_per_gpu": per_gpu, "split": bool(is_split),
            "edge_windows": edge, "interior_window": list(inner),
            "kernel_launches_per_step": per_step, "transport": transport,
            "squared_norm_after": norm,
            "roofline": {"achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                         "peak_kind": peak_kind, "algorithmic_bytes_per_site": SLAB_BYTES,
                         "note": "this rank's inner rows; halo rows recomputed by both "
                                 "neighbours are not counted"}}, clocks.summary(), launches


def slab_config(steps=SLAB_STEPS):
    return dict(vortex_config(steps), workload=f"vortex{VORTEX_N}_slabs", precision="fp64",
                split="rows, one slab per rank")


def run_slab_workload(args, rank, world, local, pg):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    res, clk, launches = slab_leg(args, rank, world, local, pg, device,
                                  per_gpu=args.slabs_per_gpu, split=not args.no_split)
    if rank != 0:
        return
    r = res["roofline"]
    line = {
        "metric": "site-steps/s", "value": res["value"], "unit": "site-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["ms"] / args.steps, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(slab_config(), parallelism=f"slabs{res['slabs']}",
                       l2="inputs larger than L2: 3 GiB moved per Trotter step in FP64"),
        "slab": res,
        "roofline": {"bound": "hbm", "achieved": r["achieved"], "peak": r["peak"],
                     "unit": "GB/s", "frac": r["frac"], "peak_kind": r["peak_kind"],
                     "traffic": None, "kernel": "tsb::step2_kernel<double, C=2, real, rotating "
                                                "frame, GPE> (look-ahead walk), edge bands + "
                                                "interior"},
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


def vortex_cpu_rate(budget_s=10.0):
    """The reference's CPUBlock (oracle/_ref) on the precision configuration's
    lattice, trap, coupling and rotating frame, on all host cores, over a
    bounded number of steps.  The reference refuses periodic boundaries with
    a rotating frame (src/model.cpp:936-940), so this runs with closed ones;
    psi0 is the normalised Gaussian of width 3 (the rate does not depend on
    the state)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import tsref
    flavour = "fast" if tsref.available("fast") else ("parity" if tsref.available() else None)
    if flavour is None:
        return None
    threads = os.cpu_count() or 1

    def run(steps):
        cfg = tsref.make_config(VORTEX_N, VORTEX_LENGTH, gaussian=(1 / 9.0, 1 / 9.0, 0.0, 0.0, 1.0, 0.0),
                                harmonic=(1.0, 1.0, 1.0, 0.0, 0.0), coupling=VORTEX_G,
                                angular_velocity=VORTEX_OMEGA, delta_t=VORTEX_DT,
                                segments=((1, False), (steps, False)), omp_threads=threads)
        _, res = tsref.run(cfg, None, None, flavour=flavour)
        return res.seg_seconds[1]

    t = run(1)
    steps = int(max(1, min(50, budget_s / max(t, 1e-6))))
    secs = run(steps)
    return {"value": VORTEX_N * VORTEX_N * steps / secs, "unit": "site-steps/s", "cores": threads,
            "kind": "reference",
            "sample": f"{VORTEX_N}x{VORTEX_N}, closed boundaries (the reference refuses periodic "
                      f"ones with a rotating frame), Omega = {VORTEX_OMEGA}, g = {VORTEX_G}, "
                      f"{steps} real-time Trotter steps after 1 warm-up step, reference CPUBlock "
                      f"({'-Ofast' if flavour == 'fast' else '-O2'} build), {threads} OpenMP threads"}


def run_vortex_workload(args, rank, world, local, pg):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=device)
    res, clk, launches = vortex_leg(args, local, pg, device, stream, conditioning=True)
    if rank != 0:
        return
    cpu = None if args.no_cpu_baseline else vortex_cpu_rate(budget_s=args.ref_budget)
    r64 = res["fp64"]["roofline"]
    line = {
        "metric": "site-steps/s", "value": res["fp64"]["value"], "unit": "site-steps/s",
        "n_gpus": world, "steps": 1, "warmup": args.warmup,
        "ms_per_step": res["fp64"]["ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": dict(vortex_config(), parallelism=f"replicas{world}",
                       l2="inputs larger than L2: 3 GiB moved per Trotter step in FP64"),
        "fp64": res["fp64"],
        "fp32_store": dict(res["fp32"], speedup_vs_fp64=res["fp32"]["value"] / res["fp64"]["value"]),
        "fp32_vs_fp64_errors": res["errors_fp32"],
        "fp64_from_fp32_rounded_psi0_vs_fp64": res["errors_fp64_from_fp32_psi0"],
        "roofline": {"bound": "hbm", "achieved": r64["achieved"], "peak": r64["peak"],
                     "unit": "GB/s", "frac": r64["frac"], "peak_kind": r64["peak_kind"],
                     "traffic": rotating_frame_traffic(),
                     "traffic_source": "ncu capture on 4096^2 scaled by the sites",
                     "algorithmic_bytes_per_launch": r64["algorithmic_bytes_per_launch"],
                     "kernel": "tsb::step2_kernel<double, C=2, real, rotating frame, GPE, 2 rows "
                               "per iteration> (look-ahead walk) + halo"},
        "cpu_baseline": cpu,
        "clocks": clk,
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------ time-dependent potential workload
# Real-time GPE in a trap whose centre oscillates along x,
# V(x, y, t) = 1/2 ((x - a sin(w t))^2 + (1.5 y)^2), FP64, on the headline
# lattice (2048^2 over length 24, closed, g = 100, dt = 1e-4) from the headline
# initial state.  The reference re-tabulates V and its exponential on the host
# before every step; DevicePotential evaluates V with torch on the GPU and
# builds the table on the device.  One bench step = 200 Trotter steps through
# Solver.evolve; the host path is timed on a bounded sample of steps.
MT_AMP, MT_FREQ = 1.0, 5.0
MT_STEPS = 200
MT_HOST_STEPS = 4


MT_TIME_BATCH = 16
# per site-step of the step that reads the potential rows: psi in + out, V
MT_BYTES = 40


def moving_trap(x, y, t):
    return 0.5 * ((x - MT_AMP * math.sin(MT_FREQ * t)) ** 2 + (OMEGA_Y * y) ** 2)


def moving_trap_batched(x, y, t):
    """moving_trap for a tensor t of step times (DevicePotential time_batch mode)."""
    import torch
    return 0.5 * ((x - MT_AMP * torch.sin(MT_FREQ * t)) ** 2 + (OMEGA_Y * y) ** 2)


def run_moving_trap_workload(args, rank, world, local, pg):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import trottersuzuki_b200 as ts
    from trottersuzuki_b200 import launch_count

    def solver_for(kind):
        grid = ts.Lattice2D(N_SIDE, LENGTH)
        state = ts.State(grid)
        info = {"dim_x": grid.dim_x, "dim_y": grid.dim_y, "delta_x": grid.delta_x,
                "delta_y": grid.delta_y}
        psi0 = initial_state(info)
        state.init_state_matrix(psi0.real, psi0.imag)
        if kind == "device":
            pot = ts.DevicePotential(grid, moving_trap_batched, device=device,
                                     time_batch=MT_TIME_BATCH)
        elif kind == "device_per_step":
            pot = ts.DevicePotential(grid, moving_trap, device=device)
        elif kind == "host":
            pot = ts.Potential(grid)
            pot.init_potential(moving_trap)
        else:
            pot = ts.HarmonicPotential(grid, OMEGA_X, OMEGA_Y)
        ham = ts.Hamiltonian(grid, pot, 1.0, G)
        return ts.Solver(grid, state, ham, DT, kernel_type="gpu"), (grid, state, pot, ham)

    def timed(solver, n, calls):
        cur = torch.cuda.current_stream(device)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if pg:
            pg.barrier()
        l0 = launch_count()
        e0.record(cur)
        for _ in range(calls):
            solver.evolve(n)
        torch.cuda.synchronize()  # the static solver queues on its kernel's own stream
        e1.record(cur)
        e1.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), pg, device), launch_count() - l0

    sites = float(N_SIDE) * N_SIDE
    dev, keep_dev = solver_for("device")
    for _ in range(args.warmup):
        dev.evolve(-MT_STEPS)
    with Clocks(local) as clocks:
        ms_dev, launches = timed(dev, -MT_STEPS, args.steps)  # state stays on the device
    ms_e2e, _ = timed(dev, MT_STEPS, max(1, args.steps // 2))  # copied into the State per call
    e2e_calls = max(1, args.steps // 2)
    del dev, keep_dev
    # one pot_function call per step (Python float t)
    dps, keep_dps = solver_for("device_per_step")
    dps.evolve(-MT_STEPS)
    ms_dps, _ = timed(dps, -MT_STEPS, args.steps)
    del dps, keep_dps
    # the same kernel with a static table: the step alone
    static, keep_static = solver_for("static")
    static.evolve(-MT_STEPS)
    ms_static, _ = timed(static, -MT_STEPS, args.steps)
    del static, keep_static
    # the host path (numpy V, host exponential, upload) on a bounded sample
    hst, keep_host = solver_for("host")
    hst.evolve(-1)
    ms_host, _ = timed(hst, -MT_HOST_STEPS, 1)
    del hst, keep_host
    if rank != 0:
        return
    v_dev = world * sites * MT_STEPS * args.steps / (ms_dev * 1e-3)
    v_static = world * sites * MT_STEPS * args.steps / (ms_static * 1e-3)
    v_host = world * sites * MT_HOST_STEPS / (ms_host * 1e-3)
    v_e2e = world * sites * MT_STEPS * e2e_calls / (ms_e2e * 1e-3)
    v_dps = world * sites * MT_STEPS * args.steps / (ms_dps * 1e-3)
    peak, peak_kind = measured_peak()
    line = {
        "metric": "site-steps/s", "value": v_dev, "unit": "site-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_dev / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "moving_trap_2048", "lattice": f"{N_SIDE}x{N_SIDE}",
                   "length": LENGTH, "boundary": "closed", "g": G, "dt": DT,
                   "potential": f"1/2((x - {MT_AMP} sin({MT_FREQ} t))^2 + ({OMEGA_Y} y)^2)",
                   "trotter_steps_per_step": MT_STEPS, "imag_time": False,
                   "time_batch": MT_TIME_BATCH,
                   "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2: 192 MiB moved per Trotter step"},
        "e2e": {"value": v_e2e, "unit": "site-steps/s", "h2d_bytes_per_step": 8 * MT_STEPS,
                "d2h_bytes_per_step": 2 * 8 * int(sites),
                "path": "Solver.evolve(200) with DevicePotential (step times uploaded, "
                        "state copied into the State after each call)"},
        "static_potential_same_kernel": {"value": v_static, "unit": "site-steps/s"},
        "device_potential_per_step_call": {"value": v_dps, "unit": "site-steps/s"},
        "roofline": {"bound": "hbm", "unit": "GB/s", "peak": peak, "peak_kind": peak_kind,
                     "achieved": MT_BYTES * v_dev / world / 1e9,
                     "frac": MT_BYTES * v_dev / world / 1e9 / peak,
                     "traffic": committed_traffic("step_kernel_moving_trap_2048.md"),
                     "algorithmic_bytes_per_site_step": MT_BYTES,
                     "note": "over the whole Trotter step, the user's torch evaluation of V "
                             "included",
                     "kernel": "tsb::step2_kernel<double, C=2, real, GPE, potential rows, "
                               "2 rows per iteration>"},
        "host_potential_path": {"value": v_host, "unit": "site-steps/s",
                                "sample": f"{MT_HOST_STEPS} Trotter steps",
                                "speedup_of_device_path": v_dev / v_host},
        "clocks": clocks.summary(),
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------ two-component workload
# Two species (Hamiltonian2Component) on the headline lattice, real time, FP64:
# species a the headline Gaussian, species b the same displaced by 1.5 in x;
# harmonic traps (1, 1.5) and (1.2, 1), g_a = 100, g_b = 80, g_ab = 60,
# mass_b = 1.2, Rabi coupling omega = 5 + 2i, dt = 1e-4.  One bench step =
# one evolve(200) of the drop-in two-state Solver.  A species-site-step is
# one site of one species advanced by one Trotter step.
TWO_STEPS = 200
TWO_BYTES = 64  # per species-site-step of the step kernel: psi in + out, table, other species


def run_two_component_workload(args, rank, world, local, pg):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import trottersuzuki_b200 as ts
    from trottersuzuki_b200 import launch_count
    grid = ts.Lattice2D(N_SIDE, LENGTH)
    info = {"dim_x": grid.dim_x, "dim_y": grid.dim_y, "delta_x": grid.delta_x,
            "delta_y": grid.delta_y}
    a0 = initial_state(info)
    b0 = np.roll(a0, int(round(1.5 / grid.delta_x)), axis=1)
    sa, sb = ts.State(grid), ts.State(grid)
    sa.init_state_matrix(a0.real, a0.imag)
    sb.init_state_matrix(b0.real, b0.imag)
    pa = ts.HarmonicPotential(grid, OMEGA_X, OMEGA_Y)
    pb = ts.HarmonicPotential(grid, 1.2, 1.0)
    ham = ts.Hamiltonian2Component(grid, pa, pb, 1.0, 1.2, G, 60.0, 80.0, 5.0, 2.0)
    solver = ts.Solver(grid, sa, ham, DT, State2=sb)
    e_start = solver.get_total_energy()
    for _ in range(args.warmup):
        solver.evolve(-TWO_STEPS)
    cur = torch.cuda.current_stream(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    l0 = launch_count()
    with Clocks(local) as clocks:
        e0.record(cur)
        for _ in range(args.steps):
            solver.evolve(-TWO_STEPS)
        torch.cuda.synchronize()
        e1.record(cur)
        e1.synchronize()
    launches = launch_count() - l0
    ms = max_over_ranks(e0.elapsed_time(e1), pg, device)
    # e2e: evolve(200) with the states copied into both States each call
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(cur)
    for _ in range(max(1, args.steps // 2)):
        solver.evolve(TWO_STEPS)
    torch.cuda.synchronize()
    t1.record(cur)
    t1.synchronize()
    ms_e2e = max_over_ranks(t0.elapsed_time(t1), pg, device)
    e_end = solver.get_total_energy()
    n_end = solver.get_squared_norm()
    if rank != 0:
        return
    sites = float(N_SIDE) * N_SIDE
    value = world * 2 * sites * TWO_STEPS * args.steps / (ms * 1e-3)
    e2e = world * 2 * sites * TWO_STEPS * max(1, args.steps // 2) / (ms_e2e * 1e-3)
    peak, peak_kind = measured_peak()
    # per species-site-step: the step kernel's 64 B; the Rabi rotation rides
    # on the next step's loads, and only the call's last one is a pass of its
    # own (32 B per species-site, once per evolve call)
    two_bytes = TWO_BYTES + 32.0 / TWO_STEPS
    achieved = two_bytes * value / world / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        cpu = two_component_cpu_rate(a0, b0, budget_s=args.ref_budget)
    line = {
        "metric": "species-site-steps/s", "value": value, "unit": "species-site-steps/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "two_component_2048", "lattice": f"{N_SIDE}x{N_SIDE}",
                   "length": LENGTH, "boundary": "closed", "g": [G, 80.0], "g_ab": 60.0,
                   "mass_b": 1.2, "rabi_omega": [5.0, 2.0], "dt": DT,
                   "trotter_steps_per_step": TWO_STEPS, "imag_time": False,
                   "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2: 384 MiB moved per Trotter step"},
        "e2e": {"value": e2e, "unit": "species-site-steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 4 * 8 * int(sites),
                "path": "two-state Solver.evolve(200), both States filled after each call"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": committed_traffic("step_kernel_two_component_2048.md"),
                     "algorithmic_bytes_per_species_site_step": two_bytes,
                     "kernel": "tsb::step2_kernel<double, C=2, real, two components, "
                               "Rabi rotation at load, 2 rows per iteration> "
                               "x 2 per Trotter step"},
        "energy_drift_rel": abs(e_end - e_start) / abs(e_start),
        "norm_after": n_end,
        "cpu_baseline": cpu,
        "clocks": clocks.summary(),
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


def two_component_cpu_rate(a0, b0, budget_s=12.0):
    """The reference's own two-state Solver (oracle/_ref) on a bounded sample
    of the two-component workload, all host threads."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import tsref
    flavour = "fast" if tsref.available("fast") else ("parity" if tsref.available() else None)
    if flavour is None:
        return None
    threads = os.cpu_count() or 1
    X = (np.arange(N_SIDE) - N_SIDE / 2 + 0.5) * (LENGTH / N_SIDE)
    Xg, Yg = np.meshgrid(X, X)
    Va = 0.5 * (OMEGA_X ** 2 * Xg ** 2 + OMEGA_Y ** 2 * Yg ** 2)
    Vb = 0.5 * (1.2 ** 2 * Xg ** 2 + Yg ** 2)

    def run(steps):
        cfg = tsref.make_config(N_SIDE, LENGTH, harmonic=None, coupling=G, delta_t=DT,
                                segments=((1, False), (steps, False)), omp_threads=threads)
        _, _, r = tsref.run2(cfg, tsref.Config2(1.2, 80.0, 60.0, 5.0, 2.0), a0, b0, Va, Vb,
                             flavour=flavour)
        return r.seg_seconds[1]

    t = run(2)
    steps = int(max(2, min(200, budget_s / max(t / 2, 1e-6))))
    secs = run(steps)
    return {"value": 2 * N_SIDE * N_SIDE * steps / secs, "unit": "species-site-steps/s",
            "cores": threads, "kind": "reference",
            "sample": f"{N_SIDE}x{N_SIDE} two species real time, {steps} Trotter steps after "
                      f"1 warm-up step, reference two-state Solver "
                      f"({'-Ofast' if flavour == 'fast' else '-O2'} build)"}


# ------------------------------------------------------ cylindrical workload
# A vortex ground state on a cylindrical (r, z) lattice: 2048 radial x 2048
# axial cells over r in [0, 12), z in [-12, 12), angular momentum l = 1,
# harmonic trap (1, 1.5), g = 100, imaginary time, dt = 1e-4, FP64; initial
# state r exp(-(r^2 + z^2) / 8) times (1 + 0.01 u).  One bench step = one
# evolve(200); the radial sweeps and the mirrored axis column run inside the
# fused step.
CYL_STEPS = 200
CYL_L = 1


def run_cylindrical_workload(args, rank, world, local, pg):
    import torch
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    import trottersuzuki_b200 as ts
    from trottersuzuki_b200 import launch_count
    from trottersuzuki_b200.api import _coordinate_grid
    grid = ts.Lattice2D(N_SIDE, LENGTH / 2, N_SIDE, LENGTH, coordinate_system="cylindrical")
    R, Z = _coordinate_grid(grid)
    rng = np.random.Generator(np.random.PCG64(SEED))
    psi0 = (R * np.exp(-(R * R + Z * Z) / 8.0) *
            (1 + 0.01 * rng.uniform(-1, 1, R.shape))).astype(np.complex128)
    state = ts.State(grid, CYL_L)
    state.init_state_matrix(psi0.real, psi0.imag)
    pot = ts.HarmonicPotential(grid, OMEGA_X, OMEGA_Y)
    ham = ts.Hamiltonian(grid, pot, 1.0, G)
    solver = ts.Solver(grid, state, ham, DT)
    for _ in range(args.warmup):
        solver.evolve(-CYL_STEPS, True)
    cur = torch.cuda.current_stream(device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    l0 = launch_count()
    with Clocks(local) as clocks:
        e0.record(cur)
        for _ in range(args.steps):
            solver.evolve(-CYL_STEPS, True)
        torch.cuda.synchronize()
        e1.record(cur)
        e1.synchronize()
    launches = launch_count() - l0
    ms = max_over_ranks(e0.elapsed_time(e1), pg, device)
    solver.evolve(0, True)
    energy = solver.get_total_energy()
    if rank != 0:
        return
    sites = float(grid.dim_x) * grid.dim_y
    value = world * sites * CYL_STEPS * args.steps / (ms * 1e-3)
    peak, peak_kind = measured_peak()
    achieved = BYTES_PER_SITE_STEP["fp64"] * value / world / 1e9
    line = {
        "metric": "site-steps/s", "value": value, "unit": "site-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "cylindrical_vortex_2048",
                   "lattice": f"{grid.dim_x}x{grid.dim_y} (r, z)",
                   "length_r": LENGTH / 2, "length_z": LENGTH, "angular_momentum": CYL_L,
                   "g": G, "omega_rz": [OMEGA_X, OMEGA_Y], "dt": DT, "imag_time": True,
                   "trotter_steps_per_step": CYL_STEPS, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2: 160 MiB moved per Trotter step"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": committed_traffic("step_kernel_cylindrical_2048.md"),
                     "algorithmic_bytes_per_site_step": BYTES_PER_SITE_STEP["fp64"],
                     "kernel": "tsb::step2_kernel<double, C=2, imaginary, cylindrical, GPE, "
                               "2 rows per iteration>"},
        "energy_after": energy,
        "clocks": clocks.summary(),
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--ref-budget", type=float, default=12.0,
                    help="seconds of reference CPU work per sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp32", action="store_true")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the precision (8192^2) and adjoint (512^2) legs of the default run")
    ap.add_argument("--no-ref-gpu", action="store_true",
                    help="reference arm: skip timing the reference's CUDA kernel")
    ap.add_argument("--split", choices=["none", "slab"], default="none",
                    help="slab: the 8192^2 vortex lattice as one lattice in slabs of rows "
                         "over the ranks (strong scaling)")
    ap.add_argument("--batch-instances", type=int, default=BATCH_N,
                    help="instances of the batch workload (the first of its seeded list; "
                         "fewer for an ncu capture)")
    ap.add_argument("--vortex-side", type=int, default=0,
                    help="lattice side of the vortex / slab workloads (default 8192; smaller "
                         "sides keep an ncu capture of their kernels within a few GB)")
    ap.add_argument("--slabs-per-gpu", type=int, default=1,
                    help="--split slab in one process: this many slabs on its GPU")
    ap.add_argument("--no-split", action="store_true",
                    help="--split slab: one launch per slab step (no edge/interior overlap)")
    ap.add_argument("--workload", choices=["gpe_imaginary_time_2048", "batch512", "adjoint512",
                                           "vortex8192", "moving_trap_2048",
                                           "two_component_2048", "cylindrical_vortex_2048"],
                    default="gpe_imaginary_time_2048")
    args = ap.parse_args()
    if args.vortex_side:
        global VORTEX_N
        VORTEX_N = int(args.vortex_side)
    args.warmup = max(3, args.warmup)
    rank, world, local, pg = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference_arm(args, rank, world, pg)
        elif args.split == "slab":
            run_slab_workload(args, rank, world, local, pg)
        elif args.workload == "batch512":
            run_batch_workload(args, rank, world, local, pg)
        elif args.workload == "adjoint512":
            run_adjoint_workload(args, rank, world, local, pg)
        elif args.workload == "vortex8192":
            run_vortex_workload(args, rank, world, local, pg)
        elif args.workload == "moving_trap_2048":
            run_moving_trap_workload(args, rank, world, local, pg)
        elif args.workload == "two_component_2048":
            run_two_component_workload(args, rank, world, local, pg)
        elif args.workload == "cylindrical_vortex_2048":
            run_cylindrical_workload(args, rank, world, local, pg)
        else:
            run_b200_arm(args, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
