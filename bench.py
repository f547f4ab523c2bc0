"""Benchmark: FP64 cell-updates/s of the 2D wave-propagation step on B200.

Workload (one "step" = one controlled time step of the whole grid):
  2D Euler shock-bubble, 1280x320 cells on [0,2]x[0,0.5], gamma=1.4, q=(rho,
  rhou,rhov,E); Mach-2 planar shock at x=0.2 moving +x into still air (rho=1,
  p=1), post-shock state from the Rankine-Hugoniot relations (p=4.5, rho=8/3,
  u=2*sqrt(1.4)*(1-3/8)); circular bubble rho=0.1, p=1, centre (0.5,0.25),
  radius 0.2 (cell-centre indicator); Roe solver with Harten-Hyman entropy fix,
  MC limiter, unsplit with transverse_waves=2, extrapolation BCs in x, walls in
  y, cfl_desired 0.9 / cfl_max 1.0.  Synthetic data of the reference's shape.

Usage:
  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One JSON line is printed by rank 0.  ``value`` is whole-job cell-updates/s
with the state resident in HBM (device-timed, L2 flushed between timed steps);
``e2e`` is the same metric through the host-buffer C ABI
(claw2_session_evolve: host state in, host state out, each call advancing
the solution by a fixed simulated interval).  With N > 1 the ranks step one
grid of 1280 x 320N cells by domain decomposition (pyclaw_b200.decomp: a
1280 x 320 slab per rank, halo rows exchanged with NCCL and the CFL number
max-reduced every step; weak scaling) and the value is the sum over ranks;
e2e stays one host-buffer session per rank.
"""
import argparse
import ctypes
import json
import math
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GAMMA = 1.4


# ---------------------------------------------------------------------------
# workload definitions (shared with the tests)
# ---------------------------------------------------------------------------
def _centers(lower, upper, n):
    delta = (upper - lower) / float(n)
    c = np.empty(n)
    for i in range(n):
        c[i] = lower + (i + 0.5) * delta
    return c, delta


def shockbubble_config(mx=1280, my=320, walls=False, split=False):
    """Returns (problem, q0, aux0, run_kwargs, tfinal) for the shock-bubble workload."""
    from pyclaw_b200 import _abi
    x, dx = _centers(0.0, 2.0, mx)
    y, dy = _centers(0.0, 0.5, my)
    X, Y = np.meshgrid(x, y, indexing='ij')
    gamma1 = GAMMA - 1.0
    # Rankine-Hugoniot post-shock state for a Mach-2 shock into rho=1, p=1, u=0
    M = 2.0
    p2 = 1.0 + 2.0 * GAMMA / (GAMMA + 1.0) * (M * M - 1.0)
    rho2 = (GAMMA + 1.0) * M * M / ((GAMMA - 1.0) * M * M + 2.0)
    u2 = M * np.sqrt(GAMMA) * (1.0 - 1.0 / rho2)
    behind = X < 0.2
    bubble = np.sqrt((X - 0.5) ** 2 + (Y - 0.25) ** 2) <= 0.2
    rho = np.where(behind, rho2, np.where(bubble, 0.1, 1.0))
    u = np.where(behind, u2, 0.0)
    p = np.where(behind, p2, 1.0)
    q = np.empty((4, mx, my), order='F')
    q[0] = rho
    q[1] = rho * u
    q[2] = 0.0
    q[3] = p / gamma1 + 0.5 * rho * u * u
    bcx = _abi.BC_WALL if walls else _abi.BC_EXTRAP
    prob = _abi.make_problem(rp=_abi.RP_EULER_4WAVE, num_eqn=4, num_waves=4, num_aux=0, mx=mx, my=my,
                             dx=dx, dy=dy, order=2, transverse=-1 if split else 2, mthlim=[4],
                             bc_lower=(bcx, _abi.BC_WALL), bc_upper=(bcx, _abi.BC_WALL),
                             params=(GAMMA, gamma1))
    smax = abs(u2) + np.sqrt(GAMMA * p2 / rho2)
    run = dict(cfl_max=1.0, cfl_desired=0.9, dt_initial=0.9 * min(dx, dy) / smax)
    return prob, q, None, run, 0.6


def acoustics_config(n=256):
    """256^2 constant-coefficient acoustics on [-1,1]^2, rho=1, K=4, walls,
    p = exp(-((r-0.25)/0.05)^2), unsplit trans=2, MC, cfl 0.9, t=0.6."""
    from pyclaw_b200 import _abi
    x, dx = _centers(-1.0, 1.0, n)
    y, dy = _centers(-1.0, 1.0, n)
    X, Y = np.meshgrid(x, y, indexing='ij')
    rho, bulk = 1.0, 4.0
    cc = np.sqrt(bulk / rho)
    zz = rho * cc
    r = np.sqrt(X ** 2 + Y ** 2)
    q = np.empty((3, n, n), order='F')
    q[0] = np.exp(-((r - 0.25) / 0.05) ** 2)
    q[1] = 0.0
    q[2] = 0.0
    prob = _abi.make_problem(rp=_abi.RP_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=0, mx=n, my=n,
                             dx=dx, dy=dy, order=2, transverse=2, mthlim=[4],
                             bc_lower=(_abi.BC_WALL, _abi.BC_WALL), bc_upper=(_abi.BC_WALL, _abi.BC_WALL),
                             params=(rho, bulk, cc, zz))
    run = dict(cfl_max=1.0, cfl_desired=0.9, dt_initial=0.9 * dx / cc)
    return prob, q, None, run, 0.6


def batched_vc_config(n=1024, seed=2024, nmin=64, nmax=384):
    """1024 variable-coefficient acoustics instances: nx, ny ~ U{64..384}; aux
    (rho, c=sqrt(K/rho)) piecewise constant over U{2..6} vertical layers with
    rho, K ~ U[1,4]; Gaussian pressure pulse of width 0.05 at a random interior
    point; MC, unsplit with transverse_waves=2, walls at the lower and
    extrapolation at the upper boundaries.  Returns (problem, instances)."""
    from pyclaw_b200 import _abi
    rng = np.random.default_rng(seed)
    insts = []
    for _ in range(n):
        nx, ny = (int(v) for v in rng.integers(nmin, nmax + 1, size=2))
        nl = int(rng.integers(2, 7))
        xs = np.sort(rng.uniform(0.0, 1.0, nl - 1))
        rho = rng.uniform(1.0, 4.0, nl)
        K = rng.uniform(1.0, 4.0, nl)
        c = np.sqrt(K / rho)
        x, dx = _centers(0.0, 1.0, nx)
        y, dy = _centers(0.0, 1.0, ny)
        X, Y = np.meshgrid(x, y, indexing='ij')
        layer = np.searchsorted(xs, x)
        aux = np.empty((2, nx, ny), order='F')
        aux[0] = rho[layer][:, None]
        aux[1] = c[layer][:, None]
        x0, y0 = rng.uniform(0.1, 0.9, size=2)
        q = np.zeros((3, nx, ny), order='F')
        q[0] = np.exp(-((X - x0) ** 2 + (Y - y0) ** 2) / 0.05 ** 2)
        insts.append(dict(q=q, aux=aux, dx=dx, dy=dy, dt=0.9 * min(dx, dy) / float(c.max())))
    prob = _abi.make_problem(rp=_abi.RP_VC_ACOUSTICS, num_eqn=3, num_waves=2, num_aux=2, mx=64, my=64,
                             dx=1.0, dy=1.0, order=2, transverse=2, mthlim=[4],
                             bc_lower=(_abi.BC_WALL, _abi.BC_WALL), bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP),
                             aux_bc_lower=(_abi.BC_WALL, _abi.BC_WALL),
                             aux_bc_upper=(_abi.BC_EXTRAP, _abi.BC_EXTRAP))
    return prob, insts


def shallow_config(n=4096):
    """Radial dam break: 4096^2 on [-2.5,2.5]^2, g = 1, h = 2 for r < 0.5 else 1,
    hu = hv = 0; Roe with the transonic fix, superbee, unsplit with
    transverse_waves=2, extrapolation BCs, cfl_desired 0.9.
    Returns (problem, q0, run settings)."""
    from pyclaw_b200 import _abi
    x, dx = _centers(-2.5, 2.5, n)
    y, dy = _centers(-2.5, 2.5, n)
    X, Y = np.meshgrid(x, y, indexing="ij")
    q = np.zeros((3, n, n), order="F")
    q[0] = np.where(X ** 2 + Y ** 2 < 0.25, 2.0, 1.0)
    prob = _abi.make_problem(rp=_abi.RP_SHALLOW_ROE, num_eqn=3, num_waves=3, num_aux=0, mx=n, my=n, dx=dx, dy=dy,
                             order=2, transverse=2, mthlim=[2], params=(1.0,))
    cmax = float(np.sqrt(2.0))
    return prob, q, dict(cfl_max=1.0, cfl_desired=0.9, dt_initial=0.9 * dx / cmax)


def adjoint_config(n=512, shots=64, nsteps=400, nrec=64, seed=7):
    """Seismic-style inversion workload on [-1,1]^2, surface at y = 1:
    variable-coefficient acoustics with a seeded target material (background
    rho = 1, K = 4 with three circular inclusions of radius 0.3, rho ~ U[1.5,3],
    K ~ U[2,8]); `shots` sources at random surface cells, each a Ricker pulse
    (peak frequency 15, delay 0.1) injected into the pressure; `nrec` receivers
    evenly spaced along the surface; MC, unsplit with transverse_waves=2;
    extrapolation on the sides and bottom, a wall at the surface; dt fixed by
    CFL 0.9 of the target material.  Returns a dict of numpy arrays and
    settings."""
    rng = np.random.default_rng(seed)
    x, dx = _centers(-1.0, 1.0, n)
    y, dy = _centers(-1.0, 1.0, n)
    X, Y = np.meshgrid(x, y, indexing="ij")
    rho_t = np.ones((n, n))
    K_t = np.full((n, n), 4.0)
    for _ in range(3):
        cx, cy = rng.uniform(-0.6, 0.6), rng.uniform(-0.7, 0.3)
        inside = (X - cx) ** 2 + (Y - cy) ** 2 < 0.3 ** 2
        rho_t[inside] = rng.uniform(1.5, 3.0)
        K_t[inside] = rng.uniform(2.0, 8.0)
    c_max = float(np.sqrt(K_t / rho_t).max())
    dt = 0.9 * min(dx, dy) / c_max
    t = dt * (np.arange(nsteps) + 1)
    from pyclaw_b200.adjoint import ricker
    wav = ricker(t, 15.0, 0.1) / (dx * dy) * dt
    src = [int(i) + n * (n - 1) for i in rng.integers(0, n, shots)]
    rec = [int(i) + n * (n - 1) for i in np.linspace(0, n - 1, nrec).round().astype(int)]
    return dict(n=n, dx=dx, dy=dy, dt=dt, rho_t=rho_t, K_t=K_t, rho0=np.ones((n, n)), K0=np.full((n, n), 4.0),
                src=src, rec=rec, wav=wav, shots=shots, nsteps=nsteps)


def make_solver(pc, prob, run):
    """A ClawSolver2D configured like `prob` (Euler shock-bubble settings)."""
    solver = pc.ClawSolver2D(pc.riemann.rp2_euler_4wave)
    solver.dimensional_split = False
    solver.transverse_waves = int(prob.transverse)
    solver.limiters = [int(prob.mthlim[w]) for w in range(prob.num_waves)]
    solver.bc_lower = [int(prob.bc_lower[0]), int(prob.bc_lower[1])]
    solver.bc_upper = [int(prob.bc_upper[0]), int(prob.bc_upper[1])]
    solver.cfl_max = run['cfl_max']
    solver.cfl_desired = run['cfl_desired']
    solver.dt_initial = run['dt_initial']
    return solver


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def _ncu_record(key):
    """Per-launch counters of one kernel from one ncu capture, kept in
    profiles/ncu_metrics.json (written from the capture that the profile
    summary of the same name describes); None if absent."""
    path = os.path.join(ROOT, "profiles", "ncu_metrics.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f).get(key)


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler(object):
    """nvidia-smi clock/throttle sampling during the timed region."""
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        # the raw samples go to $CLAW2_CLOCKS_DIR (default: the system temp dir)
        import tempfile
        d = os.environ.get("CLAW2_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(d, "clocks_bench_%d_%d.csv" % (gpu_index, os.getpid()))

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "20"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for ln in f:
                parts = [s.strip() for s in ln.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    mx = float(parts[2])
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist_init():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if torch.cuda.is_available():
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    elif torch.cuda.is_available():
        torch.cuda.set_device(local)
    return world, rank, local


def _barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda" if torch.cuda.is_available() else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


# ---------------------------------------------------------------------------
# CPU arms (oracle = C restatement of the reference Fortran step)
# ---------------------------------------------------------------------------
def cpu_build():
    """The host-native timing build of the oracle: (library, its flags, CPU model)."""
    from oracle import oracle as O
    lib = O.load(timing=True)
    return lib, lib.build_flags, lib.cpu_model


def cpu_rate(prob, q, run, omp, max_seconds=15.0, max_steps=None):
    """Time whole-grid oracle steps (BC fill + step + dt control) on the host
    with the oracle's host-native timing build (-O3 -march=native, FMA
    allowed); returns (cell-updates/s, steps timed, threads, seconds)."""
    from oracle import oracle as O
    lib, _, _ = cpu_build()
    qbc = O.new_qbc(prob, q)
    ctrl = O.control_init(0.0, run['dt_initial'], 1e9, run['cfl_max'], run['cfl_desired'], lib=O.load())
    threads = lib.orc_num_threads() if omp else 1
    cells = prob.mx * prob.my
    steps = 0
    accepted0 = ctrl.numsteps
    t0 = time.perf_counter()
    while True:
        ctrl.done = 0
        ctrl.error = 0
        ctrl.max_steps = ctrl.iter + 1
        rc = O.evolve(prob, qbc, None, ctrl, omp=omp, lib=lib)
        if rc not in (0, 5):
            raise RuntimeError("oracle evolve failed: %d" % rc)
        steps += 1
        el = time.perf_counter() - t0
        if el >= max_seconds or (max_steps is not None and steps >= max_steps):
            break
    accepted = ctrl.numsteps - accepted0
    return accepted * cells / el, steps, threads, el


def run_reference_arm(args, world, rank):
    """--impl reference: the oracle (OpenMP gather form, all host threads)."""
    if rank != 0:
        return
    prob, q, aux, run, tfinal = shockbubble_config(split=args.split)
    from oracle import oracle as O
    lib, flags, model = cpu_build()
    qbc = O.new_qbc(prob, q)
    ctrl = O.control_init(0.0, run['dt_initial'], 1e9, run['cfl_max'], run['cfl_desired'], lib=O.load())
    threads = lib.orc_num_threads()
    cells = prob.mx * prob.my

    def one_step():
        ctrl.done = 0
        ctrl.error = 0
        ctrl.max_steps = ctrl.iter + 1
        rc = O.evolve(prob, qbc, None, ctrl, omp=True, lib=lib)
        if rc not in (0, 5):
            raise RuntimeError("oracle evolve failed: %d" % rc)

    for _ in range(args.warmup):
        one_step()
    a0 = ctrl.numsteps
    t0 = time.perf_counter()
    for _ in range(args.steps):
        one_step()
    el = time.perf_counter() - t0
    acc = ctrl.numsteps - a0
    value = acc * cells / el
    line = {
        "impl": "reference", "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": el / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "euler_shockbubble_1280x320", "mx": prob.mx, "my": prob.my,
                   "solver": "euler_roe_efix_4wave", "limiter": "MC", "transverse_waves": -1 if args.split else 2,
                       "mode": "dimensional splitting" if args.split else "unsplit"},
        "cpu_baseline": {"value": value, "unit": "cell-updates/s", "cores": threads, "kind": "port",
                         "sample": "%d whole-grid steps (BC fill + step + dt control) of the 1280x320 "
                                   "shock bubble, oracle OpenMP gather form, %d threads" % (args.steps, threads),
                         "build": flags, "cpu_model": model, "nproc": os.cpu_count()},
        "e2e": {"value": value, "unit": "cell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_ours(args, world, rank, local):
    import torch
    import pyclaw_b200 as pc
    from pyclaw_b200 import _abi, _lib
    from pyclaw_b200.device import DeviceState

    lib = _lib.load()
    prob, q, aux, run, tfinal = shockbubble_config(split=args.split)
    cells = prob.mx * prob.my
    c = _abi.Control()
    _lib.check(lib.claw2_control_init(ctypes.byref(c), 0.0, run['dt_initial'], 1e9, run['cfl_max'],
                                      run['cfl_desired'], 1e99, 1, 0, 1 << 40, run['cfl_desired']),
               "claw2_control_init")
    if world == 1:
        dev = DeviceState(prob, torch.device("cuda", local))
        dev.upload_q(q)

        def advance(n):
            _lib.check(lib.claw2_advance(ctypes.byref(prob), dev.ptr(dev.q[0]), dev.ptr(dev.q[1]),
                                         dev.ptr(dev.aux), dev.ptr(dev.ctrl), dev.ptr(dev.scratch), int(n),
                                         dev.stream), "claw2_advance")
    else:
        # weak scaling by domain decomposition: one grid of 1280 x (320 N)
        # cells (the shock-bubble setup stacked N times along y), one slab of
        # 1280 x 320 per rank; every step exchanges two halo rows with the
        # neighbours (NCCL) and takes the max of the CFL numbers over ranks
        from pyclaw_b200 import decomp
        gp = _abi.Problem.from_buffer_copy(prob)
        gp.my = prob.my * world
        slab = decomp.Slab(gp, world, rank, torch.device("cuda", local))
        slab.upload(np.concatenate([q] * world, axis=2))
        dev = slab.dev
        transport = decomp.DistTransport(slab)

        def advance(n):
            for _ in range(int(n)):
                decomp.step_all([slab], transport)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    host = _abi.Control.from_address(dev.ctrl_host.data_ptr())
    ctypes.memmove(ctypes.addressof(host), ctypes.addressof(c), ctypes.sizeof(c))
    dev.ctrl.copy_(dev.ctrl_host)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device="cuda")   # 256 MB > L2
    _barrier(world)
    # set-up: run the flow on to a developed state (the shock through the
    # bubble), so that the timed steps see the run's mix of shocked, smooth and
    # still cells rather than the first steps from t = 0
    if args.develop > 0:
        advance(args.develop)
        torch.cuda.synchronize()
    dev.ctrl_host.copy_(dev.ctrl)
    torch.cuda.synchronize()
    t_timed0 = host.t
    dt_timed0 = host.dt
    # the e2e legs start from the same developed state (one grid: rank 0's)
    q_timed0 = dev.download_q() if world == 1 else q

    for _ in range(max(3, args.warmup)):
        flush.fill_(1.0)
        advance(1)
    torch.cuda.synchronize()
    dev.ctrl_host.copy_(dev.ctrl)
    n0 = host.numsteps
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clocks = ClockSampler(torch.cuda.current_device()) if rank == 0 or world > 1 else None
    if clocks:
        clocks.start()
        time.sleep(0.3)                       # let the sampler start before the timed region
    _barrier(world)
    torch.cuda.synchronize()
    w0 = time.perf_counter()
    for k in range(args.steps):
        flush.fill_(float(k))                 # evict the state from L2 (not timed)
        ev[k][0].record(stream)
        advance(1)
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    _barrier(world)
    wall = time.perf_counter() - w0
    clk = clocks.stop() if clocks else None
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_dev = sum(step_ms) / 1e3
    dev.ctrl_host.copy_(dev.ctrl)
    torch.cuda.synchronize()
    accepted = host.numsteps - n0
    if host.error:
        raise RuntimeError("device loop error %d" % host.error)
    t_max = _max_over_ranks(t_dev, world)
    total_updates = _sum_over_ranks(float(accepted * cells), world)
    value = total_updates / t_max

    # ---- roofline of the step kernel ----------------------------------------
    peak, peak_kind = _peaks()
    alg_bytes = 8 * (2 * prob.num_eqn + prob.num_aux) * cells   # per launch (one step)
    avg_kernel_s = t_dev / args.steps
    achieved = alg_bytes / avg_kernel_s / 1e9
    rec = _ncu_record("step_kernel_split_euler1280x320" if args.split else "lean_step_kernel_euler1280x320")
    traffic = (rec["dram_bytes_read"] + rec["dram_bytes_write"]) if rec else None
    # FP64 pipe: the step's real bound (about 1,900 FP64 instructions per cell,
    # IEEE divisions and square roots, no FMA contraction): lane-slots of the
    # FP64 pipe used per launch (ncu warp instructions x 32) per second, against
    # SMs x 64 FP64 lanes x the SM clock
    fp64 = None
    if rec and rec.get("fp64_pipe_warp_inst"):
        nsm = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        f_mhz = (clk or {}).get("sm_max_mhz") or 1965.0
        lanes = 32.0 * rec["fp64_pipe_warp_inst"]
        fp64 = {"achieved": lanes / avg_kernel_s / 1e12, "peak": nsm * 64 * f_mhz * 1e6 / 1e12,
                "unit": "T FP64 lane-ops/s", "frac": None,
                "fp64_lane_ops_per_launch": lanes, "fp64_lane_ops_per_cell": lanes / cells,
                "source": "ncu smsp__inst_executed_pipe_fp64.sum x 32 of one launch (%s); peak = %d SMs x 64 "
                          "FP64 lanes x %.0f MHz" % (rec.get("capture", "profiles/ncu_metrics.json"), nsm, f_mhz)}
        fp64["frac"] = fp64["achieved"] / fp64["peak"]

    # ---- e2e through the host-buffer C ABI (claw2_session_evolve) ----------
    e2e = e2e_s2 = None
    if rank == 0 or world > 1:
        t_e, dt_e = (t_timed0, dt_timed0) if world == 1 else (0.0, None)
        e2e = _e2e(lib, prob, q_timed0, run, args, t_e, dt_e)
        e2e_s2 = _e2e_step2(lib, prob, q_timed0, run, args, dt_e)
    e2e_val = _sum_over_ranks(e2e["value"], world) if e2e else None
    e2e_s2_val = _sum_over_ranks(e2e_s2["value"], world) if e2e_s2 else None

    # ---- CPU baseline (oracle, all host threads; bounded sample) ---------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rate, n, thr, el = cpu_rate(prob, q, run, omp=True, max_seconds=12.0)
        rate1, n1, _, el1 = cpu_rate(prob, q, run, omp=False, max_seconds=8.0)
        _, flags, model = cpu_build()
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": thr, "kind": "port",
               "sample": "%d whole-grid steps (%.1f s) of the 1280x320 shock bubble from t = 0 through the "
                         "oracle's OpenMP gather form on %d threads; serial: %.4g cell-updates/s over %d steps"
                         % (n, el, thr, rate1, n1),
               "serial_value": rate1, "build": flags, "cpu_model": model, "nproc": os.cpu_count()}

    if rank == 0:
        line = {
            "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "euler_shockbubble_1280x320", "mx": prob.mx, "my": prob.my,
                       "solver": "euler_roe_efix_4wave", "limiter": "MC", "transverse_waves": -1 if args.split else 2,
                       "mode": "dimensional splitting" if args.split else "unsplit",
                       "parallelism": ("domain decomposition: %d slabs of 1280x320 along y of one 1280x%d grid, "
                                       "NCCL halo exchange + CFL max all-reduce per step" % (world, 320 * world))
                       if world > 1 else "single",
                       "l2": "flushed (256 MB write) before every timed step",
                       "develop_steps": int(args.develop), "t_first_timed_step": t_timed0,
                       "accepted_steps": int(accepted)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic,
                         "traffic_note": "dram read+write of one cold ncu launch; most of the 13 MB of results "
                                         "stay resident in L2 during the launch" if traffic else None,
                         "peak_source": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes,
                         "fp64": fp64},
            "cpu_baseline": cpu,
            # one call = one output interval of Controller.run: the state goes up
            # once, the steps of the interval run on the device, the state comes back
            "e2e": {"value": e2e_val, "unit": "cell-updates/s",
                    "h2d_bytes_per_step": e2e["h2d"] / e2e["steps"], "d2h_bytes_per_step": e2e["d2h"] / e2e["steps"],
                    "h2d_bytes_per_call": e2e["h2d"], "d2h_bytes_per_call": e2e["d2h"],
                    "steps_per_call": e2e["steps"], "calls": e2e["calls"],
                    "api": "claw2_session_evolve (one Controller.run output interval per call; the steps of a "
                           "call run back to back, L2 not flushed)",
                    "start": "the developed state of the timed steps (t = %.4f), uploaded from pinned host memory"
                             % t_timed0 if world == 1 else "t = 0",
                    "per_step_f2py_contract": {
                        "value": e2e_s2_val, "unit": "cell-updates/s", "api": "claw2_session_step2",
                        "h2d_bytes_per_step": e2e_s2["h2d"], "d2h_bytes_per_step": e2e_s2["d2h"],
                        "steps": e2e_s2["steps"]} if e2e_s2 else None} if e2e else None,
            "gpu_launches": int(args.steps),
            "clocks": clk,
            "wall_s": wall,
        }
        if world == 1 and not args.headline_only:
            # the metric's other parts, each measured in its own timed region
            # with its own clock record: the batched form and the adjoint
            # against the plain step, and configs 1 and 3
            line["workloads"] = {}
            for name, fn in (("batched", run_batched), ("adjoint", run_adjoint), ("shallow", run_shallow),
                             ("acoustics", run_acoustics)):
                try:
                    line["workloads"][name] = fn(args)
                except Exception as e:          # one failing part must not cost the headline line
                    line["workloads"][name] = {"error": "%s: %s" % (type(e).__name__, e)}
                torch.cuda.empty_cache()
        print(json.dumps(line), flush=True)


def _e2e(lib, prob, q, run, args, t_start=0.0, dt_start=None):
    """claw2_session_evolve from pinned host buffers: each call uploads the
    state, advances it by a fixed simulated interval with on-device dt
    control, and downloads it again.  q is the state at t_start (dt_start:
    the controller's dt there)."""
    import torch
    s = ctypes.c_void_p()
    from pyclaw_b200 import _lib
    _lib.check(lib.claw2_session_create(ctypes.byref(prob), ctypes.byref(s)), "claw2_session_create")
    try:
        host = torch.from_numpy(np.asfortranarray(q).ravel(order='K')).clone().pin_memory()
        hq = host.numpy()
        t = ctypes.c_double(t_start)
        dt = ctypes.c_double(dt_start if dt_start else run['dt_initial'])
        status = (ctypes.c_double * 5)()
        interval = 40 * run['dt_initial']
        def call():
            return lib.claw2_session_evolve(s, hq.ctypes.data, None, ctypes.byref(t), ctypes.byref(dt),
                                            t.value + interval, run['cfl_max'], run['cfl_desired'], 1e99,
                                            100000, status)
        _lib.check(call(), "claw2_session_evolve")     # warm-up
        calls = max(2, min(args.steps, 8))
        steps = 0
        t0 = time.perf_counter()
        for _ in range(calls):
            _lib.check(call(), "claw2_session_evolve")
            steps += int(status[3])
        el = time.perf_counter() - t0
        nbytes = 8 * prob.num_eqn * prob.mx * prob.my
        return {"value": steps * prob.mx * prob.my / el, "h2d": nbytes, "d2h": nbytes,
                "steps": steps / calls, "calls": calls}
    finally:
        lib.claw2_session_destroy(s)


def _ghosted(prob, q):
    """q with two ghost layers filled as Solver.apply_q_bcs does
    (src/pyclaw/solver.py:368-434): x sides over all rows, then y sides over
    all columns; extrapolation copies the edge cell, a wall mirrors and negates
    the normal momentum.  Only the extrapolation and wall sides of the
    shock-bubble workload are needed here."""
    g = 2
    qbc = np.zeros((q.shape[0], q.shape[1] + 2 * g, q.shape[2] + 2 * g), order='F')
    qbc[:, g:-g, g:-g] = q
    for axis in (0, 1):
        for side, bc in ((0, int(prob.bc_lower[axis])), (1, int(prob.bc_upper[axis]))):
            n = q.shape[1 + axis]
            for k in range(g):
                dst = g - 1 - k if side == 0 else n + g + k
                if bc == 1:                                   # extrapolation
                    src = g if side == 0 else n + g - 1
                elif bc == 3:                                 # wall
                    src = g + k if side == 0 else n + g - 1 - k
                else:
                    raise ValueError("only extrapolation and wall sides here")
                a = qbc[:, dst, :] if axis == 0 else qbc[:, :, dst]
                a[...] = qbc[:, src, :] if axis == 0 else qbc[:, :, src]
                if bc == 3:
                    a[1 + axis] = -a[1 + axis]
    return qbc


def _e2e_step2(lib, prob, q, run, args, dt_step=None):
    """claw2_session_step2, the per-step f2py contract of step2: every call
    copies the ghosted state in the reference's layout from pinned host
    memory, converts it, takes one step, converts back and copies the result
    and the CFL number to the host."""
    import torch
    from pyclaw_b200 import _lib
    s = ctypes.c_void_p()
    _lib.check(lib.claw2_session_create(ctypes.byref(prob), ctypes.byref(s)), "claw2_session_create")
    try:
        qbc = _ghosted(prob, q)
        bufs = [torch.from_numpy(qbc.ravel(order='F')).clone().pin_memory() for _ in range(2)]
        arrs = [b.numpy() for b in bufs]
        cfl = ctypes.c_double()
        dt = dt_step if dt_step else run['dt_initial']

        def call(k):
            return lib.claw2_session_step2(s, arrs[k & 1].ctypes.data, arrs[(k + 1) & 1].ctypes.data, None, dt,
                                           ctypes.byref(cfl))
        for k in range(2):
            _lib.check(call(k), "claw2_session_step2")      # warm-up
        n = max(4, min(args.steps, 40))
        t0 = time.perf_counter()
        for k in range(n):
            _lib.check(call(k), "claw2_session_step2")
        el = time.perf_counter() - t0
        nbytes = 8 * prob.num_eqn * (prob.mx + 4) * (prob.my + 4)
        return {"value": n * prob.mx * prob.my / el, "h2d": nbytes, "d2h": nbytes + 8, "steps": n}
    finally:
        lib.claw2_session_destroy(s)


def run_batched(args):
    """Config 4: 1024 uneven vc-acoustics instances, 300 controlled steps each:
    the batched persistent kernel (autotuned, CUDA graph) against looping the
    plain device step over the same instances one at a time."""
    import torch
    from pyclaw_b200 import _abi, _lib
    from pyclaw_b200.batch import BatchSolver
    from pyclaw_b200.device import DeviceState
    nsteps = 300
    prob, insts = batched_vc_config(n=args.instances)
    cells = [i["q"].shape[1] * i["q"].shape[2] for i in insts]
    bs = BatchSolver(prob, insts)
    tuning = bs.autotune(steps=3, repeats=2)
    bs.init_controls([i["dt"] for i in insts], max_steps=nsteps)
    bs.advance_graph(0)
    torch.cuda.synchronize()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    bs.advance_graph(nsteps, chunk=50)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_batch = e0.elapsed_time(e1) / 1e3
    ctrls = bs.controls()
    if not all(c.done for c in ctrls):
        raise RuntimeError("batched run did not finish every instance")
    upd_batch = sum(c.numsteps * n for c, n in zip(ctrls, cells))
    # looped plain step: each instance alone through the device-controlled loop
    lib = _lib.load()
    t_loop = 0.0
    t_loop_dev = 0.0
    upd_loop = 0
    check = {0, len(insts) // 2, len(insts) - 1}
    same = True
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    for k, inst in enumerate(insts):
        pk = bs.problems[k]
        dev = DeviceState(pk)
        dev.upload_aux(inst["aux"])
        dev.upload_q(inst["q"])
        c = _abi.Control()
        lib.claw2_control_init(ctypes.byref(c), 0.0, inst["dt"], 1e300, 1.0, 0.9, 1e99, 1, 0, nsteps, 0.9)
        torch.cuda.synchronize()
        d0, d1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        w0 = time.perf_counter()
        d0.record()
        out = dev.evolve(c)
        d1.record()
        t_loop += time.perf_counter() - w0
        torch.cuda.synchronize()
        t_loop_dev += d0.elapsed_time(d1) / 1e3
        upd_loop += out.numsteps * cells[k]
        if k in check:
            same = same and bool(np.array_equal(dev.download_q(), bs.solution(k)))
        del dev
    clk_loop = clocks.stop()
    line = {
        "metric": "cell_updates_per_s", "value": upd_batch / t_batch, "unit": "cell-updates/s", "n_gpus": 1,
        "steps": nsteps, "higher_is_better": True, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batched_vc_acoustics_%d" % len(insts), "sizes": "nx,ny ~ U{64..384}",
                   "cells_total": int(sum(cells)), "tiles": bs.ntiles, "autotune": tuning},
        "batched_seconds": t_batch, "looped_seconds": t_loop,
        "looped_value": upd_loop / t_loop, "speedup_vs_looped_plain_step": (upd_batch / t_batch) / (upd_loop / t_loop),
        "timing": "batched: CUDA events around the graph replays; looped: host wall time of each instance's "
                  "device-controlled loop (launches, controller polls), its device time beside it",
        "looped_device_seconds": t_loop_dev,
        "speedup_vs_looped_device_time": (upd_batch / t_batch) / (upd_loop / t_loop_dev),
        "spot_check_bit_identical": same,
        "clocks": clk, "clocks_looped": clk_loop,
    }
    bs.close()
    return line


def run_batched_sharded(args, world, rank):
    """Config 4 on N GPUs: the 1024 instances split across the ranks by
    pyclaw_b200.partition (whole instances, balanced by tile count); each rank
    steps its share with its own batched kernel and CUDA graphs, with no
    exchange while stepping; the final states are gathered on rank 0 once,
    after the timed region.  Strong scaling: the batch is the same at every N."""
    import torch
    from pyclaw_b200 import partition
    nsteps = 300
    prob, insts = batched_vc_config(n=args.instances)
    sb = partition.ShardedBatch(prob, insts, rank, world)
    tuning = sb.autotune(steps=3, repeats=2)
    sb.init_controls([i["dt"] for i in insts], max_steps=nsteps)
    torch.cuda.synchronize()
    _barrier(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sb.advance_graph(nsteps, chunk=50)
    e1.record()
    torch.cuda.synchronize()
    _barrier(world)
    t_local = e0.elapsed_time(e1) / 1e3
    res = sb.local_results()
    upd_local = sum(ns * q.shape[1] * q.shape[2] for _, q, ns, _ in res)
    t_max = _max_over_ranks(t_local, world)
    upd = _sum_over_ranks(float(upd_local), world)
    tiles = [None] * world if rank == 0 else None
    import torch.distributed as dist
    dist.gather_object(sb.tiles, tiles, dst=0)
    out = sb.gather(dst=0)
    if rank == 0:
        states, steps, _ = out
        if min(steps) != nsteps:
            raise RuntimeError("sharded batched run did not finish every instance")
        line = {
            "metric": "cell_updates_per_s", "value": upd / t_max, "unit": "cell-updates/s", "n_gpus": world,
            "steps": nsteps, "ms_per_step": t_max / nsteps * 1e3, "higher_is_better": True, "scaling": "strong",
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": "batched_vc_acoustics_%d" % len(insts), "sizes": "nx,ny ~ U{64..384}",
                       "parallelism": "instances partitioned across %d ranks (tile-balanced), no exchange "
                                      "while stepping, one gather at the end" % world,
                       "tiles_per_rank": tiles, "autotune_rank0": tuning},
            "batched_seconds": t_max,
        }
        print(json.dumps(line), flush=True)
    sb.close()


def run_shallow(args):
    """The 4096^2 shallow-water dam break: 500 controlled steps through the
    device loop (claw2_advance), one CUDA-event pair around the whole run; the
    state (403 MB per buffer) does not fit in L2, so nothing is flushed."""
    import torch
    from pyclaw_b200 import _abi, _lib
    from pyclaw_b200.device import DeviceState
    lib = _lib.load()
    nsteps = args.sw_steps
    prob, q, run = shallow_config(args.sw_n)
    cells = prob.mx * prob.my
    dev = DeviceState(prob, torch.device("cuda"))
    host = _abi.Control.from_address(dev.ctrl_host.data_ptr())

    def reset(max_steps):
        dev.upload_q(q)
        c = _abi.Control()
        _lib.check(lib.claw2_control_init(ctypes.byref(c), 0.0, run["dt_initial"], 1e9, run["cfl_max"],
                                          run["cfl_desired"], 1e99, 1, 0, int(max_steps), run["cfl_desired"]),
                   "claw2_control_init")
        ctypes.memmove(ctypes.addressof(host), ctypes.addressof(c), ctypes.sizeof(c))
        dev.ctrl.copy_(dev.ctrl_host)
        torch.cuda.synchronize()

    def advance(n):
        _lib.check(lib.claw2_advance(ctypes.byref(prob), dev.ptr(dev.q[0]), dev.ptr(dev.q[1]), dev.ptr(dev.aux),
                                     dev.ptr(dev.ctrl), dev.ptr(dev.scratch), int(n), dev.stream), "claw2_advance")

    reset(max(3, args.warmup))
    advance(max(3, args.warmup))
    reset(nsteps)
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    advance(nsteps)
    e1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    t = e0.elapsed_time(e1) / 1e3
    dev.ctrl_host.copy_(dev.ctrl)
    torch.cuda.synchronize()
    # a fixed step count ends with the controller's max-steps status (the
    # reference's "Maximum number of timesteps have been taken")
    if host.error not in (0, _abi.ERR_MAX_STEPS) or host.iter != nsteps:
        raise RuntimeError("device loop error %d after %d steps" % (host.error, host.iter))
    acc = host.numsteps
    value = acc * cells / t
    peak, peak_kind = _peaks()
    alg = 8 * 2 * prob.num_eqn * cells
    achieved = alg / (t / nsteps) / 1e9
    cpu = None
    if not args.no_cpu:
        rate, n, thr, el = cpu_rate(prob, q, run, omp=True, max_seconds=10.0)
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": thr, "kind": "port",
               "sample": "%d whole-grid steps (%.1f s) of the 4096^2 dam break, oracle OpenMP gather form, "
                         "%d threads" % (n, el, thr)}
    line = {
        "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s", "n_gpus": 1,
        "steps": nsteps, "ms_per_step": t / nsteps * 1e3, "higher_is_better": True, "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "shallow_water_dam_break_%dx%d" % (prob.mx, prob.my), "solver": "shallow_roe_efix",
                   "limiter": "superbee", "transverse_waves": 2, "accepted_steps": int(acc),
                   "t_final": host.t, "l2": "state (%d MB per buffer) larger than L2" % (8 * 3 * cells >> 20)},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind},
        "clocks": clk, "cpu_baseline": cpu,
    }
    return line


def run_acoustics(args):
    """Config 1: 256^2 constant-coefficient acoustics (walls, unsplit with
    transverse_waves=2, MC, cfl_desired 0.9) from t = 0 to 0.6 through the
    device-controlled loop (one launch per step, the light tile body); the
    whole run is timed with CUDA events, the oracle's OpenMP form times the
    same run on the host cores."""
    import torch
    from pyclaw_b200 import _abi, _lib
    from pyclaw_b200.device import DeviceState
    lib = _lib.load()
    prob, q, aux, run, tfinal = acoustics_config()
    cells = prob.mx * prob.my
    dev = DeviceState(prob, torch.device("cuda"))

    def once():
        dev.upload_q(q)
        dev.cur = 0
        c = _abi.Control()
        _lib.check(lib.claw2_control_init(ctypes.byref(c), 0.0, run["dt_initial"], tfinal, run["cfl_max"],
                                          run["cfl_desired"], 1e99, 1, 0, 1 << 40, run["cfl_desired"]),
                   "claw2_control_init")
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = dev.evolve(c)
        e1.record()
        torch.cuda.synchronize()
        return out, e0.elapsed_time(e1) / 1e3

    for _ in range(max(1, args.warmup // 3)):
        once()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    out, t = once()
    clk = clocks.stop()
    if out.error:
        raise RuntimeError("device loop error %d" % out.error)
    value = out.numsteps * cells / t
    cpu = None
    if not args.no_cpu:
        rate, n, thr, el = cpu_rate(prob, q, run, omp=True, max_seconds=8.0)
        cpu = {"value": rate, "unit": "cell-updates/s", "cores": thr, "kind": "port",
               "sample": "%d whole-grid steps (%.1f s) of the 256^2 acoustics run, oracle OpenMP gather form, "
                         "%d threads" % (n, el, thr)}
    line = {
        "metric": "cell_updates_per_s", "value": value, "unit": "cell-updates/s", "n_gpus": 1,
        "steps": int(out.numsteps), "ms_per_step": t / out.numsteps * 1e3, "higher_is_better": True,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "acoustics_256x256_walls_t0.6", "solver": "acoustics", "limiter": "MC",
                   "transverse_waves": 2, "t_final": out.t, "run_seconds": t,
                   "timing": "whole run to t=0.6 incl. the host polling of the controller every batch of steps"},
        "cpu_baseline": cpu, "clocks": clk,
    }
    return line


def run_adjoint(args):
    """The adjoint workload: traces of `shots` shots over `nsteps` steps for the
    starting material, the L2 misfit against the target material's traces,
    and its gradient with respect to per-cell (rho, K) and the initial state
    through the hand-written adjoint (checkpoint every 20 steps).  Times the
    plain forward, the taped forward and the backward with CUDA events."""
    import torch
    from pyclaw_b200.adjoint import AcousticShots, material_aux, shots_traces
    cfg = adjoint_config(n=args.adj_n, shots=args.adj_shots, nsteps=args.adj_steps)
    n, S = cfg["n"], cfg["shots"]
    dev = torch.device("cuda")
    r = AcousticShots(n, n, cfg["dx"], cfg["dy"], S, cfg["src"], cfg["rec"], cfg["wav"], cfg["dt"],
                      bc_lower=(1, 1), bc_upper=(1, 3), aux_bc_lower=(1, 1), aux_bc_upper=(1, 1),
                      order=2, transverse=2, limiters=(4, 4), checkpoint=("uniform", 20))
    t64 = dict(dtype=torch.float64, device=dev)
    q0 = torch.zeros((S, 3, n, n), **t64)
    with torch.no_grad():
        target = shots_traces(q0, material_aux(torch.tensor(cfg["rho_t"], **t64), torch.tensor(cfg["K_t"], **t64)),
                              r).clone()
    rho = torch.tensor(cfg["rho0"], **t64).requires_grad_(True)
    K = torch.tensor(cfg["K0"], **t64).requires_grad_(True)
    p0 = torch.zeros((n, n), **t64).requires_grad_(True)
    z = torch.zeros((n, n), **t64)

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def once():
        q = torch.stack([torch.stack([p0, z, z])] * S)
        e0, e1, e2 = ev(), ev(), ev()
        e0.record()
        tr = shots_traces(q, material_aux(rho, K), r)
        loss = 0.5 * ((tr - target) ** 2).sum()
        e1.record()
        loss.backward()
        e2.record()
        torch.cuda.synchronize()
        return loss.item(), e0.elapsed_time(e1) / 1e3, e1.elapsed_time(e2) / 1e3

    def plain_forward():
        e0, e1 = ev(), ev()
        st, nx_ = r.new_states(1)[0], r.new_states(1)[0]
        with torch.no_grad():
            r.set_aux(material_aux(rho, K))
            r.set_state(st, torch.stack([torch.stack([p0, z, z])] * S))
        torch.cuda.synchronize()
        e0.record()
        r.advance(st, nx_, 0, cfg["nsteps"])
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3

    for _ in range(max(1, args.warmup // 3)):
        once()
        for x in (rho, K, p0):
            x.grad = None
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    time.sleep(0.3)
    t_plain = min(plain_forward() for _ in range(2))
    loss, t_fwd, t_bwd = once()
    clk = clocks.stop()
    g_rho, g_K, g_p0 = (x.grad for x in (rho, K, p0))
    cells = n * n * S * cfg["nsteps"]
    line = {
        "metric": "adjoint_gradient_cost_over_forward", "value": (t_fwd + t_bwd) / t_plain, "unit": "x",
        "n_gpus": 1, "steps": cfg["nsteps"], "higher_is_better": False, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "vc_acoustics_adjoint_%dx%d_%dshots_%dsteps" % (n, n, S, cfg["nsteps"]),
                   "receivers": len(cfg["rec"]), "checkpoint": "uniform every 20 steps",
                   "inclusions": "3 circles of radius 0.3"},
        "forward_seconds": t_plain, "taped_forward_seconds": t_fwd, "backward_seconds": t_bwd,
        "backward_over_forward": t_bwd / t_plain,
        "forward_cell_updates_per_s": cells / t_plain,
        "loss": loss,
        "grad_norms": {"rho": float(g_rho.norm()), "K": float(g_K.norm()), "p0": float(g_p0.norm())},
        "grad_finite": bool(torch.isfinite(g_rho).all() and torch.isfinite(g_K).all() and torch.isfinite(g_p0).all()),
        "clocks": clk,
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--headline-only", action="store_true",
                    help="only the shock-bubble line, without the batched / adjoint / shallow / acoustics parts")
    ap.add_argument("--develop", type=int, default=1500,
                    help="untimed steps of set-up before the warm-up (shock bubble)")
    ap.add_argument("--split", action="store_true",
                    help="shock bubble with dimensional splitting (the reference's default mode)")
    ap.add_argument("--workload", default="shockbubble", choices=["shockbubble", "batched", "adjoint", "shallow", "acoustics"])
    ap.add_argument("--sw-n", type=int, default=4096)
    ap.add_argument("--sw-steps", type=int, default=500)
    ap.add_argument("--instances", type=int, default=1024)
    ap.add_argument("--adj-n", type=int, default=512)
    ap.add_argument("--adj-shots", type=int, default=64)
    ap.add_argument("--adj-steps", type=int, default=400)
    args = ap.parse_args()
    world, rank, local = _dist_init()
    try:
        if args.workload == "batched":
            if world > 1:
                run_batched_sharded(args, world, rank)
            elif rank == 0:
                print(json.dumps(run_batched(args)), flush=True)
        elif args.workload == "adjoint":
            if rank == 0:
                print(json.dumps(run_adjoint(args)), flush=True)
        elif args.workload == "shallow":
            if rank == 0:
                print(json.dumps(run_shallow(args)), flush=True)
        elif args.workload == "acoustics":
            if rank == 0:
                print(json.dumps(run_acoustics(args)), flush=True)
        elif args.impl == "reference":
            run_reference_arm(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
