#!/usr/bin/env python
"""Benchmark: reacting cell-updates/s of JANC's per-step path on B200.

Workload (one "step" = one full time step of the whole grid): the 2D H2-air
detonation channel, 1024 x 256 cells over 0.2 m x 0.05 m, stoichiometric
H2:O2:N2 = 2:1:3.76 at 1 atm / 300 K, at rest; an ignition slab over x-columns
0..20 (2 % of 1024, rounded) at 30 atm and 3000 K with eight seeded Gaussian
temperature blobs of +-5 % (radius 2-6 cells, numpy default_rng(1)); slip
walls on all four sides; WENO5-JS + global Lax-Friedrichs splitting, SSP-RK3,
point-implicit chemistry of the 9-species / 19-reaction mechanism; CFL time
steps.  CFL is 0.05 for the channel and 0.1 for the rotating-detonation
workload: at larger CFL numbers the reference's own algorithm goes
non-finite (first-order point-implicit chemistry burns a slab-edge cell in
one step; tests/golden/config0_cfl05.npz records it for config 0 at CFL 0.5,
and the channel at CFL 0.1 fails between steps 20 and 50 in the float64 path
too), while at 0.05 it runs the full 2000 steps.  The work per step does not
depend on the CFL number.

Arms:
  default            our CUDA path, mixed precision (float32 flux arithmetic;
                     float64 state, temperature solve and chemistry) unless
                     --precision; device-timed with inputs resident (value)
                     and end to end through the public API from pinned host
                     buffers (e2e).  The float64 path is timed beside it and
                     the per-field relative L1 error of mixed against float64
                     after --accuracy-steps steps is reported.
  --impl reference   the reference algorithm's CPU implementation: the
                     NumPy oracle restating src/janc_v2 (JAX is not available
                     on the box), run as independent replicas on all host
                     cores
Batched ensemble (--workload ensemble, run with --steps 2000): 64 1D H2-air
detonation tubes of log-uniform length 1000-16000 cells (dx = 50 um), equivalence
ratio U(0.6, 1.4) and ignition temperature U(2500, 3500) K (numpy
default_rng(4)), ignition slab over the first 2 % of each tube at 30 atm,
reflective left / outflow right, CFL 0.1 per tube; one "step" advances every
tube one time step, all K steps run as ONE persistent kernel replayed from a
CUDA graph with the autotuned launch shape.  Compared with the 64 tubes run
one after another through the single-case float64 path, and the mixed result
is checked against those float64 runs per tube.

Adjoint (--workload adjoint, run with --steps 200): the 2D channel physics on
512 x 128 cells over 0.1 m x 0.025 m (slab = first 10 columns, 8 seeded blobs,
slip walls, CFL 0.05), float64; loss = sum over steps of dt times the mean
pressure over a 4 x 4 probe centred at x = 0.8 L, y = H / 2; gradients with
respect to the initial temperature field (65536 values) and the 19 ln A_i
through the hand-written adjoint, checkpointed every 20 steps.  The metric is
the time of the backward pass (recomputation included) over the time of the
forward pass; the gradients are checked against central finite differences
of the float64 forward (h = 1e-6 relative, 16 seeded unit directions each).

Block AMR (--workload amr): one refinement level of 64 x 16 blocks of 20 x 20
cells of the channel physics through the drop-in AMR_Simulator, with a
device block layer standing in for the external jaxamr package (also the
default line's configs.amr).

Multi-GPU: the path does not shard in this build (replicas only): each rank
advances its own copy of the workload; value = total cells x steps / max time.
"""
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

NX, NY = 1024, 256
LX, LY = 0.2, 0.05
SLAB = 21
CFL_BY_WORKLOAD = {"channel": 0.05, "rdc": 0.1}
CFL = CFL_BY_WORKLOAD["channel"]
METRIC = "reacting cell-updates/s"
UNIT = "cell-updates/s"
BYTES_CHEM_PER_CELL = 224      # read U,aux (112 B) + write U,aux (112 B), float64
BYTES_STEP_PER_CELL = 864 + 224  # fused-step minimum + separate chemistry pass (2D)
BYTES_FLUX_STAGE_PER_CELL = 288  # one RK stage of the fused minimum: (224 + 320 + 320) / 3
# DRAM bytes per cell measured with ncu (dram__bytes_read.sum + dram__bytes_write.sum,
# each launch cold) on the 1024x256 channel, mixed precision, with this tree's
# kernels: one RK stage 2/3 (k_sweep_x 27.35 + 0.00 MB, k_flux_y_rk 67.43 +
# 5.98 MB) and one chemistry launch (27.38 + 3.46 MB); the capture and its
# command are in profiles/launches_channel1024x256_mixed.md.  Per cell-step of
# the persistent ensemble kernel: profiles/k_ensemble_64tubes.md.
TRAFFIC_PER_CELL = {"flux": 384.3, "chem": 117.6}
TRAFFIC_SOURCE = "profiles/launches_channel1024x256_mixed.md"
TRAFFIC_ENS_PER_CELL_STEP = 764.0


ENS_N, ENS_SEED, ENS_CFL = 64, 4, 0.1
# 1D step, float64, each pass reading its inputs once and writing its outputs
# once (fields: 11 conserved, aux gamma and T, 6 Halley iterates).  fp64
# (global stop): stage 1 (12 in, 17 out), select 1 (12 in, 2 out), stages 2
# and 3 (23 in, 17 out), select 2 (14), chemistry (12 in, 17 out), select 4
# (14) -> 180 doubles.  mixed (per-cell solves, no select passes): stage 1
# (12 in, 13 out), stages 2 and 3 (23 in, 13 out), chemistry (12 in, 13 out)
# -> 122 doubles.
BYTES_ENS_STEP_PER_CELL = {"fp64": 1440, "mixed": 976}

RDC_NX, RDC_NY = 1600, 1000
RDC_ND = {"P0": 10 * 101325, "T0": 300, "R0": 369, "x0": 0.08}


def rdc_fields(nx=RDC_NX, ny=RDC_NY):
    """Rotating-detonation annulus (unrolled), nondimensional with the
    injection-manifold scales of the reference's example 2: ambient air at
    1 atm / 300 K; a fresh stoichiometric layer whose height falls linearly
    from 360 cells at x = 0 to 0 at x = nx/2; a 40 x 100-cell kernel at the
    bottom-left at 3000 K / 30 atm inside the layer.  Returns (P, T, Y, Yinj)."""
    import numpy as np
    P0, T0 = RDC_ND["P0"], RDC_ND["T0"]
    yH2 = (1.0 / 8 * 0.232) / (1 + 1.0 / 8 * 0.232)
    yO2 = 0.232 / (1 + 1.0 / 8 * 0.232)
    Yenv = np.array([0, 0.232, 0, 0, 0, 0, 0, 0.0])
    Yfill = np.array([yH2, yO2, 0, 0, 0, 0, 0, 0.0])
    Yinj = np.concatenate([[yH2, yO2], 1e-20 * np.ones(6)])
    x = np.arange(nx)[:, None]
    y = np.arange(ny)[None, :]
    height = np.maximum(0.0, 360.0 * (1.0 - x / (nx / 2)))
    fresh = (y < height)
    Y = np.where(fresh[None], Yfill[:, None, None], Yenv[:, None, None])
    P = np.full((1, nx, ny), 101325.0 / P0)
    T = np.full((1, nx, ny), 300.0 / T0)
    P[0, :40, :100] = 30 * 101325.0 / P0
    T[0, :40, :100] = 3000.0 / T0
    return np.ascontiguousarray(P), np.ascontiguousarray(T), np.ascontiguousarray(Y), Yinj


def c1_fields(nx=NX, ny=NY, slab=SLAB, seed=1):
    """(P, T, Y) of the channel workload as float64 numpy arrays."""
    import numpy as np
    from janc_b200 import mechanism as jm
    mech = jm.load()
    rng = np.random.default_rng(seed)
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    Y = np.ascontiguousarray(np.tile(jm.stoichiometric_Y(mech, 1.0)[:, None, None], (1, nx, ny)))
    xs = np.arange(slab)[:, None]
    ys = np.arange(ny)[None, :]
    bump = np.zeros((slab, ny))
    for _ in range(8):
        a = rng.uniform(-0.05, 0.05)
        sig = rng.uniform(2.0, 6.0)
        cx = rng.uniform(0, slab)
        cy = rng.uniform(0, ny)
        bump += a * np.exp(-((xs - cx) ** 2 + (ys - cy) ** 2) / (2 * sig ** 2))
    P[0, :slab] = 30 * 101325.0
    T[0, :slab] = 3000.0 * (1 + bump)
    return P, T, Y


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=5.0):
        """Wait until the sampler has reported once (nvidia-smi's start-up,
        whose driver queries can delay kernel launches, is then over)."""
        t0 = time.time()
        while self.proc is not None and not self.lines and time.time() - t0 < timeout:
            time.sleep(0.02)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return None, 0, 1
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    lr = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(lr)
    dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    return dist, dist.get_rank(), ws


def max_over_ranks(dist, x, device="cuda"):
    """Largest value of x over all ranks (a device-timed duration); x itself
    when not distributed.  Every rank must call it."""
    if not dist:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(world_size, cells_per_rank, steps, ms_max):
    """Whole-job throughput: all ranks' cell-updates over the slowest rank's
    device time (each rank advances its own replica)."""
    return world_size * cells_per_rank * steps / (ms_max * 1e-3)


def count_kernel_launches(fn):
    """Kernel launches of fn(), counted as the kernel nodes of a CUDA graph
    that captures it (driver API cuGraphGetNodes / cuGraphNodeGetType)."""
    import ctypes
    import torch
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        fn()  # warm-up on a side stream, as graph capture requires
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph(keep_graph=True)
    with torch.cuda.graph(g, capture_error_mode="relaxed"):
        fn()
    torch.cuda.synchronize()
    cu = ctypes.CDLL("libcuda.so.1")
    h = ctypes.c_void_p(g.raw_cuda_graph())
    n = ctypes.c_size_t(0)
    if cu.cuGraphGetNodes(h, None, ctypes.byref(n)) != 0:
        return None
    nodes = (ctypes.c_void_p * n.value)()
    cu.cuGraphGetNodes(h, nodes, ctypes.byref(n))
    kernels = 0
    for i in range(n.value):
        t = ctypes.c_int(-1)
        cu.cuGraphNodeGetType(ctypes.c_void_p(nodes[i]), ctypes.byref(t))
        kernels += t.value == 0  # CU_GRAPH_NODE_TYPE_KERNEL
    del g
    return kernels


def fp64_peak_tflops(L, torch):
    """Measured FP64 FMA throughput of this device (TFLOP/s)."""
    import ctypes
    props = torch.cuda.get_device_properties(torch.cuda.current_device())
    blocks = props.multi_processor_count * 8
    iters = 2000
    scratch = torch.empty(blocks, dtype=torch.float64, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    ptr = ctypes.c_void_p(scratch.data_ptr())
    for _ in range(2):
        L.jb_probe_fp64_fma(blocks, iters, ptr, st)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        L.jb_probe_fp64_fma(blocks, iters, ptr, st)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / 5
    flops = blocks * 256.0 * iters * 16 * 8 * 2
    return flops / (ms * 1e-3) / 1e12


def chem_flops_per_cell():
    """Algorithmic FP64 operations of one chemistry cell-update (+, -, x,
    FMA = 1 each; exp/log/pow/div/sqrt counted separately), from the
    mechanism's sparsity, as the kernel evaluates it."""
    import numpy as np
    from janc_b200 import mechanism as jm
    t = jm.load().tables
    vf, vb, tb = t["vf"], t["vb"], t["third_body"]
    nreac, nr = vf.shape
    ns = tb.shape[1]
    arith, special = 0, 0
    arith += 8 + ns * 2 + nr * 12 + 1   # fill_Y, X and clip, gibbs polynomials (h, s)
    special += nr + 1 + nr * 1          # log X, log T, h/T
    for i in range(nreac):
        arith += 2 + 2 * ns + 2 + 3 * 2 * nr + 4   # kf_i, third body, exponent sums, kb
        special += 5                               # pow, 3 exp, exp(-Ea/T), plus divisions below
        for k in range(nr):
            if vb[i, k] - vf[i, k] == 0:
                continue
            arith += 3
            for n in range(nr):
                if tb[i, n] != 0 or vf[i, n] != 0 or vb[i, n] != 0:
                    arith += 8
    arith += nr * nr + nr               # scale by M_k, A = I/dt - J
    arith += 2 * nr ** 3 // 3 + nr ** 2  # LU + substitution
    special += nr + nr                  # divisions by pivots, dY = x / rho
    arith += 4 * nr                     # clip and S
    arith += 5 * (3 * ns * 16)          # Halley iterates: 5 x thermo (cp, dcp, h over 9 species)
    return arith, special


def _setup_workload(args, precision):
    global CFL
    CFL = CFL_BY_WORKLOAD[args.workload]
    import torch
    from janc_b200.solver import Solver
    theta = None
    if args.workload == "channel":
        nx, ny = NX, NY
        dx, dy = LX / NX, LY / NY
        bc = {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
        visc = "on" if args.viscous else "off"
        fc = {"solver_type": "flux_splitting", "interface_reconstruction": args.recon, "split_method": args.flux,
              "viscosity": visc}
        if args.flux not in ("LF", "SW"):
            fc = {"solver_type": "godunov", "interface_reconstruction": args.recon,
                  "riemann_solver": args.flux, "viscosity": visc}
        tc = ({"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number", "Pr": 0.72,
               "species_diffusivity_model": "Lewis number", "Le": 1.0} if args.viscous else None)
        s = Solver(2, nx, ny, dx, dy, bc, precision=precision, flux_config=fc, transport_config=tc)
        P, T, Y = c1_fields()
        rname = "WENO5-JS" if args.recon == "WENO5_JS" else "MUSCL (minmod)"
        scheme = (f"{rname} + LF" if args.flux == "LF" else f"{rname} + Steger-Warming" if args.flux == "SW" else
                  f"Godunov ({rname} on primitives + {args.flux}, float64)")
        if args.viscous:
            scheme += " + laminar viscous fluxes (Sutherland, Pr 0.72, Le 1, CENTRAL6)"
        workload = ("2D H2-air detonation channel 1024x256 (0.2 m x 0.05 m), 9sp/19r mechanism, "
                    "30 atm / 3000 K slab with 8 seeded +-5% blobs, slip walls, "
                    f"{scheme} + SSP-RK3 + point-implicit chemistry")
    else:
        nx, ny = RDC_NX, RDC_NY
        dx = dy = 1e-4 / RDC_ND["x0"]
        bc = {"left_boundary": "periodic", "right_boundary": "periodic",
              "bottom_boundary": "rdc_injector", "top_boundary": "pressure_outlet"}
        s = Solver(2, nx, ny, dx, dy, bc, nondim_config=RDC_ND, precision=precision)
        P, T, Y, Yinj = rdc_fields()
        theta = {"Yinj": Yinj, "Pb": 101325.0 / RDC_ND["P0"]}
        s.set_theta(theta)
        workload = ("2D unrolled rotating-detonation annulus 1600x1000 (dx = 0.1 mm, nondimensional "
                    "P0 = 10 atm, T0 = 300 K, R0 = 369, x0 = 0.08 m), periodic x, choked-injector "
                    "bottom, pressure outlet top (Pb = 1 atm), linear reactant layer, 40x100 kernel")
    U0, aux0 = s.state_from_PTY(torch.tensor(P, device="cuda"), torch.tensor(T, device="cuda"),
                                torch.tensor(Y, device="cuda"))
    return s, U0, aux0, theta, nx * ny, workload


def _time_path(args, s, U0, aux0, theta, ncell, dist, clocks=None):
    """Device-timed steps (L2 flushed between steps), per-kernel split and the
    end-to-end leg for one solver.  Returns a dict of measurements."""
    import torch
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    U, aux, _ = s.advance(U0, aux0, max(args.warmup, 3), cfl=CFL, theta=theta)
    torch.cuda.synchronize()
    # external: recorded as event nodes of the graph below, timed at replay
    ev = [(torch.cuda.Event(enable_timing=True, external=True), torch.cuda.Event(enable_timing=True, external=True))
          for _ in range(args.steps)]
    # The K timed steps (each: L2 flush, then one step) are captured in one
    # CUDA graph and replayed, so that host-side stalls (driver calls blocked
    # by the clock sampler, Python) cannot open gaps inside the timed region.
    Ug, auxg = U.clone(), aux.clone()
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        s.advance(Ug, auxg, 1, cfl=CFL, theta=theta)  # warm the side stream
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, capture_error_mode="relaxed"):
        Uk, auxk = Ug, auxg
        for k in range(args.steps):
            flush.zero_()
            ev[k][0].record()
            Uk, auxk, _ = s.advance(Uk, auxk, 1, cfl=CFL, theta=theta)
            ev[k][1].record()
    graph.replay()  # warm replay
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
        clocks.wait_first()
        # the same replayed steps for ~0.45 s up to the timed replay (every
        # replay starts from the same state), so that the 200 ms sampler
        # records the clocks and throttle reasons under this load right up
        # to the timed region, which is a few ms long
        t_soak = time.time() + 0.45
        while time.time() < t_soak:
            graph.replay()
            torch.cuda.synchronize()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
    t_wall0 = time.time()
    graph.replay()
    torch.cuda.synchronize()
    t_wall = time.time() - t_wall0
    clk = clocks.stop() if clocks else None
    if clk is not None:
        clk["sampled"] = "under the same replayed steps during the 0.45 s before and through the timed replay"
    ms_total = max_over_ranks(dist, sum(a.elapsed_time(b) for a, b in ev))
    U, aux = Uk.clone(), auxk.clone()
    del graph
    status = s.status()
    # per-kernel split (events around each launch)
    s.set_kernel_timing(True)
    kt_steps = min(args.steps, 5)
    acc = {"flux": [0.0, 0], "select": [0.0, 0], "chem": [0.0, 0], "other": [0.0, 0]}
    for _ in range(kt_steps):
        flush.zero_()
        U, aux, _ = s.advance(U, aux, 1, cfl=CFL, theta=theta)
        for kk, (ms, n) in s.kernel_times().items():
            acc[kk][0] += ms
            acc[kk][1] += n
        s.set_kernel_timing(True)
    s.set_kernel_timing(False)
    # end to end through the public API: pinned host state in, state out
    hU = U.cpu().pin_memory()
    haux = aux.cpu().pin_memory()
    oU = torch.empty_like(hU).pin_memory()
    oaux = torch.empty_like(haux).pin_memory()
    e2e_steps = max(5, min(args.steps, 20))
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    legs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(e2e_steps)]
    e0.record()
    for k in range(e2e_steps):
        legs[k][0].record()
        dU = hU.to("cuda", non_blocking=True)
        daux = haux.to("cuda", non_blocking=True)
        legs[k][1].record()
        rU, raux, _ = s.advance(dU, daux, 1, cfl=CFL, theta=theta)
        legs[k][2].record()
        oU.copy_(rU, non_blocking=True)
        oaux.copy_(raux, non_blocking=True)
        legs[k][3].record()
    e1.record()
    torch.cuda.synchronize()
    # per-step end-to-end time; the median keeps one-off host stalls (other
    # processes, driver calls) out of the rate, the mean is reported beside it
    per_step = sorted(lg[0].elapsed_time(lg[3]) for lg in legs)
    e2e_mean = e0.elapsed_time(e1) / e2e_steps
    serial_ms = max_over_ranks(dist, statistics.median(per_step) * e2e_steps)
    leg_ms = [sum(lg[i].elapsed_time(lg[i + 1]) for lg in legs) / e2e_steps for i in range(3)]
    # the public host-buffer entry point: e2e_steps host states (pinned), each
    # copied in, advanced one step and copied out, the copies overlapping the
    # neighbouring items' steps (Solver.advance_host)
    ins = [(hU, haux)] * e2e_steps
    outs = [(torch.empty_like(hU).pin_memory(), torch.empty_like(haux).pin_memory()) for _ in range(2)]
    outs = [outs[k % 2] for k in range(e2e_steps)]
    s.advance_host(ins[:2], outs[:2], 1, cfl=CFL, theta=theta)  # warm-up (streams, buffers)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    p0, p1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    p0.record()
    s.advance_host(ins, outs, 1, cfl=CFL, theta=theta)
    p1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(dist, p0.elapsed_time(p1))
    ws = dist.get_world_size() if dist else 1
    return {"value": job_value(ws, ncell, args.steps, ms_total), "ms_per_step": ms_total / args.steps,
            "status": status, "clocks": clk, "t_wall": t_wall,
            "kernel_ms_per_step": {k: v[0] / kt_steps for k, v in acc.items()},
            "kernel_ms_per_launch": {k: v[0] / max(v[1], 1) for k, v in acc.items()},
            "e2e": {"value": job_value(ws, ncell, e2e_steps, e2e_ms), "unit": UNIT,
                    "h2d_bytes_per_step": (hU.numel() + haux.numel()) * 8,
                    "d2h_bytes_per_step": (hU.numel() + haux.numel()) * 8,
                    "steps": e2e_steps, "api": "Solver.advance_host (copies overlapped with the steps)",
                    "serial": {"value": job_value(ws, ncell, e2e_steps, serial_ms),
                               "api": "Solver.advance per step, copies on the same stream",
                               "h2d_ms": leg_ms[0], "step_ms": leg_ms[1], "d2h_ms": leg_ms[2],
                               "statistic": "median step", "mean_step_ms": e2e_mean}}}


def _accuracy(args, s_test, s_ref, U0, aux0, theta, steps):
    """Per-field relative L1 of the tested path against the float64 path after
    `steps` steps from the same state, and the detonation-front offset."""
    import torch
    from janc_b200 import mechanism as jm
    mech = s_ref.mech
    Ua, auxa, _ = s_test.advance(U0, aux0, steps, cfl=CFL, theta=theta)
    Ub, auxb, _ = s_ref.advance(U0, aux0, steps, cfl=CFL, theta=theta)
    invM = torch.tensor(1.0 / mech.tables["species_M"], device="cuda")

    def prim(U, aux):
        rho = U[0]
        Y8 = U[4:] / rho
        Yf = torch.cat([Y8, (1.0 - Y8.sum(0))[None]], 0)
        R = (invM[:, None, None] * Yf).sum(0)
        return rho, rho * R * aux[1], aux[1], Y8

    ra, pa, Ta, Ya = prim(Ua, auxa)
    rb, pb, Tb, Yb = prim(Ub, auxb)

    def l1(a, b):
        return float((a - b).abs().sum() / b.abs().sum().clamp_min(1e-300))

    errs = {"rho": l1(ra, rb), "p": l1(pa, pb), "T": l1(Ta, Tb)}
    for k, name in enumerate(mech.species[:8]):
        if float(Yb[k].abs().sum()) > 1e-30:
            errs["Y_" + name] = l1(Ya[k], Yb[k])
    pamb = float(pb.min())

    def front(p):
        mask = p > 2 * pamb
        idx = torch.arange(p.shape[0], device="cuda")[:, None].expand_as(p)
        return torch.where(mask, idx, torch.full_like(idx, -1)).max(0).values

    dfront = int((front(pa) - front(pb)).abs().max())
    return {"steps": steps, "l1_rel": errs, "front_max_offset_cells": dfront}


def run_ours(args):
    import torch
    from janc_b200 import _native

    dist, rank, ws = _dist()
    dev = torch.cuda.current_device()
    s, U0, aux0, theta, ncell, workload = _setup_workload(args, args.precision)
    head = _time_path(args, s, U0, aux0, theta, ncell, dist, ClockSampler(dev))
    other = None
    plain = None
    acc = None
    if args.precision != "fp64" and not args.no_compare:
        sr, _, _, _, _, _ = _setup_workload(args, "fp64")
        other = _time_path(args, sr, U0, aux0, theta, ncell, dist)
        Uw, auxw, _ = sr.advance(U0, aux0, max(args.warmup, 3), cfl=CFL, theta=theta)
        acc = _accuracy(args, s, sr, Uw, auxw, theta, args.accuracy_steps)
    if args.precision != "fp64_strict" and not args.no_compare:
        # the plain float64 CUDA path: reference operation order, no FMA
        # contraction, table-driven chemistry
        sp, _, _, _, _, _ = _setup_workload(args, "fp64_strict")
        plain = _time_path(args, sp, U0, aux0, theta, ncell, dist)
    launches_per_step = count_kernel_launches(lambda: s.advance(U0, aux0, 1, cfl=CFL, theta=theta))
    kms = head["kernel_ms_per_launch"]
    chem_ms = kms["chem"]
    flux_ms = kms["flux"]
    L = _native.lib()
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    hbm_peak, hbm_src = 6650.0, "fallback"
    if os.path.exists(peaks_path):
        try:
            hbm_peak = float(json.load(open(peaks_path))["hbm_gbs"])
            hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
        except Exception:
            pass
    fp64_peak = fp64_peak_tflops(L, torch)
    arith, special = chem_flops_per_cell()
    # dominant kernel of the headline path
    dom = "chem" if head["kernel_ms_per_step"]["chem"] >= head["kernel_ms_per_step"]["flux"] else "flux"
    bytes_cell = BYTES_CHEM_PER_CELL if dom == "chem" else BYTES_FLUX_STAGE_PER_CELL
    launch_ms = chem_ms if dom == "chem" else flux_ms
    achieved = bytes_cell * ncell / (launch_ms * 1e-3) / 1e9
    chem_tflops = arith * ncell / (chem_ms * 1e-3) / 1e12
    step_gbs = BYTES_STEP_PER_CELL * ncell / (head["ms_per_step"] * 1e-3) / 1e9

    subs = None
    if args.workload == "channel" and ws == 1 and not args.no_sub:
        subs = sub_records(args)
    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and args.workload == "channel":
        cpu = cpu_baseline(args.cpu_steps)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if args.precision != "mixed" else "f32 flux / f64 state, T-solve, chemistry",
        "data": "synthetic", "precision": args.precision,
        "config": {"workload": workload, "cells": ncell, "cfl": CFL, "precision": args.precision,
                   "l2": "flushed between timed steps (256 MB write)",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
        "status_bits": head["status"],
        "kernel_ms_per_step": head["kernel_ms_per_step"],
        # kernels of one timed step (one jb_advance call), counted as the
        # kernel nodes of a captured graph of that call, times the steps
        "gpu_launches": launches_per_step * args.steps if launches_per_step is not None else None,
        "gpu_launches_per_step": launches_per_step,
        "roofline": {"bound": "hbm", "kernel": {
                         "chem": "k_chem (point-implicit chemistry + final Halley)",
                         "flux": ("k_god2d (reconstruction on primitives + Riemann solver + RK stage + Halley)"
                                  if args.flux not in ("LF", "SW") else
                                  "flux stage: k_sweep_x + k_flux_y_rk (LF + WENO5 + RK stage + Halley)"
                                  if args.precision == "mixed" and args.flux == "LF" and args.recon == "WENO5_JS"
                                  else f"k_flux2d ({args.flux} splitting + reconstruction + RK stage + Halley)")}[dom],
                     "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "traffic": (TRAFFIC_PER_CELL[dom] * ncell if args.workload == "channel" and
                                 args.flux == "LF" and args.recon == "WENO5_JS" and not args.viscous and
                                 args.precision == "mixed" else None),
                     "traffic_source": "ncu dram bytes of one stage's launches on this workload, each "
                                       "launch cold (mixed precision): " + TRAFFIC_SOURCE,
                     "peak_source": hbm_src,
                     "algorithmic_bytes_per_cell": bytes_cell, "launch_ms": launch_ms,
                     "step_achieved_gbs": step_gbs,
                     "step_algorithmic_bytes_per_cell": BYTES_STEP_PER_CELL},
        "compute_roofline": {"bound": "fp64", "kernel": "k_chem", "achieved": chem_tflops,
                             "peak": fp64_peak, "unit": "TFLOP/s", "frac": chem_tflops / fp64_peak,
                             "peak_source": "measured live (jb_probe_fp64_fma)",
                             "flops_per_cell": arith, "special_ops_per_cell": special, "launch_ms": chem_ms},
        "e2e": head["e2e"],
        "clocks": head["clocks"],
        "wall_s_timed_region": head["t_wall"],
    }
    if other is not None:
        line["fp64"] = {"value": other["value"], "ms_per_step": other["ms_per_step"],
                        "kernel_ms_per_step": other["kernel_ms_per_step"], "e2e": other["e2e"]["value"],
                        "status_bits": other["status"]}
        # the mixed-precision gain: the same step with float64 fluxes (FMA
        # contraction, generated chemistry, the reference's global Halley stop)
        line["speedup_vs_fp64"] = head["value"] / other["value"]
    if plain is not None:
        line["fp64_strict"] = {"value": plain["value"], "ms_per_step": plain["ms_per_step"],
                               "kernel_ms_per_step": plain["kernel_ms_per_step"], "e2e": plain["e2e"]["value"],
                               "build": "the parity build: reference operation order, -fmad=false, "
                                        "table-driven chemistry, the reference's global Halley stop"}
        line["speedup_vs_fp64_strict"] = head["value"] / plain["value"]
    if acc is not None:
        line["accuracy_vs_fp64"] = acc
    if subs is not None:
        line["configs"] = subs
    if cpu is not None:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def sub_records(args):
    """The other workloads of the benchmark set, each with its own clocks, on
    one GPU: the rotating-detonation annulus (mixed precision, 10 timed steps;
    fp64 rate; accuracy against the fp64 path after 100 steps), the 64-tube
    batched ensemble (mixed, args.sub_steps steps, against the tubes one by
    one through the single-case fp64 path) and the adjoint (args.sub_steps
    steps: 200 is the configuration's length)."""
    import copy
    import torch
    global CFL
    out = {}
    cfl_keep = CFL
    a = copy.copy(args)
    a.workload, a.steps, a.viscous, a.flux, a.recon = "rdc", 10, False, "LF", "WENO5_JS"
    dev = torch.cuda.current_device()
    s, U0, aux0, theta, ncell, workload = _setup_workload(a, "mixed")
    r = _time_path(a, s, U0, aux0, theta, ncell, None, ClockSampler(dev))
    launches = count_kernel_launches(lambda: s.advance(U0, aux0, 1, cfl=CFL, theta=theta))
    sr, _, _, _, _, _ = _setup_workload(a, "fp64")
    rf = _time_path(a, sr, U0, aux0, theta, ncell, None)
    Uw, auxw, _ = sr.advance(U0, aux0, 3, cfl=CFL, theta=theta)
    acc = _accuracy(a, s, sr, Uw, auxw, theta, 100)
    out["rdc"] = {
        "metric": METRIC, "value": r["value"], "unit": UNIT, "steps": a.steps, "ms_per_step": r["ms_per_step"],
        "precision": "mixed", "cfl": CFL, "config": {"workload": workload, "cells": ncell},
        "hbm_gbs_fused_step_minimum": BYTES_STEP_PER_CELL * ncell / (r["ms_per_step"] * 1e-3) / 1e9,
        "kernel_ms_per_step": r["kernel_ms_per_step"], "gpu_launches_per_step": launches,
        "e2e": r["e2e"], "status_bits": r["status"], "clocks": r["clocks"],
        "fp64": {"value": rf["value"], "ms_per_step": rf["ms_per_step"]},
        "speedup_vs_fp64": r["value"] / rf["value"], "accuracy_vs_fp64": acc,
    }
    del s, sr
    CFL = cfl_keep
    out["ensemble"] = ensemble_record(args, None, 0, 1, args.sub_steps, "mixed", with_cpu=False)
    out["adjoint"] = adjoint_record(args, None, 1, args.sub_steps)
    out["amr"] = amr_record(args)
    return out


# --------------------------------------------------------------- AMR blocks
AMR_NBX, AMR_NBY, AMR_B = 64, 16, 20


class DeviceBlockLayer:
    """A single-level block layer on the device standing in for the external
    jaxamr package (which JANC's AMR step calls for its blocks' ghost
    layers): nbx x nby blocks of b x b cells tiling a rectangle; a block's
    3-cell ghost layers are its neighbours' cells, mirrored (zero gradient)
    outside the rectangle; one gather per fill."""

    def __init__(self, nbx, nby, b, device):
        import torch
        X, Y = nbx * b, nby * b

        def mirror(n):
            return [2 - j for j in range(3)] + list(range(n)) + [n - 1 - j for j in range(3)]
        mx, my = torch.tensor(mirror(X)), torch.tensor(mirror(Y))
        src = []
        for k in range(nbx * nby):
            i0, j0 = (k // nby) * b, (k % nby) * b
            gx = mx[i0:i0 + b + 6][:, None]
            gy = my[j0:j0 + b + 6][None, :]
            src.append(((gx // b) * nby + gy // b) * b * b + (gx % b) * b + gy % b)
        self.src = torch.stack(src).reshape(-1).to(device)
        self.nb, self.b = nbx * nby, b

    def get_ghost_block_data(self, blk, info=None):
        nf = blk.shape[1]
        flat = blk.reshape(self.nb, nf, self.b * self.b).permute(1, 0, 2).reshape(nf, -1)
        g = flat[:, self.src].reshape(nf, self.nb, self.b + 6, self.b + 6)
        return g.permute(1, 0, 2, 3).contiguous()

    def update_external_boundary(self, level, blk_data, interior, info=None):
        return interior


def amr_record(args, steps=10):
    """Block-AMR step of the channel physics (set_simulator.py:496-532
    AMR_Simulator through the drop-in mirror): one level of 64 x 16 blocks
    of 20 x 20 cells (the block size of the reference's AMR example) over
    1280 x 320 cells at the channel's spacing, float64 blocks, dt from CFL
    0.05 of the initial state; the ghost fills of a device block layer
    between the stages are inside the timed step (value), and the native
    launches alone (3 jb_amr_stage + 1 jb_amr_chem) are timed apart."""
    import numpy as np
    import torch
    from janc_b200 import mechanism as jm
    from janc_b200.janc.simulation import set_simulator as ss
    from janc_b200.janc.simulation import time_step as ts
    from janc_b200.janc import _state
    dev = torch.cuda.current_device()
    nbx, nby, b = AMR_NBX, AMR_NBY, AMR_B
    nx, ny = nbx * b, nby * b
    d = LX / NX
    P, T, Y = c1_fields(nx=nx, ny=ny)
    mpath = jm.DEFAULT_MECHANISM
    cfg = {"thermo_config": {"thermo_model": "nasa7", "mechanism_directory": mpath},
           "reaction_config": {"is_detailed_chemistry": True, "mechanism_directory": mpath},
           "flux_config": {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                           "split_method": "LF", "viscosity": "off"},
           "boundary_config": BC_SLIP4, "time_config": {"temporal_evolution_scheme": "TVD_RK3", "dt": 1.0},
           "precision": "fp64"}
    layer = DeviceBlockLayer(nbx, nby, b, "cuda")
    ts.set_amr_module(layer)
    try:
        adv_amr, _ = ss.AMR_Simulator(cfg)
        s = _state.solver_for_amr()
        from janc_b200.solver import Solver
        s1 = Solver(2, nx, ny, d, d, BC_SLIP4, jm.load(), precision="fp64")
        cu = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
        U0, a0 = s1.state_from_PTY(cu(P), cu(T), cu(Y))
        dt = float(s1.cfl_dt(U0, a0, CFL))
        grid = torch.cat([U0, a0], dim=0)
        blk0 = grid.reshape(14, nbx, b, nby, b).permute(1, 3, 0, 2, 4).reshape(nbx * nby, 14, b, b).contiguous()
        del s1

        def step(blk):
            return adv_amr(1, blk, d, d, dt, blk, None)
        blk = blk0
        for _ in range(max(args.warmup, 3)):
            blk = step(blk)
        clocks = ClockSampler(dev)
        clocks.start()
        clocks.wait_first()
        # the timed steps repeated from the same blocks for ~0.45 s up to the
        # timed region, so that the 200 ms sampler sees the clocks under
        # this load (the timed region itself is a few tens of ms)
        t_soak = time.time() + 0.45
        while time.time() < t_soak:
            blk = blk0
            for _ in range(steps):
                blk = step(blk)
            torch.cuda.synchronize()
        blk = blk0
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(steps):
            blk = step(blk)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / steps
        # the native launches alone, on fixed inputs
        G = layer.get_ghost_block_data(blk0)
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        k0.record()
        for _ in range(steps):
            o1 = s.amr_stage(G, None, 1, d, d, dt)
            o2 = s.amr_stage(G, G, 2, d, d, dt)
            o3 = s.amr_stage(G, G, 3, d, d, dt)
            s.amr_chem(blk0, dt)
        k1.record()
        torch.cuda.synchronize()
        kms = k0.elapsed_time(k1) / steps
        clk = clocks.stop()
        fin = bool(torch.isfinite(blk).all())
        st = s.status()
        del o1, o2, o3
    finally:
        ts.set_amr_module(None)
    cells = nx * ny
    pc = (b + 6) ** 2 / b ** 2  # padded entries per interior cell
    # each stage reads G (14 fields) and, in stages 2 and 3, U0 (12), and
    # writes out (14) over the padded blocks; the chemistry reads and writes
    # 14 fields of the unpadded blocks
    kbytes = 8 * cells * (pc * (28 + 2 * 40) + 28)
    return {"metric": METRIC, "value": job_value(1, cells, 1, ms), "unit": UNIT, "steps": steps,
            "ms_per_step": ms, "precision": "fp64 (float64 blocks)",
            "config": {"workload": "block AMR level: 64 x 16 blocks of 20 x 20 cells (1280 x 320) of the channel "
                                   "physics at dx = 0.2 m / 1024, slip walls around the level, device block "
                                   "layer (mirror outside the level), dt from CFL 0.05",
                       "cells": cells, "blocks": nbx * nby, "block": [b, b]},
            "kernel_ms_per_step": kms, "gpu_launches_per_step": 4,
            "kernel_hbm_gbs": kbytes / (kms * 1e-3) / 1e9,
            "kernel_bytes_note": "padded block arrays read / written once per stage, chemistry blocks once",
            "finite": fin, "status_bits": st, "clocks": clk}


# ------------------------------------------------------------- adjoint arm
ADJ_NX, ADJ_NY, ADJ_SLAB, ADJ_CFL, ADJ_K = 512, 128, 10, 0.05, 20
BC_SLIP4 = {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}


def run_adjoint(args):
    dist, rank, ws = _dist()
    line = adjoint_record(args, dist, ws, args.steps)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def adjoint_record(args, dist, ws, N):
    """The adjoint workload (config 3) on this rank; returns its record."""
    import numpy as np
    import torch
    from janc_b200.adjoint import Trajectory, probe_trajectory
    from janc_b200.solver import Solver
    dev = torch.cuda.current_device()
    nx, ny = ADJ_NX, ADJ_NY
    dx = 0.1 / nx
    P, T, Y = c1_fields(nx=nx, ny=ny, slab=ADJ_SLAB, seed=1)
    s = Solver(2, nx, ny, dx, dx, BC_SLIP4, precision="fp64")
    probe = (int(round(0.8 * nx)) - 2, ny // 2 - 2, 4, 4)
    traj = Trajectory(s, ADJ_CFL, probe, checkpoint=ADJ_K)
    cu = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    Pc, Yc, Tc = cu(P), cu(Y), cu(T)

    U0, a0 = s.state_from_PTY(Pc, Tc, Yc)

    def fwd_bwd():
        """The stepping cost alone: forward N steps (checkpoints kept), then
        the adjoint sweep (recomputation included) seeded with dL/ddt_n =
        p_n and dL/dp_n = dt_n."""
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ev[0].record()
        _, _, dts, pps, ckpts = traj.run(U0, a0, N)
        ev[1].record()
        traj.backward(ckpts, N, pps, dts)
        ev[2].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])

    for _ in range(max(args.warmup, 3)):
        fwd_bwd()
    clocks = ClockSampler(dev)
    clocks.start()
    clocks.wait_first()
    time.sleep(0.1)
    reps = [fwd_bwd() for _ in range(3)]
    clk = clocks.stop()
    f_ms = max_over_ranks(dist, statistics.median(r[0] for r in reps))
    b_ms = max_over_ranks(dist, statistics.median(r[1] for r in reps))
    # the gradients through the public autograd path
    Tg = Tc.clone().requires_grad_()
    lg = torch.zeros(19, dtype=torch.float64, device="cuda", requires_grad=True)
    dts, pps = probe_trajectory(traj, Pc, Tg, Yc, lg, N)
    lossT = (dts * pps).sum()
    lossT.backward()
    loss, gT, gA = float(lossT.detach()), Tg.grad, lg.grad
    # central finite differences of the float64 forward
    def loss_at(Tn, dA):
        traj.set_log_A_offset(dA)
        U0, a0 = s.state_from_PTY(Pc, Tn, Yc)
        _, _, dts, pps, _ = traj.run(U0, a0, N)
        return float((dts * pps).sum())
    rng = np.random.default_rng(3)
    h = 1e-6
    nd = args.fd_directions
    gTn, gAn = gT.cpu().numpy(), gA.cpu().numpy()
    Tn = T.copy()
    fd = {"T_full_field": [], "T_ignition_slab": [], "lnA": []}
    for kind in fd:
        for _ in range(nd):
            if kind == "lnA":
                e = rng.standard_normal(19)
                e /= np.linalg.norm(e)
                f = (loss_at(Tc, h * e) - loss_at(Tc, -h * e)) / (2 * h)
                a = float((gAn * e).sum())
            else:
                d = rng.standard_normal(T.shape)
                if kind == "T_ignition_slab":
                    d[:, ADJ_SLAB:] = 0.0
                d /= np.linalg.norm(d)
                f = (loss_at(cu(Tn * (1 + h * d)), None) - loss_at(cu(Tn * (1 - h * d)), None)) / (2 * h)
                a = float((gTn * Tn * d).sum())
            fd[kind].append(abs(f - a) / max(abs(f), 1e-300))
    traj.set_log_A_offset(None)
    # (1) h-sweep along two full-field directions: on the exactly uniform
    # ambient gas the central difference plateaus away from the adjoint
    # instead of converging to it
    sweep = []
    rng_s = np.random.default_rng(5)
    for _ in range(2):
        d = rng_s.standard_normal(T.shape)
        d /= np.linalg.norm(d)
        a = float((gTn * Tn * d).sum())
        row = {"adjoint": a}
        for hh in (1e-3, 1e-4, 1e-5, 1e-6, 1e-7, 1e-8, 1e-9):
            f = (loss_at(cu(Tn * (1 + hh * d)), None) - loss_at(cu(Tn * (1 - hh * d)), None)) / (2 * hh)
            row[f"{hh:.0e}"] = abs(f - a) / max(abs(f), 1e-300)
        sweep.append(row)
    # (2) the same workload with 1 % seeded noise on the ambient temperature
    # (no exactly uniform region): the full-field directions against the
    # adjoint of that state
    Tz = T.copy()
    Tz[:, ADJ_SLAB:] *= 1.0 + 0.01 * np.random.default_rng(6).standard_normal(Tz[:, ADJ_SLAB:].shape)
    Tzc = cu(Tz)
    Tg2 = Tzc.clone().requires_grad_()
    dts2, pps2 = probe_trajectory(traj, Pc, Tg2, Yc, None, N)
    (dts2 * pps2).sum().backward()
    gTz = Tg2.grad.cpu().numpy()
    # the central difference at h and at 10 h: in a direction whose
    # derivative is small against the others the h = 1e-6 difference is
    # dominated by the forward's round-off (its error grows as 1/h), which
    # the 10 h column shows
    noised, noised10, adj_n, err_abs = [], [], [], []
    rng_n = np.random.default_rng(7)
    for _ in range(nd):
        d = rng_n.standard_normal(T.shape)
        d /= np.linalg.norm(d)
        f = (loss_at(cu(Tz * (1 + h * d)), None) - loss_at(cu(Tz * (1 - h * d)), None)) / (2 * h)
        h10 = 10 * h
        f10 = (loss_at(cu(Tz * (1 + h10 * d)), None) - loss_at(cu(Tz * (1 - h10 * d)), None)) / (2 * h10)
        a = float((gTz * Tz * d).sum())
        noised.append(abs(f - a) / max(abs(f), 1e-300))
        noised10.append(abs(f10 - a) / max(abs(f10), 1e-300))
        adj_n.append(abs(a))
        err_abs.append(abs(f - a))
    scale = statistics.median(adj_n)
    cells = nx * ny
    fd_sum = {k: {"directions": len(v), "max_rel_err": max(v), "median_rel_err": statistics.median(v)}
              for k, v in fd.items() if v}
    line = {
        "metric": "adjoint/forward cost", "value": b_ms / f_ms, "unit": "ratio", "n_gpus": ws, "steps": N,
        "warmup": max(args.warmup, 3), "ms_per_step": b_ms / N, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "adjoint of the 2D H2-air channel, 512x128 cells (0.1 m x 0.025 m), slab = first "
                               "10 columns with 8 seeded +-5% blobs, slip walls, CFL 0.05; loss = sum_n dt_n * "
                               "mean p over a 4x4 probe at x = 0.8 L, y = H/2; gradients w.r.t. the initial T "
                               "field (65536) and ln A (19); checkpoint every 20 steps",
                   "cells": cells, "checkpoint": ADJ_K, "probe": probe,
                   "l2": "working set 29 MB per step record, not flushed (the backward re-reads its records)",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
        "forward_ms": f_ms, "backward_ms": b_ms, "forward_ms_per_step": f_ms / N,
        "backward_ms_per_step": b_ms / N,
        "forward_cell_updates_per_s": job_value(ws, cells, N, f_ms),
        "e2e": {"value": job_value(ws, cells, N, f_ms + b_ms), "unit": "cell-steps of value and gradient / s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "loss": loss,
        "finite_difference_check": {"h_rel": h, **fd_sum,
                                    "T_full_field_noised_ambient": {
                                        "directions": len(noised), "max_rel_err": max(noised),
                                        "median_rel_err": statistics.median(noised),
                                        "max_rel_err_h1e-5": max(noised10),
                                        "median_rel_err_h1e-5": statistics.median(noised10),
                                        "max_err_over_median_directional_derivative": max(err_abs) / scale,
                                        "min_over_median_directional_derivative": min(adj_n) / scale,
                                        "state": "the same workload with 1 % seeded noise (default_rng(6)) on "
                                                 "the ambient temperature"},
                                    "T_full_field_h_sweep": sweep,
                                    "note": "full-field directions perturb the exactly uniform ambient gas, "
                                            "where WENO5-JS (eps = 1e-6 against split fluxes ~1e8) is linear "
                                            "only below ~1e-11 relative perturbations"},
        # forward: 9 per step (step begin, 3 flux stages, 2 selects, chemistry,
        # final select, probe) + 2 per checkpoint segment; backward: the
        # recorded recomputation (10 per step: + the stage-3 select) + 2 per
        # segment and 8 adjoint kernels per step (begin, chemistry VJP, and a
        # sweep and a merge per RK stage)
        "gpu_launches": 27 * N + 4 * ((N + ADJ_K - 1) // ADJ_K), "clocks": clk,
        "tube_1d": adjoint_1d_record(args, dist, N),
    }
    return line


def adjoint_1d_record(args, dist, N):
    """The 1D form of the adjoint workload: config-0 physics (2000 cells over
    0.1 m, the first 40 at 30 atm / 3000 K with seeded +-5 % noise, 1 %
    seeded noise on the ambient temperature, slip wall left, zero gradient
    right), CFL 0.1, N steps checkpointed every 20, loss = sum_n dt_n * mean
    p over cells 1600..1603; cost ratio and central finite differences
    (h = 1e-6 relative, 8 seeded unit directions each for T and ln A)."""
    import numpy as np
    import torch
    from janc_b200 import mechanism as jm
    from janc_b200.adjoint import Trajectory, probe_trajectory
    from janc_b200.solver import Solver
    n, dx = 2000, 0.1 / 2000
    mech = jm.load()
    rng = np.random.default_rng(8)
    P = np.full((1, n), 101325.0)
    T = 300.0 * (1 + 0.01 * rng.standard_normal((1, n)))
    P[0, :40] = 30 * 101325.0
    T[0, :40] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, 40))
    Y = np.ascontiguousarray(np.tile(jm.stoichiometric_Y(mech, 1.0)[:, None], (1, n)))
    s = Solver(1, n, None, dx, None, {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"},
               mech, precision="fp64")
    traj = Trajectory(s, 0.1, (1600, 4), checkpoint=ADJ_K)
    cu = lambda a: torch.as_tensor(a, dtype=torch.float64, device="cuda")
    Pc, Tc, Yc = cu(P), cu(T), cu(Y)
    U0, a0 = s.state_from_PTY(Pc, Tc, Yc)

    def fwd_bwd():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        torch.cuda.synchronize()
        ev[0].record()
        _, _, dts, pps, ckpts = traj.run(U0, a0, N)
        ev[1].record()
        traj.backward(ckpts, N, pps, dts)
        ev[2].record()
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    for _ in range(3):
        fwd_bwd()
    reps = [fwd_bwd() for _ in range(3)]
    f_ms = max_over_ranks(dist, statistics.median(r[0] for r in reps))
    b_ms = max_over_ranks(dist, statistics.median(r[1] for r in reps))
    Tg = Tc.clone().requires_grad_()
    lg = torch.zeros(19, dtype=torch.float64, device="cuda", requires_grad=True)
    dts, pps = probe_trajectory(traj, Pc, Tg, Yc, lg, N)
    (dts * pps).sum().backward()
    gT, gA = Tg.grad.cpu().numpy(), lg.grad.cpu().numpy()

    def loss_at(Tn, dA):
        traj.set_log_A_offset(dA)
        U, a = s.state_from_PTY(Pc, Tn, Yc)
        _, _, d, p, _ = traj.run(U, a, N)
        return float((d * p).sum())
    h, rng_d = 1e-6, np.random.default_rng(13)
    errT, errA = [], []
    for _ in range(8):
        d = rng_d.standard_normal(T.shape)
        d /= np.linalg.norm(d)
        f = (loss_at(cu(T * (1 + h * d)), None) - loss_at(cu(T * (1 - h * d)), None)) / (2 * h)
        errT.append(abs(f - float((gT * T * d).sum())) / abs(f))
        e = rng_d.standard_normal(19)
        e /= np.linalg.norm(e)
        f = (loss_at(Tc, h * e) - loss_at(Tc, -h * e)) / (2 * h)
        errA.append(abs(f - float((gA * e).sum())) / abs(f))
    traj.set_log_A_offset(None)
    return {"workload": "1D tube, 2000 cells (config-0 physics, 1 % noise on the ambient temperature), CFL 0.1, "
                        f"{N} steps, checkpoint every {ADJ_K}; loss = sum_n dt_n * mean p over cells 1600..1603",
            "value": b_ms / f_ms, "unit": "adjoint/forward cost", "forward_ms_per_step": f_ms / N,
            "backward_ms_per_step": b_ms / N,
            "finite_difference_check": {"h_rel": h,
                                        "T": {"directions": len(errT), "max_rel_err": max(errT),
                                              "median_rel_err": statistics.median(errT)},
                                        "lnA": {"directions": len(errA), "max_rel_err": max(errA),
                                                "median_rel_err": statistics.median(errA)}}}


# ------------------------------------------------------------ ensemble arm
BC1 = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient"}


def _ens_setup(precision):
    from janc_b200.ensemble import Ensemble, detonation_tubes
    tubes = detonation_tubes(ENS_N, seed=ENS_SEED)
    ens = Ensemble([t["nx"] for t in tubes], [t["dx"] for t in tubes], cfl=ENS_CFL, precision=precision)
    init = []
    for i, t in enumerate(tubes):
        U, aux = ens.state_from_PTY(t["P"], t["T"], t["Y"])
        ens.set_state(i, U, aux)
        init.append((U, aux))
    return ens, tubes, init


def _ens_reset(ens, init):
    for i, (U, aux) in enumerate(init):
        ens.set_state(i, U, aux)


def _prim_1d(mech, U, aux):
    """rho, p, T of a 1D state (U: rho, rho u, rho E, rho Y_1..8)."""
    import torch
    invM = torch.tensor(1.0 / mech.tables["species_M"], device=U.device)
    rho = U[0]
    Y8 = U[3:] / rho
    Yf = torch.cat([Y8, (1.0 - Y8.sum(0))[None]], 0)
    R = (invM[:, None] * Yf).sum(0)
    return rho, rho * R * aux[1], aux[1]


def run_ensemble(args):
    if args.precision not in ("fp64", "mixed"):
        raise SystemExit("the ensemble runs in 'fp64' or 'mixed' precision")
    dist, rank, ws = _dist()
    line = ensemble_record(args, dist, rank, ws, args.steps, args.precision,
                           with_cpu=rank == 0 and ws == 1 and not args.no_cpu_baseline)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)


def ensemble_record(args, dist, rank, ws, K, precision, with_cpu):
    """The batched-ensemble workload (config 4) on this rank; returns its record."""
    import torch
    from janc_b200 import _native
    from janc_b200.solver import Solver
    dev = torch.cuda.current_device()
    ens, tubes, init = _ens_setup(precision)
    cells = ens.total_cells
    if args.ens_shape:
        block, bpsm = (int(v) for v in args.ens_shape.split("x"))
        ens.configure(block, bpsm)
        tune = {"skipped": f"launch shape fixed by --ens-shape {args.ens_shape}"}
    else:
        tune = ens.autotune(trial_steps=20)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > 126 MB L2
    _ens_reset(ens, init)
    ens.advance(args.warmup)
    _ens_reset(ens, init)
    ens.advance(K)  # captures the K-step graph replayed below
    _ens_reset(ens, init)
    flush.zero_()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(dev)
    clocks.start()
    clocks.wait_first()
    time.sleep(0.1)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_wall0 = time.time()
    e0.record()
    ens.advance(K)
    e1.record()
    torch.cuda.synchronize()
    t_wall = time.time() - t_wall0
    clk = clocks.stop()
    ms = max_over_ranks(dist, e0.elapsed_time(e1))
    status, per_status = ens.status()
    shape = ens.launch_shape()
    final = [ens.get_state(i) for i in range(ENS_N)]
    n_finite = sum(int(torch.all(torch.isfinite(U)).item()) for U, _ in final)
    value = job_value(ws, cells, K, ms)
    # end to end through the public API: pinned host states in, K steps, states out
    hU = [U.cpu().pin_memory() for U, _ in init]
    ha = [a.cpu().pin_memory() for _, a in init]
    oU = [torch.empty_like(x).pin_memory() for x in hU]
    oa = [torch.empty_like(x).pin_memory() for x in ha]
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    legs = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    legs[0].record()
    for i in range(ENS_N):
        Ud, ad = ens.state(i)
        Ud.copy_(hU[i], non_blocking=True)
        ad.copy_(ha[i], non_blocking=True)
    legs[1].record()
    ens.advance(K)
    legs[2].record()
    for i in range(ENS_N):
        Ud, ad = ens.state(i)
        oU[i].copy_(Ud, non_blocking=True)
        oa[i].copy_(ad, non_blocking=True)
    legs[3].record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(dist, legs[0].elapsed_time(legs[3]))
    io_bytes = sum(x.numel() for x in hU + ha) * 8
    # the 64 tubes one after another through the single-case float64 path
    seq_steps = getattr(args, "seq_steps", 0) or K
    seq_ms, seq_final = 0.0, []
    for i, t in enumerate(tubes):
        s = Solver(1, t["nx"], dx=t["dx"], boundary_config=BC1, precision="fp64")
        s.advance(init[i][0], init[i][1], 3, cfl=ENS_CFL)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        U, aux, _ = s.advance(init[i][0], init[i][1], seq_steps, cfl=ENS_CFL)
        b.record()
        torch.cuda.synchronize()
        seq_ms += a.elapsed_time(b)
        seq_final.append((U, aux))
        del s
    seq_ms = max_over_ranks(dist, seq_ms)
    seq_value = job_value(ws, cells, seq_steps, seq_ms)
    acc = None
    if seq_steps == K:
        worst = {"rho": 0.0, "p": 0.0, "T": 0.0}
        dfront = 0
        for (Ua, aa), (Ub, ab) in zip(final, seq_final):
            pa = _prim_1d(ens.mech, Ua, aa)
            pb = _prim_1d(ens.mech, Ub, ab)
            for name, x, y in zip(("rho", "p", "T"), pa, pb):
                worst[name] = max(worst[name], float((x - y).abs().sum() / y.abs().sum()))
            pamb = float(pb[1][-1])
            fa = int(torch.nonzero(pa[1] > 2 * pamb).max()) if bool((pa[1] > 2 * pamb).any()) else -1
            fb = int(torch.nonzero(pb[1] > 2 * pamb).max()) if bool((pb[1] > 2 * pamb).any()) else -1
            dfront = max(dfront, abs(fa - fb))
        acc = {"steps": K, "l1_rel_max_over_tubes": worst, "front_max_offset_cells": dfront,
               "reference": "the same tubes through the single-case float64 path"}
    hbm_peak, hbm_src = 6650.0, "fallback"
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        try:
            hbm_peak = float(json.load(open(peaks_path))["hbm_gbs"])
            hbm_src = "measured (MEASURED_PEAKS.json hbm_gbs)"
        except Exception:
            pass
    fp64_peak = fp64_peak_tflops(_native.lib(), torch)
    arith, special = chem_flops_per_cell()
    achieved = BYTES_ENS_STEP_PER_CELL[precision] * cells * K / (ms * 1e-3) / 1e9
    chem_tflops = arith * cells * K / (ms * 1e-3) / 1e12
    cpu = cpu_baseline_ensemble(args.cpu_steps) if with_cpu else None
    sizes = [t["nx"] for t in tubes]
    line = {
        "metric": "total " + METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K,
        "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if precision == "fp64" else "f32 flux / f64 state, T-solve, chemistry",
        "data": "synthetic", "precision": precision,
        "config": {"workload": f"batched ensemble: {ENS_N} 1D H2-air detonation tubes, lengths "
                               f"log-uniform 1000-16000 cells (dx 50 um), phi U(0.6,1.4), T_ign "
                               f"U(2500,3500) K, default_rng({ENS_SEED}); 30 atm slab over the first 2 %; "
                               f"reflective left / outflow right; CFL {ENS_CFL} per tube",
                   "cells": cells, "tubes": ENS_N, "cells_min": min(sizes), "cells_max": max(sizes),
                   "launch": "one persistent cooperative kernel for all steps, replayed from a CUDA graph",
                   "launch_shape": shape, "autotune": tune,
                   "l2": "flushed once before the timed launch (256 MB write); inside the persistent "
                         "launch each tube's working set stays wherever the cache keeps it",
                   "parallelism": f"replicas x{ws}" if ws > 1 else "single GPU"},
        "status_bits": status, "tubes_finite": n_finite,
        "gpu_launches": 1,
        "roofline": {"bound": "hbm", "kernel": "k_ensemble (all phases of all steps)", "achieved": achieved,
                     "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     "traffic": TRAFFIC_ENS_PER_CELL_STEP * cells * K if precision == "mixed" else None,
                     "traffic_source": "ncu dram bytes of a 20-step launch, scaled to this launch's cell-steps",
                     "peak_source": hbm_src, "algorithmic_bytes_per_cell_step": BYTES_ENS_STEP_PER_CELL[precision],
                     "launch_ms": ms},
        "compute_roofline": {"bound": "fp64", "kernel": "k_ensemble (chemistry share of the flops only)",
                             "achieved": chem_tflops, "peak": fp64_peak, "unit": "TFLOP/s",
                             "frac": chem_tflops / fp64_peak, "peak_source": "measured live (jb_probe_fp64_fma)"},
        "e2e": {"value": job_value(ws, cells, K, e2e_ms), "unit": UNIT,
                "h2d_bytes_per_step": io_bytes / K, "d2h_bytes_per_step": io_bytes / K,
                "h2d_bytes_per_call": io_bytes, "d2h_bytes_per_call": io_bytes, "steps_per_call": K,
                "h2d_ms": legs[0].elapsed_time(legs[1]), "run_ms": legs[1].elapsed_time(legs[2]),
                "d2h_ms": legs[2].elapsed_time(legs[3])},
        "sequential_fp64": {"value": seq_value, "steps": seq_steps, "ms_total": seq_ms,
                            "path": "64 tubes one after another, single-case float64 solver (11 launches/step)"},
        "speedup_vs_sequential_fp64": value / seq_value,
        "clocks": clk, "wall_s_timed_region": t_wall,
    }
    if acc is not None:
        line["accuracy_vs_fp64"] = acc
    if cpu is not None:
        line["cpu_baseline"] = cpu
    return line


def _oracle_tube(args):
    """One replica: the NumPy oracle advancing ensemble tube i for `steps` steps."""
    i, steps, warm = args
    import warnings
    warnings.simplefilter("ignore")
    sys.path.insert(0, ROOT)
    from oracle import janc_oracle as jo
    from janc_b200.ensemble import detonation_tubes
    from janc_b200.mechanism import DEFAULT_MECHANISM
    m = jo.load_mechanism(DEFAULT_MECHANISM)
    t = detonation_tubes(ENS_N, seed=ENS_SEED)[i]
    U, aux = jo.state_from_PTY(m, t["P"], t["T"], t["Y"])
    s = jo.Solver(m, "1D", t["dx"], None, BC1, ENS_CFL)
    tt = 0.0
    for _ in range(warm):  # untimed warm-up steps
        U, aux, tt, _ = s.advance_func(U, aux, tt)
    t0 = time.perf_counter()
    for _ in range(steps):
        U, aux, tt, _ = s.advance_func(U, aux, tt)
    return time.perf_counter() - t0, t["nx"] * steps


def cpu_baseline_ensemble(steps, warm=1):
    """The oracle on all host cores, one ensemble tube per process."""
    import concurrent.futures as cf
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    nrep = max(1, min(cores, ENS_N))
    env_keep = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
    for k in env_keep:
        os.environ[k] = "1"
    t0 = time.perf_counter()
    with cf.ProcessPoolExecutor(nrep, mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_oracle_tube, [(i, steps, warm) for i in range(nrep)]))
    wall = time.perf_counter() - t0
    for k, v in env_keep.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    slowest = max(r[0] for r in res)
    cells = sum(r[1] for r in res)
    return {"value": cells / slowest, "unit": UNIT, "cores": nrep, "kind": "port",
            "sample": f"tubes 0..{nrep - 1} of the {ENS_N}-tube ensemble, {steps} steps each, one process "
                      f"per core (NumPy oracle restating src/janc_v2)",
            "wall_s": wall}


# ----------------------------------------------------------------- CPU side
def _oracle_replica(args):
    """One replica: the NumPy oracle advancing a 32 x 256 strip of the channel
    (slab columns included, same boundaries and CFL) for `steps` steps."""
    nx, steps, warm = args
    import warnings
    import numpy as np
    warnings.simplefilter("ignore")
    sys.path.insert(0, ROOT)
    from oracle import janc_oracle as jo
    from janc_b200.mechanism import DEFAULT_MECHANISM
    m = jo.load_mechanism(DEFAULT_MECHANISM)
    P, T, Y = c1_fields(nx=nx, ny=NY)
    U, aux = jo.state_from_PTY(m, P, T, Y)
    bc = {k: "slip_wall" for k in ("left_boundary", "right_boundary", "bottom_boundary", "top_boundary")}
    s = jo.Solver(m, "2D", LX / NX, LY / NY, bc, CFL)
    t = 0.0
    for _ in range(warm):  # untimed warm-up steps
        U, aux, t, _ = s.advance_func(U, aux, t)
    t0 = time.perf_counter()
    for _ in range(steps):
        U, aux, t, _ = s.advance_func(U, aux, t)
    return time.perf_counter() - t0, nx * NY * steps


def cpu_baseline(steps, warm=1):
    """The oracle on all host cores as independent replicas (spawned
    processes, one BLAS thread each); returns the cpu_baseline record."""
    import concurrent.futures as cf
    import multiprocessing as mp
    cores = os.cpu_count() or 1
    nrep = max(1, min(cores, 64))
    nx = 32
    env_keep = {k: os.environ.get(k) for k in ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS")}
    for k in env_keep:
        os.environ[k] = "1"
    t0 = time.perf_counter()
    with cf.ProcessPoolExecutor(nrep, mp_context=mp.get_context("spawn")) as ex:
        res = list(ex.map(_oracle_replica, [(nx, steps, warm)] * nrep))
    wall = time.perf_counter() - t0
    for k, v in env_keep.items():
        if v is None:
            os.environ.pop(k, None)
        else:
            os.environ[k] = v
    slowest = max(r[0] for r in res)
    cells = sum(r[1] for r in res)
    return {"value": cells / slowest, "unit": UNIT, "cores": nrep, "kind": "port",
            "sample": f"{nrep} replicas x {nx}x{NY} cells x {steps} steps of the same channel physics "
                      f"(NumPy oracle restating src/janc_v2; one process per core)",
            "wall_s": wall}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    # the driver's warm-up count, bounded so that the run stays short
    warm = max(1, min(args.warmup, 5))
    if args.workload == "ensemble":
        steps = max(1, min(args.steps, 10))
        cpu = cpu_baseline_ensemble(steps, warm)
        line = {"impl": "reference", "metric": "total " + METRIC, "value": cpu["value"], "unit": UNIT,
                "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": steps, "warmup": warm,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic",
                "config": {"workload": f"batched ensemble of {ENS_N} 1D tubes, CPU reference path", "cfl": ENS_CFL},
                "cpu_baseline": cpu,
                "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return
    steps = max(1, min(args.steps, 20))
    cpu = cpu_baseline(steps, warm)
    line = {"impl": "reference", "metric": METRIC, "value": cpu["value"], "unit": UNIT,
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": steps, "warmup": warm,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "2D H2-air detonation channel (strips of 32x256 cells of the 1024x256 "
                                   "workload), CPU reference path", "cfl": CFL},
            "cpu_baseline": cpu,
            "e2e": {"value": cpu["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "JAX is not installed here; the reference's CPU path is the NumPy oracle, a "
                    "bitwise-pinned restatement of src/janc_v2 (tests/test_oracle_golden.py)"}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "fp64_strict", "mixed"])
    ap.add_argument("--no-compare", action="store_true", help="skip the float64 comparison run")
    ap.add_argument("--accuracy-steps", type=int, default=2000,
                    help="steps of the mixed-vs-fp64 comparison (2000: the channel configuration's length)")
    ap.add_argument("--no-sub", action="store_true",
                    help="channel: skip the sub-records of the other workloads (rdc, ensemble, adjoint)")
    ap.add_argument("--sub-steps", type=int, default=200,
                    help="steps of the ensemble and adjoint sub-records")
    ap.add_argument("--workload", default="channel", choices=["channel", "rdc", "ensemble", "adjoint", "amr"])
    ap.add_argument("--viscous", action="store_true",
                    help="channel workload with the laminar viscous fluxes")
    ap.add_argument("--flux", default="LF", choices=["LF", "SW", "HLLC", "AUSMPW_plus"],
                    help="advective flux of the channel workload (LF or Steger-Warming flux splitting, "
                         "or a Godunov Riemann solver)")
    ap.add_argument("--recon", default="WENO5_JS", choices=["WENO5_JS", "MUSCL"],
                    help="face reconstruction of the channel workload")
    ap.add_argument("--fd-directions", type=int, default=16,
                    help="adjoint: finite-difference directions per kind")
    ap.add_argument("--ens-shape", default="",
                    help="ensemble: fixed launch shape BLOCKxCTAS_PER_SM instead of the autotuner")
    ap.add_argument("--seq-steps", type=int, default=0,
                    help="ensemble: steps of the sequential float64 comparison (default: --steps)")
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "ensemble":
        run_ensemble(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "amr":
        print(json.dumps(amr_record(args, steps=args.steps)), flush=True)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
