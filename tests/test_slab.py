"""x-slab decomposition (the reference's is_parallel mode: parallel/*.py,
set_simulator.py pmin of the CFL step).

CPU: the per-slab side kinds, the column split, the ring transport and the
CFL MIN reduction over ``gloo`` ranks (world size 2 and 3), and oracle
identities: each slab's padded arrays equal windows of the global pad away
from the corners, so with a Riemann-solver flux (no global wave speed) the
slabs' flux_func equals the single-domain one exactly.
GPU (through the C ABI): slabs as ``gloo`` ranks, one process each on one
GPU (their kernels never wait on one another: the exchange runs on the host
between launches), against the oracle's lockstep SlabSolver.  Tolerances:
``fp64_strict`` 1e-12 relative L1 per field over steps, ``fp64`` 1e-10,
``mixed`` 1e-4 per field and 1e-6 on the density.
"""
import datetime
import os
import socket

import numpy as np
import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

from oracle import janc_oracle as jo  # noqa: E402

KEYS2 = ["left_boundary", "right_boundary", "bottom_boundary", "top_boundary"]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, size, port):
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=60))


@pytest.fixture(scope="module")
def omech():
    from janc_b200.mechanism import DEFAULT_MECHANISM
    return jo.load_mechanism(DEFAULT_MECHANISM)


def field_err(a, b):
    errs = []
    for i in range(a.shape[0]):
        den = np.sum(np.abs(b[i]))
        if den > 1e-30:
            errs.append(np.sum(np.abs(a[i] - b[i])) / den)
    return max(errs)


# ---------------------------------------------------------------- CPU
def test_slab_boundary_kinds():
    from janc_b200 import _native
    from janc_b200.slab import Slab
    K = _native.BC_KIND
    H = _native.BC_HALO
    walls = [K["slip_wall"], K["pressure_outlet"], K["slip_wall"], K["zero_gradient"]]
    assert Slab(rank=0, size=3).boundary_kinds(walls) == [K["slip_wall"], H, K["slip_wall"], K["zero_gradient"]]
    assert Slab(rank=1, size=3).boundary_kinds(walls) == [H, H, K["slip_wall"], K["zero_gradient"]]
    assert Slab(rank=2, size=3).boundary_kinds(walls) == [H, K["pressure_outlet"], K["slip_wall"],
                                                          K["zero_gradient"]]
    per = [K["periodic"]] * 4
    for r in range(3):
        assert Slab(rank=r, size=3).boundary_kinds(per) == [H, H, 0, 0]
    assert Slab(rank=0, size=1).boundary_kinds(walls) == walls
    assert Slab(rank=0, size=1).boundary_kinds(per) == [H, H, 0, 0]
    s = Slab(rank=2, size=4)
    assert (s.left, s.right) == (1, 3) and Slab(rank=3, size=4).right == 0
    assert s.columns(64) == (32, 16)
    with pytest.raises(AssertionError):
        s.columns(30)
    with pytest.raises(ValueError):
        Slab(rank=4, size=4)


def test_split_grid_cpu():
    from janc_b200.slab import Slab, split_and_distribute_grid
    g = np.arange(3 * 12 * 5, dtype=np.float64).reshape(3, 12, 5)
    parts = [split_and_distribute_grid(g, Slab(rank=r, size=4), device="cpu") for r in range(4)]
    assert all(p.shape == (3, 3, 5) and p.is_contiguous() for p in parts)
    assert np.array_equal(np.concatenate([p.numpy() for p in parts], axis=1), g)
    with pytest.raises(AssertionError):
        split_and_distribute_grid(g, Slab(rank=0, size=5), device="cpu")


def _transport_worker(rank, size, port, out):
    from janc_b200 import _native
    from janc_b200.slab import Slab, SlabExchange, gather_grid
    _init(rank, size, port)
    try:
        slab = Slab()
        x = SlabExchange(slab, nv=2, ny=3, device="cpu")
        # send[side][q][layer][y] = 1000 rank + 100 side + 10 layer + y (q shifts by 0.5)
        s, q, l, y = np.meshgrid(np.arange(2), np.arange(4), np.arange(3), np.arange(3), indexing="ij")
        x.send.copy_(torch.as_tensor(1000.0 * rank + 100 * s + 10 * l + y + 0.5 * q))
        x.red.copy_(torch.tensor([7 + rank, -(rank == size - 1)], dtype=torch.int64))
        x.transfer(_native.XCH_DT | _native.XCH_HALO)
        g = gather_grid(torch.full((1, 2, 1), float(rank)), slab)
        np.savez(os.path.join(out, f"r{rank}.npz"), halo=x.halo.numpy(), red=x.red.numpy(), g=g.numpy())
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("size", [2, 3])
def test_ring_transport_gloo(tmp_path, size):
    """halo[0] = left neighbour's send[1], halo[1] = right neighbour's send[0],
    ring-wrapped; the CFL pair is the MIN over the ranks."""
    mp.start_processes(_transport_worker, args=(size, _free_port(), str(tmp_path)), nprocs=size,
                       start_method="spawn")
    s, q, l, y = np.meshgrid(np.arange(2), np.arange(4), np.arange(3), np.arange(3), indexing="ij")
    for r in range(size):
        d = np.load(tmp_path / f"r{r}.npz")
        left, right = (r - 1) % size, (r + 1) % size
        assert np.array_equal(d["halo"][0], (1000.0 * left + 100 + 10 * l + y + 0.5 * q)[0])
        assert np.array_equal(d["halo"][1], (1000.0 * right + 10 * l + y + 0.5 * q)[1])
        assert d["red"].tolist() == [7, -1]
        assert d["g"].ravel().tolist() == sum(([float(k)] * 2 for k in range(size)), [])


def _dead_peer_worker(rank, size, port, out):
    from janc_b200 import _native
    from janc_b200.slab import Slab, SlabExchange
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=size,
                            timeout=datetime.timedelta(seconds=3))
    try:
        if rank == 1:
            return  # leaves between steps, before the exchange
        x = SlabExchange(Slab(), nv=2, ny=3, device="cpu")
        rc = x._callback(None, _native.XCH_HALO, None)
        with open(os.path.join(out, "r0.txt"), "w") as f:
            f.write(f"{rc} {type(x.error).__name__} {x.calls}")
    finally:
        if rank == 0:
            dist.destroy_process_group()


def test_exchange_with_a_departed_peer_fails_on_the_host(tmp_path):
    """Failure detection on the slab path: the peer never joins the exchange;
    the group's timeout ends the transfer with an error, which the callback
    turns into a failed return (the library then fails the call)."""
    mp.start_processes(_dead_peer_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    rc, err, calls = (tmp_path / "r0.txt").read_text().split()
    assert rc == "1" and calls == "0" and err != "NoneType"


def _state2d(om, nx, ny, seed):
    rng = np.random.default_rng(seed)
    P = np.full((1, nx, ny), 101325.0)
    T = np.full((1, nx, ny), 300.0)
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None, None], (1, nx, ny))
    P[:, :4] = 30 * 101325.0
    T[:, :4] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, 4, ny)))
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * rng.uniform(-50.0, 50.0, (nx, ny))
    U[2] += U[0] * rng.uniform(-50.0, 50.0, (nx, ny))
    return U, jo.update_aux(om, U, aux)


def _state1d(om, nx, seed):
    rng = np.random.default_rng(seed)
    P = np.full((1, nx), 101325.0)
    T = np.full((1, nx), 300.0)
    Y = np.tile(jo.stoich_Y(om, 1.0)[:, None], (1, nx))
    P[:, :6] = 30 * 101325.0
    T[:, :6] = 3000.0
    U, aux = jo.state_from_PTY(om, P, T, Y)
    U[1] += U[0] * rng.uniform(-50.0, 50.0, nx)
    return U, jo.update_aux(om, U, aux)


@pytest.mark.parametrize("dim", [1, 2])
def test_oracle_slab_pad_is_global_pad_window(omech, dim):
    bc = dict(zip(KEYS2, ["slip_wall", "pressure_outlet", "no_slip_wall", "zero_gradient"]))
    U, a = _state2d(omech, 24, 8, 1) if dim == 2 else _state1d(omech, 24, 1)
    if dim == 1:
        bc = {k: bc[k] for k in KEYS2[:2]}
    theta = {"Pb": 101325.0}
    Up, Ap = jo.boundary_conditions(omech, U, a, bc, theta)
    for P in (2, 3, 4):
        Us, As = np.split(U, P, axis=1), np.split(a, P, axis=1)
        n = 24 // P
        for r in range(P):
            up, ap = jo.parallel_boundary_conditions(omech, Us, As, r, bc, theta)
            win = (slice(None), slice(r * n, r * n + n + 6)) + ((slice(3, -3),) if dim == 2 else ())
            assert np.array_equal(up[win[:1] + (slice(None),) + win[2:]], Up[win])
            assert np.array_equal(ap[win[:1] + (slice(None),) + win[2:]], Ap[win])


def test_oracle_slab_godunov_flux_equals_single_domain(omech):
    """No global wave speed on the Godunov path and no corner reads without
    viscosity: the slabs' fluxes are the single-domain flux, bit for bit."""
    fc = {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": "HLLC",
          "viscosity": "off"}
    bc = dict(zip(KEYS2, ["slip_wall", "zero_gradient", "slip_wall", "slip_wall"]))
    U, a = _state2d(omech, 24, 10, 2)
    ref = jo.Solver(omech, "2D", 1e-4, 1e-4, bc, 0.5, flux_config=fc).flux_func(U, a, 1e-4, 1e-4, 1e-8)
    o = jo.SlabSolver(omech, "2D", 1e-4, 1e-4, bc, 0.5, flux_config=fc)
    got = o.flux_func(np.split(U, 3, axis=1), np.split(a, 3, axis=1), 1e-4, 1e-4, 1e-8)
    assert np.array_equal(np.concatenate(got, axis=1), ref)


# ---------------------------------------------------------------- GPU
CASES = {
    # name: (dim, nx, ny, bc, flux_config, transport key or None, steps)
    "lf_walls": (2, 48, 20, ["slip_wall", "zero_gradient", "slip_wall", "slip_wall"], None, None, 3),
    "lf_periodic": (2, 48, 20, ["periodic"] * 4, None, None, 3),
    "lf_outlet_nsw": (2, 48, 20, ["pressure_outlet", "pressure_outlet", "no_slip_wall", "pressure_outlet"],
                      None, None, 3),
    "hllc_walls": (2, 48, 20, ["slip_wall", "zero_gradient", "slip_wall", "slip_wall"],
                   {"solver_type": "godunov", "interface_reconstruction": "WENO5_JS", "riemann_solver": "HLLC",
                    "viscosity": "off"}, None, 3),
    "visc_walls": (2, 48, 20, ["slip_wall", "zero_gradient", "no_slip_wall", "slip_wall"],
                   {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS", "split_method": "LF",
                    "viscosity": "on"}, "sutherland", 2),
    "lf_1d": (1, 300, None, ["slip_wall", "pressure_outlet"], None, None, 4),
    "lf_1d_periodic": (1, 300, None, ["periodic", "periodic"], None, None, 4),
}
TRANSPORT = {"sutherland": {"viscosity_model": "Sutherland", "thermal_conductivity_model": "Prandtl number",
                            "Pr": 0.72, "species_diffusivity_model": "Lewis number", "Le": 1.0}}


def _case_state(om, case):
    dim, nx, ny = CASES[case][:3]
    if dim == 2:
        U, a = _state2d(om, nx, ny, 5)
    else:
        U, a = _state1d(om, nx, 5)
    return U, a


def _case_bc(case):
    dim, bc = CASES[case][0], CASES[case][3]
    return dict(zip(KEYS2[: 2 * dim], bc))


def _gpu_worker(rank, size, port, out, case, precs):
    from janc_b200.mechanism import DEFAULT_MECHANISM
    from janc_b200.slab import Slab, split_and_distribute_grid
    from janc_b200.solver import Solver
    torch.cuda.set_device(0)
    _init(rank, size, port)
    try:
        om = jo.load_mechanism(DEFAULT_MECHANISM)
        dim, nx, ny, _, fc, tkey, steps = CASES[case]
        U, a = _case_state(om, case)
        slab = Slab()
        Ul = split_and_distribute_grid(U, slab)
        al = split_and_distribute_grid(a, slab)
        dx = 1e-4 if tkey is None else 2e-5
        theta = {"Pb": 101325.0 * 1.2}
        for prec in precs:
            s = Solver(dim, nx // size, ny, dx, dx if dim == 2 else None, _case_bc(case), precision=prec,
                       flux_config=fc, transport_config=TRANSPORT.get(tkey), slab=slab)
            rhs = s.flux_func(Ul, al, dx, dx if dim == 2 else None, 1e-8, theta)
            Upad, Apad = s.boundary_conditions(Ul, al, theta)
            calls0 = s._exchange.calls
            Uo, ao, dts = s.advance(Ul, al, steps, cfl=0.4, theta=theta)
            torch.cuda.synchronize()
            np.savez(os.path.join(out, f"{prec}_{rank}.npz"), rhs=rhs.cpu().numpy(), U=Uo.cpu().numpy(),
                     aux=ao.cpu().numpy(), dts=dts.cpu().numpy(), status=s.status(),
                     calls=s._exchange.calls - calls0 + 1, Upad=Upad.cpu().numpy(), Apad=Apad.cpu().numpy())
            s.close()
    finally:
        dist.destroy_process_group()


def _oracle_run(om, case, size):
    dim, nx, ny, _, fc, tkey, steps = CASES[case]
    U, a = _case_state(om, case)
    dx = 1e-4 if tkey is None else 2e-5
    o = jo.SlabSolver(om, "2D" if dim == 2 else "1D", dx, dx if dim == 2 else None, _case_bc(case), 0.4,
                      flux_config=fc, transport_config=TRANSPORT.get(tkey))
    theta = [{"Pb": 101325.0 * 1.2}] * size
    Us, As = np.split(U, size, axis=1), np.split(a, size, axis=1)
    rhs = o.flux_func(Us, As, dx, dx if dim == 2 else None, 1e-8, theta)
    t, dts = 0.0, []
    for _ in range(steps):
        Us, As, t, dt = o.advance_func(Us, As, t, theta)
        dts.append(dt)
    return rhs, Us, As, dts


@pytest.mark.gpu
@pytest.mark.parametrize("case,size,precs", [
    ("lf_walls", 2, ("fp64_strict", "fp64", "mixed")), ("lf_walls", 3, ("fp64",)),
    ("lf_periodic", 2, ("fp64_strict", "mixed")), ("lf_outlet_nsw", 3, ("fp64_strict",)),
    ("hllc_walls", 2, ("fp64_strict", "mixed")), ("visc_walls", 2, ("fp64_strict", "fp64")),
    ("lf_1d", 3, ("fp64_strict", "mixed")), ("lf_1d_periodic", 2, ("fp64",))])
def test_slabs_vs_oracle(omech, tmp_path, case, size, precs):
    mp.start_processes(_gpu_worker, args=(size, _free_port(), str(tmp_path), case, precs), nprocs=size,
                       start_method="spawn")
    rhs, Us, As, dts = _oracle_run(omech, case, size)
    U0, a0 = _case_state(omech, case)
    Us0, As0 = np.split(U0, size, axis=1), np.split(a0, size, axis=1)
    steps = CASES[case][6]
    for prec in precs:
        tol = {"fp64_strict": 1e-12, "fp64": 1e-10, "mixed": 1e-4}[prec]
        for r in range(size):
            d = np.load(tmp_path / f"{prec}_{r}.npz")
            assert int(d["status"]) == 0
            assert int(d["calls"]) == 1 + 3 * steps  # flux_func, then (CFL + halo) + 2 halos per step
            assert field_err(d["U"], Us[r]) < tol, (prec, r)
            assert field_err(d["U"][:1], Us[r][:1]) < (1e-6 if prec == "mixed" else tol)
            assert field_err(d["aux"], As[r]) < (1e-6 if prec == "mixed" else tol)
            assert np.max(np.abs(d["dts"] - np.array(dts)) / np.array(dts)) < (1e-6 if prec == "mixed" else tol)
            if prec != "mixed":
                assert field_err(d["rhs"], rhs[r]) < (1e-12 if prec == "fp64_strict" else 1e-11)
            if prec == "fp64_strict":  # parallel/boundary.py padding, ring corners included
                Ur, Ar = jo.parallel_boundary_conditions(omech, Us0, As0, r, _case_bc(case), {"Pb": 101325.0 * 1.2})
                np.testing.assert_array_equal(d["Upad"], Ur)
                np.testing.assert_array_equal(d["Apad"], Ar)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["lf_periodic", "lf_walls", "lf_1d_periodic"])
def test_single_slab_in_process(omech, case):
    """One slab without a process group: a periodic x axis closes the ring on
    itself (cell-periodic, unlike the single-domain node-periodic pad)."""
    from janc_b200.slab import Slab
    from janc_b200.solver import Solver
    dim, nx, ny, _, fc, tkey, steps = CASES[case]
    U, a = _case_state(omech, case)
    s = Solver(dim, nx, ny, 1e-4, 1e-4 if dim == 2 else None, _case_bc(case), precision="fp64_strict",
               slab=Slab(rank=0, size=1))
    cu = lambda x: torch.as_tensor(x, device="cuda")  # noqa: E731
    Ug, ag, _ = s.advance(cu(U), cu(a), steps, cfl=0.4, theta={"Pb": 101325.0 * 1.2})
    _, Us, As, _ = _oracle_run(omech, case, 1)
    assert field_err(Ug.cpu().numpy(), Us[0]) < 1e-12
    assert field_err(ag.cpu().numpy(), As[0]) < 1e-12
    if case == "lf_periodic":  # differs from the single-domain (node-periodic) pad
        o = jo.Solver(omech, "2D", 1e-4, 1e-4, _case_bc(case), 0.4)
        Ur, ar, t = U, a, 0.0
        for _ in range(steps):
            Ur, ar, t, _ = o.advance_func(Ur, ar, t)
        assert field_err(Ug.cpu().numpy(), Ur) > 1e-8


# ------------------------------------------------- drop-in Simulator mode
def _sim_config(is_parallel):
    from janc_b200.mechanism import DEFAULT_MECHANISM as MECH
    return {"dimension": "2D", "grid_config": {"dx": 1e-4, "dy": 1e-4},
            "thermo_config": {"thermo_model": "nasa7", "mechanism_directory": MECH},
            "reaction_config": {"is_detailed_chemistry": True, "mechanism_directory": MECH},
            "flux_config": {"solver_type": "flux_splitting", "interface_reconstruction": "WENO5_JS",
                            "split_method": "LF", "viscosity": "off"},
            "boundary_config": dict(zip(KEYS2, ["slip_wall", "zero_gradient", "slip_wall", "slip_wall"])),
            "time_config": {"temporal_evolution_scheme": "TVD_RK3", "t_end": 1.0, "CFL": 0.4},
            "computation_config": {"is_parallel": is_parallel}, "precision": "fp64"}


def test_simulator_parallel_needs_process_group():
    from janc_b200.janc.simulation.set_simulator import Simulator
    if dist.is_initialized():
        pytest.skip("a process group is already initialised")
    with pytest.raises(RuntimeError, match="process group"):
        Simulator(_sim_config(True))


def _sim_worker(rank, size, port, out):
    from janc_b200.janc.parallel.grid_partion import gather_grid, split_and_distribute_grid
    from janc_b200.janc.simulation.set_simulator import Simulator
    from janc_b200.mechanism import DEFAULT_MECHANISM
    torch.cuda.set_device(0)
    _init(rank, size, port)
    try:
        om = jo.load_mechanism(DEFAULT_MECHANISM)
        U, a = _case_state(om, "lf_walls")
        sim = Simulator(_sim_config(True))
        Ul, al = split_and_distribute_grid(U), split_and_distribute_grid(a)
        t = 0.0
        for _ in range(3):
            Ul, al, t, dt = sim.advance_func(Ul, al, t, None)
        Ug = gather_grid(Ul)
        np.savez(os.path.join(out, f"s{rank}.npz"), U=Ug.cpu().numpy(), t=float(t))
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
def test_simulator_is_parallel_vs_oracle(omech, tmp_path):
    """The reference's calling pattern: Simulator with is_parallel, the grid
    split with grid_partion.split_and_distribute_grid, advance_func on the
    slabs, gather_grid at the end."""
    mp.start_processes(_sim_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    _, Us, _, dts = _oracle_run(omech, "lf_walls", 2)
    ref = np.concatenate(Us, axis=1)
    for r in range(2):
        d = np.load(tmp_path / f"s{r}.npz")
        assert field_err(d["U"], ref) < 1e-10
        assert abs(float(d["t"]) - sum(dts)) < 1e-10 * sum(dts)


# ------------------------------------------- rotating detonation, x slabs
RDC_ND = {"P0": 10 * 101325, "T0": 300, "R0": 369, "x0": 0.08}
BC_RDC = {"left_boundary": "periodic", "right_boundary": "periodic",
          "bottom_boundary": "rdc_injector", "top_boundary": "pressure_outlet"}


def _rdc_inputs(golden):
    g = np.load(os.path.join(golden, "step2d_rdc.npz"))
    nx = g["U0"].shape[1]
    x = np.arange(nx)
    Yinj = g["Yinj"][:, None] * (1 + 0.05 * np.cos(2 * np.pi * x / nx))[None, :]  # per-column injection
    return g, Yinj


def _rdc_worker(rank, size, port, out, golden, prec):
    from janc_b200.slab import Slab, split_and_distribute_grid
    from janc_b200.solver import Solver
    torch.cuda.set_device(0)
    _init(rank, size, port)
    try:
        g, Yinj = _rdc_inputs(golden)
        nx, ny = g["U0"].shape[1:]
        dx, dy = float(g["dx"]), float(g["dy"])
        slab = Slab()
        s = Solver(2, nx // size, ny, dx, dy, BC_RDC, nondim_config=RDC_ND, precision=prec, slab=slab)
        theta = {"Yinj": Yinj, "Pb": float(g["Pb"])}  # the global width: each slab takes its columns
        U, a = split_and_distribute_grid(g["U0"], slab), split_and_distribute_grid(g["aux0"], slab)
        rhs = s.flux_func(U, a, dx, dy, 1e-3, theta)
        Uo, ao, dts = s.advance(U, a, 3, cfl=0.4, theta=theta)
        torch.cuda.synchronize()
        np.savez(os.path.join(out, f"rdc{rank}.npz"), rhs=rhs.cpu().numpy(), U=Uo.cpu().numpy(),
                 aux=ao.cpu().numpy(), dts=dts.cpu().numpy(), status=s.status())
    finally:
        dist.destroy_process_group()


@pytest.mark.gpu
@pytest.mark.parametrize("size", [2, 4])
@pytest.mark.parametrize("prec", ["fp64_strict", "fp64"])
def test_rdc_slabs_vs_oracle(golden_dir, tmp_path, size, prec):
    """The injector (bottom) and outlet (top) on every slab, a periodic x
    axis closed through the ring, per-column Yinj cut to each slab
    (the reference's PartitionDict along x), nondimensional units."""
    from janc_b200.mechanism import DEFAULT_MECHANISM
    mp.start_processes(_rdc_worker, args=(size, _free_port(), str(tmp_path), str(golden_dir), prec), nprocs=size,
                       start_method="spawn")
    g, Yinj = _rdc_inputs(str(golden_dir))
    om = jo.load_mechanism(DEFAULT_MECHANISM, RDC_ND)
    dx, dy = float(g["dx"]), float(g["dy"])
    o = jo.SlabSolver(om, "2D", dx, dy, BC_RDC, 0.4)
    cols = np.split(np.arange(g["U0"].shape[1]), size)
    thetas = [{"Yinj": Yinj[:, c][:, :, None], "Pb": float(g["Pb"])} for c in cols]
    Us, As = np.split(g["U0"], size, axis=1), np.split(g["aux0"], size, axis=1)
    rhs = o.flux_func(Us, As, dx, dy, 1e-3, thetas)
    t, dts = 0.0, []
    for _ in range(3):
        Us, As, t, dt = o.advance_func(Us, As, t, thetas)
        dts.append(dt)
    tol = 1e-12 if prec == "fp64_strict" else 1e-10

    def rel(a, b):
        """relative L1 per field; a field below 1e-6 of the largest field's
        size is measured against that floor: the x momentum rhs of this
        nearly x-uniform state is zero in exact arithmetic (2.7e-12 here
        against 1 for its neighbours), so FMA rounding alone moves it by
        1e-5 of itself"""
        mags = [np.sum(np.abs(b[i])) for i in range(b.shape[0])]
        floor = 1e-6 * max(mags)
        return max(np.sum(np.abs(a[i] - b[i])) / max(mags[i], floor) for i in range(b.shape[0]) if mags[i] > 0)
    for r in range(size):
        d = np.load(tmp_path / f"rdc{r}.npz")
        assert int(d["status"]) == 0
        assert rel(d["rhs"], rhs[r]) < (1e-13 if prec == "fp64_strict" else 1e-10)
        assert rel(d["U"], Us[r]) < tol and rel(d["aux"], As[r]) < tol
        assert np.max(np.abs(d["dts"] - np.array(dts)) / np.array(dts)) < tol
