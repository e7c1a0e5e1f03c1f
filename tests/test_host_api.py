"""Solver.advance_host: independent host states through the device with the
copies overlapped with the steps (copy-in, steps and copy-out of
neighbouring items on three streams).  The results must equal the plain
per-item advance bit for bit, whatever the overlap."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from oracle import janc_oracle as jo  # noqa: E402


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_advance_host_matches_advance(prec):
    from janc_b200.mechanism import DEFAULT_MECHANISM
    from janc_b200.solver import Solver
    om = jo.load_mechanism(DEFAULT_MECHANISM)
    nx, ny = 64, 48
    bc = {"left_boundary": "slip_wall", "right_boundary": "zero_gradient",
          "bottom_boundary": "slip_wall", "top_boundary": "slip_wall"}
    s = Solver(2, nx, ny, 1e-4, 1e-4, bc, precision=prec)
    rng = np.random.default_rng(0)
    ins, outs = [], []
    for k in range(5):
        P = np.full((1, nx, ny), 101325.0)
        T = np.full((1, nx, ny), 300.0)
        P[:, :4 + k] = 30 * 101325.0
        T[:, :4 + k] = 3000.0 * (1 + 0.05 * rng.uniform(-1, 1, (1, 4 + k, ny)))
        U, a = jo.state_from_PTY(om, P, T, np.tile(jo.stoich_Y(om, 1.0)[:, None, None], (1, nx, ny)))
        ins.append((torch.as_tensor(U).pin_memory(), torch.as_tensor(a).pin_memory()))
        outs.append((torch.empty_like(ins[-1][0]).pin_memory(), torch.empty_like(ins[-1][1]).pin_memory()))
    s.advance_host(ins, outs, 2, cfl=0.3)
    torch.cuda.synchronize()
    for (hU, ha), (oU, oa) in zip(ins, outs):
        U, a, _ = s.advance(hU.cuda(), ha.cuda(), 2, cfl=0.3)
        assert torch.equal(U.cpu(), oU) and torch.equal(a.cpu(), oa)
    with pytest.raises(ValueError):
        s.advance_host([(ins[0][0].clone(), ins[0][1])], outs[:1], 1, cfl=0.3)  # not pinned
