"""The field adjoint: its forward against the engine, its gradient against f64.

The forward, driven by the owner trajectory an engine run records, must land
on the engine's own f32 fields bit for bit. The f32 adjoint gradient of an
MSE loss against the f64 forward at parameters perturbed by 10% must match
PyTorch f64 autograd of a plain stencil and FP64 central finite differences
(h = 1e-6) to 1e-4 relative in the infinity norm over the parameters (and
each component to 1e-3 of itself plus 1e-5 of the largest), and must be bit-identical for every checkpoint
interval, since its sums run in a fixed order.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from glazier_b200.blueprint import CellType, Model, Species, Start

pytestmark = pytest.mark.gpu

# (width, height, depth, cell side, cells per axis, steps, diffusion per species)
CASES = {
    # D 0.3 takes two sub-steps in a plane, 0.1 one; medium along two edges
    "plane": (64, 48, 1, 8, (7, 5, 1), 12, (0.3, 0.1)),
    # D 0.2 takes two sub-steps in 3D (limit 1/6), 0.05 one
    "cube": (16, 16, 12, 4, (4, 4, 2), 7, (0.2, 0.05)),
    # rows of 66 sites, not a multiple of four: the one-site round kernels
    # (the cases above take the four-site ones)
    "odd-rows": (66, 40, 1, 6, (10, 6, 1), 9, (0.3, 0.1)),
}


def _model(case) -> Model:
    w, h, d, side, _, _, diff = CASES[case]
    vt = float(side ** (3 if d > 1 else 2))
    return Model(
        width=w,
        height=h,
        depth=d,
        contact=[0.0, 16.0, 16.0, 16.0, 8.0, 10.0, 16.0, 10.0, 8.0],
        types=[CellType(), CellType(target_volume=vt, lambda_volume=2.0),
               CellType(target_volume=0.75 * vt, lambda_volume=2.0)],
        temperature=10.0,
        neighbour_order=2,
        seed=17,
        species=[Species("virus", diff[0], 0.01, 0.0), Species("interferon", diff[1], 0.02, 0.0)],
        secretion=[[0.0, 0.0], [0.05, 0.0], [0.3, 0.2]],
        uptake=[[0.0, 0.0], [0.02, 0.01], [0.0, 0.03]],
        chemotaxis=[[0.0, 0.0], [0.0, 0.0], [0.0, 0.0]],
    )


def _params(m: Model) -> np.ndarray:
    """D and decay per species, then secretion and uptake per type and species."""
    return np.concatenate([[s.diffusion for s in m.species], [s.decay for s in m.species],
                           np.asarray(m.secretion, dtype=np.float64).reshape(-1),
                           np.asarray(m.uptake, dtype=np.float64).reshape(-1)])


def _torch_forward(params, f0, traj, n_types, shape):
    """The field step in plain f64 PyTorch: rolls for the Laplacian, masks for
    the exchange. `shape` is (depth, height, width). Runs where `f0` lies."""
    import torch

    S = f0.shape[0]
    dim = 3 if shape[0] > 1 else 2
    axes = (0, 1, 2) if dim == 3 else (1, 2)
    D, dec = params[:S], params[S:2 * S]
    sec = params[2 * S:2 * S + n_types * S].reshape(n_types, S)
    upt = params[2 * S + n_types * S:].reshape(n_types, S)
    f = [f0[s].reshape(shape) for s in range(S)]
    for t in range(traj.shape[0]):
        own = torch.from_numpy(traj[t].astype(np.int64)).reshape(shape).to(f0.device)
        owned = own != 255
        idx = torch.where(owned, own, torch.zeros_like(own))
        nxt = []
        for s in range(S):
            dv = float(D[s].detach())
            k = max(1, math.ceil(dv / (1.0 / (2 * dim)))) if dv > 0 else 1
            d, e = D[s] / k, dec[s] / k
            u = f[s]
            for _ in range(k):
                lap = -2.0 * dim * u
                for ax in axes:
                    lap = lap + torch.roll(u, 1, ax) + torch.roll(u, -1, ax)
                u = u + d * lap - e * u
            v1 = u + sec[idx, s]
            v2 = v1 - upt[idx, s] * v1
            nxt.append(torch.where(owned, torch.clamp(v2, min=0.0), u))
        f = nxt
    return torch.stack([x.reshape(-1) for x in f])


@pytest.fixture(scope="module", params=sorted(CASES))
def recorded(request, device):
    """An engine run of the case's steps with two species: its start, initial
    fields, owner trajectory and final f32 fields."""
    from glazier_b200.adjoint import record_trajectory

    case = request.param
    _, _, _, side, (nx, ny, nz), steps, _ = CASES[case]
    m = _model(case)
    st = Start.tiled_grid(m, side, nx, ny, nz)
    st.cell_type[1::3] = 2
    f0 = np.random.default_rng(3).uniform(0.5, 2.0, size=(2, m.sites))
    sim = device.GpuSimulation.from_start(st, f0)
    traj = record_trajectory(sim, steps)
    final = np.stack([sim.field(k) for k in range(2)]).astype(np.float32)
    sim.close()
    assert (traj == 255).any() and (traj == 1).any() and (traj == 2).any()
    return st, f0, traj, final


def _adjoint(st, traj, every):
    from glazier_b200.adjoint import FieldAdjoint

    m = st.model
    return FieldAdjoint(m.width, m.height, m.depth, 2, m.n_types, traj, checkpoint_every=every)


def _shape(st):
    return (st.model.depth, st.model.height, st.model.width)


def test_the_forward_is_the_engines_field_step(recorded):
    import torch

    st, f0, traj, final = recorded
    adj = _adjoint(st, traj, 5)
    out = adj.forward(_params(st.model), torch.from_numpy(f0.astype(np.float32)).cuda())
    assert np.array_equal(out.cpu().numpy(), final)
    adj.close()


def _target(st, traj, f0):
    """The MSE target: the f64 forward at parameters perturbed by 10%
    uniform noise."""
    import torch

    p = _params(st.model)
    perturbed = p * (1.0 + 0.1 * np.random.default_rng(11).uniform(-1.0, 1.0, size=p.size))
    return _torch_forward(torch.from_numpy(perturbed), torch.from_numpy(f0), traj, st.model.n_types, _shape(st))


def _device_gradient(st, traj, f0, target, every):
    import torch

    adj = _adjoint(st, traj, every)
    out = adj.forward(_params(st.model), torch.from_numpy(f0.astype(np.float32)).cuda())
    grad_final = 2.0 * (out - target.to(torch.float32).cuda()) / out.numel()
    gp, gf = adj.backward(grad_final)
    adj.close()
    return gp, gf


def test_the_adjoint_matches_f64_autograd_and_finite_differences(recorded):
    import torch

    st, f0, traj, _ = recorded
    target = _target(st, traj, f0)
    p = _params(st.model)
    gp, _ = _device_gradient(st, traj, f0, target, every=5)
    f0_64 = torch.from_numpy(f0)

    def loss(params):
        out = _torch_forward(params, f0_64, traj, st.model.n_types, _shape(st))
        return ((out - target) ** 2).mean()

    pt = torch.from_numpy(p.copy()).requires_grad_(True)
    loss(pt).backward()
    auto = pt.grad.numpy()
    scale = np.abs(auto).max()
    assert scale > 0
    assert np.abs(gp - auto).max() / scale < 1e-4, (gp, auto)
    live = np.abs(auto) > 0
    assert np.all(gp[~live] == 0.0)
    # component by component, with a floor for sums that nearly cancel
    assert np.all(np.abs(gp - auto) <= 1e-3 * np.abs(auto) + 1e-5 * scale), (gp, auto)

    h = 1e-6
    fd = np.zeros_like(p)
    with torch.no_grad():
        for i in range(p.size):
            up, dn = p.copy(), p.copy()
            up[i] += h
            dn[i] -= h
            fd[i] = (loss(torch.from_numpy(up)).item() - loss(torch.from_numpy(dn)).item()) / (2 * h)
    assert np.abs(gp - fd).max() / np.abs(fd).max() < 1e-4, (gp, fd)


def test_the_gradient_does_not_depend_on_the_checkpoint_interval(recorded):
    st, f0, traj, _ = recorded
    target = _target(st, traj, f0)
    base, gf_base = _device_gradient(st, traj, f0, target, every=traj.shape[0])
    for every in (1, 3, 5):
        gp, gf = _device_gradient(st, traj, f0, target, every=every)
        assert np.array_equal(gp, base)
        assert np.array_equal(gf.cpu().numpy(), gf_base.cpu().numpy())


def test_the_initial_field_gradient_matches_autograd(recorded):
    import torch

    st, f0, traj, _ = recorded
    target = _target(st, traj, f0)
    _, gf = _device_gradient(st, traj, f0, target, every=3)
    f0_64 = torch.from_numpy(f0.copy()).requires_grad_(True)
    out = _torch_forward(torch.from_numpy(_params(st.model)), f0_64, traj, st.model.n_types, _shape(st))
    ((out - target) ** 2).mean().backward()
    auto = f0_64.grad.numpy()
    assert np.abs(gf.cpu().numpy() - auto).max() / np.abs(auto).max() < 1e-4


@pytest.mark.parametrize("n_types", [6, 12])
def test_more_owner_types_give_the_same_gradient(recorded, n_types):
    """The backward keeps its exchange gradients per owner type in registers
    for up to 4 or 8 types and reduces them warp by warp past that: the same
    trajectory declared with unused extra types (their rates zero) gives the
    same gradient for the rates it uses and exactly zero for the others."""
    import torch

    from glazier_b200.adjoint import FieldAdjoint

    st, f0, traj, _ = recorded
    m = st.model
    target = _target(st, traj, f0)
    base, gf_base = _device_gradient(st, traj, f0, target, every=4)
    T, S = m.n_types, 2
    p = _params(m)
    sec = np.zeros((n_types, S))
    upt = np.zeros((n_types, S))
    sec[:T] = np.asarray(m.secretion, dtype=np.float64)
    upt[:T] = np.asarray(m.uptake, dtype=np.float64)
    padded = np.concatenate([p[:2 * S], sec.reshape(-1), upt.reshape(-1)])
    adj = FieldAdjoint(m.width, m.height, m.depth, S, n_types, traj, checkpoint_every=4)
    out = adj.forward(padded, torch.from_numpy(f0.astype(np.float32)).cuda())
    gp, gf = adj.backward(2.0 * (out - target.to(torch.float32).cuda()) / out.numel())
    adj.close()
    g_sec = gp[2 * S:2 * S + n_types * S].reshape(n_types, S)
    g_upt = gp[2 * S + n_types * S:].reshape(n_types, S)
    want_sec = base[2 * S:2 * S + T * S].reshape(T, S)
    want_upt = base[2 * S + T * S:].reshape(T, S)
    scale = np.abs(base).max()
    assert np.array_equal(gp[:2 * S], base[:2 * S])  # diffusion and decay sum the same way
    assert np.abs(g_sec[:T] - want_sec).max() <= 1e-12 * scale
    assert np.abs(g_upt[:T] - want_upt).max() <= 1e-12 * scale
    assert np.all(g_sec[T:] == 0.0) and np.all(g_upt[T:] == 0.0)
    assert torch.equal(gf, gf_base)


def test_the_autograd_function_carries_the_gradient(recorded):
    import torch

    from glazier_b200.adjoint import field_trajectory

    st, f0, traj, _ = recorded
    target = _target(st, traj, f0)
    adj = _adjoint(st, traj, 4)
    params = torch.from_numpy(_params(st.model)).requires_grad_(True)
    fields0 = torch.from_numpy(f0.astype(np.float32)).cuda().requires_grad_(True)
    out = field_trajectory(params, fields0, adj)
    loss = ((out - target.to(torch.float32).cuda()) ** 2).mean()
    loss.backward()
    gp, gf = _device_gradient(st, traj, f0, target, every=4)
    assert np.array_equal(params.grad.numpy(), gp)
    assert torch.equal(fields0.grad, gf)
    adj.close()


def test_bad_arguments_are_refused(recorded):
    import torch

    from glazier_b200.adjoint import FieldAdjoint
    from glazier_b200.engine import GpuError

    st, f0, traj, _ = recorded
    m = st.model
    bad = traj.copy()
    bad[0, 0] = 7  # a type past the three the model has
    with pytest.raises(GpuError, match="owner type"):
        FieldAdjoint(m.width, m.height, m.depth, 2, m.n_types, bad)
    adj = _adjoint(st, traj, 4)
    with pytest.raises(GpuError, match="backward before forward"):
        adj.backward(torch.zeros(adj.shape, device="cuda"))
    p = _params(m)
    p[0] = -0.1
    with pytest.raises(GpuError, match="diffusion and decay"):
        adj.forward(p, torch.from_numpy(f0.astype(np.float32)).cuda())
    adj.close()


def test_the_adjoint_matches_at_the_benchmark_shape(device):
    """The benchmark's field-adjoint workload itself: a 512^2 lattice of 4096
    cells (healthy, infected, immune), the owner trajectory of 50 MCS of the
    engine, two fields from zero, checkpoints every 10 steps, the MSE against
    the f64 forward at parameters perturbed by 10% uniform noise. The f32
    adjoint gradient is within 1e-4 (infinity norm, relative) of f64 autograd
    of the plain stencil, and within 1e-4 of FP64 central differences
    (h = 1e-6) beyond their own distance from autograd, all run on the GPU in
    f64."""
    import torch

    from glazier_b200.adjoint import FieldAdjoint, owner_types
    from glazier_b200.workloads import adjoint_start, uniform01

    start = adjoint_start()
    m = start.model
    assert (m.width, m.height, start.n_cells) == (512, 512, 4096)
    sim = device.GpuSimulation.from_start(start)
    traj = np.empty((50, m.sites), dtype=np.uint8)
    for t in range(50):
        sim.step(1)
        traj[t] = owner_types(sim.labels(), sim.cell_types())
    sim.close()
    p = _params(m)
    noise = np.array([2.0 * uniform01(1, i, 9) - 1.0 for i in range(p.size)])
    shape = (1, m.height, m.width)
    dev = torch.device("cuda", 0)
    f0_64 = torch.zeros((2, m.sites), dtype=torch.float64, device=dev)
    target = _torch_forward(torch.from_numpy(p * (1.0 + 0.1 * noise)).to(dev), f0_64, traj, m.n_types, shape)

    adj = FieldAdjoint(m.width, m.height, 1, 2, m.n_types, traj, checkpoint_every=10)
    out = adj.forward(p, torch.zeros(adj.shape, dtype=torch.float32, device=dev))
    gp, _ = adj.backward(2.0 * (out - target.to(torch.float32)) / out.numel())
    adj.close()

    def loss(params):
        return ((_torch_forward(params, f0_64, traj, m.n_types, shape) - target) ** 2).mean()

    pt = torch.from_numpy(p.copy()).to(dev).requires_grad_(True)
    loss(pt).backward()
    auto = pt.grad.cpu().numpy()
    scale = np.abs(auto).max()
    assert scale > 0
    with torch.no_grad():
        want = _torch_forward(torch.from_numpy(p).to(dev), f0_64, traj, m.n_types, shape)
        drift = float((out.double() - want).abs().max() / want.abs().max())  # the f32 forward's own error
    rel_auto = float(np.abs(gp - auto).max() / scale)
    assert rel_auto < 1e-4, f"adjoint vs f64 autograd {rel_auto:.3e} (f32 forward off by {drift:.3e})"

    h = 1e-6
    fd = np.zeros_like(p)
    with torch.no_grad():
        for i in range(p.size):
            if auto[i] == 0.0 and gp[i] == 0.0:
                continue  # a rate no site uses (the medium's, say): both sides exactly zero
            up, dn = p.copy(), p.copy()
            up[i] += h
            dn[i] -= h
            fd[i] = (loss(torch.from_numpy(up).to(dev)).item() - loss(torch.from_numpy(dn).to(dev)).item()) / (2 * h)
    # At this shape the differences carry an error of their own: exact f64
    # autograd is about 2.2e-4 (relative, infinity norm) from them, and the
    # adjoint, within 1e-4 of autograd, sits as close to them as autograd
    # does. The bar is the differences' own distance from autograd plus 1e-4.
    rel_fd = float(np.abs(gp - fd).max() / np.abs(fd).max())
    auto_fd = float(np.abs(auto - fd).max() / np.abs(fd).max())
    assert rel_fd < auto_fd + 1e-4, f"adjoint vs central differences {rel_fd:.3e} (autograd vs them {auto_fd:.3e})"
