"""Warm-start network: its tensor-core convolution layer (forward, input and
weight gradients through torch autograd) against the FP64 CPU oracle in
oracle/conv_oracle.py, and the predictor's plumbing on the SIMP cantilever.

Tolerances: forward 1e-2 of max |ref| (BF16 output); gradients 1e-2 of max
|ref| (BF16 dy / dx); bias gradient 1e-3."""
import importlib

import numpy as np
import pytest
import torch

from oracle import conv_oracle as co


def _ws():
    return importlib.import_module("jax_fem_b200.warmstart")


@pytest.mark.gpu
@pytest.mark.parametrize("N,D,H,W,Cin,Cout,relu", [(2, 8, 16, 16, 16, 32, True), (8, 4, 2, 2, 32, 16, False),
                                                    (2, 4, 8, 8, 64, 64, True)])
def test_conv_layer_gradients_match_oracle(pkg, cuda, N, D, H, W, Cin, Cout, relu):
    ws = _ws()
    g = torch.Generator().manual_seed(Cin + Cout)
    x = torch.randn(N, D, H, W, Cin, generator=g).to(cuda, torch.bfloat16).requires_grad_(True)
    w = (torch.randn(Cout, 27, Cin, generator=g) / (27 * Cin) ** 0.5).to(cuda).requires_grad_(True)
    b = torch.randn(Cout, generator=g).to(cuda).requires_grad_(True)
    y = ws.ConvTC.apply(x, w, b, relu)
    dy = torch.randn(y.shape, generator=g).to(cuda, torch.bfloat16)
    y.backward(dy)
    # oracle on exactly the operands the kernels saw (bf16-rounded x, w, dy)
    xn = x.detach().float().cpu().numpy().astype(np.float64)
    wn = w.detach().to(torch.bfloat16).float().cpu().numpy().astype(np.float64)
    bn = b.detach().cpu().numpy().astype(np.float64)
    yr = co.conv3d(xn, wn, bn, relu)
    dx, dw, db = co.conv3d_backward(xn, wn, dy.float().cpu().numpy().astype(np.float64),
                                    y.detach().float().cpu().numpy(), relu)
    assert np.abs(y.detach().float().cpu().numpy() - yr).max() <= 1e-2 * np.abs(yr).max()
    assert np.abs(x.grad.float().cpu().numpy() - dx).max() <= 1e-2 * np.abs(dx).max()
    assert np.abs(w.grad.cpu().numpy() - dw).max() <= 1e-2 * np.abs(dw).max()
    assert np.abs(b.grad.cpu().numpy() - db).max() <= 1e-3 * np.abs(db).max()


@pytest.mark.gpu
def test_network_trains_and_predicts(pkg, cuda):
    """Tiny synthetic regression: the U-Net's loss decreases under Adam, and
    the predictor returns a full displacement vector honouring the clamp."""
    ws = _ws()
    torch.manual_seed(0)
    net = ws.WarmStartNet(seed=3).to(cuda)
    B = 8
    g = torch.Generator().manual_seed(2)
    rho = 0.01 + 0.99 * torch.rand(B, ws.NX, ws.NY, ws.NZ, generator=g)
    load = torch.zeros(B, ws.NX + 1, ws.NY + 1, ws.NZ + 1)
    load[:, -1, :, :4] = 1.0
    target = torch.randn(B, ws.CD, ws.CH, ws.CW, 3, generator=g) * 0.1
    hist = ws.train(net, {"rho": rho, "load": load, "target": target}, epochs=8, batch=8, lr=3e-3, log=None)
    assert hist[-1] < hist[0]
    prob = ws.cantilever_problem(z0=0.0)
    prob.set_params(ws.cell_rho_to_torch(rho[0], cuda))
    u = ws.Predictor(net)(prob)
    assert u.shape == (prob.num_total_dofs_all_vars,) and bool(torch.isfinite(u).all())
    mask, ubc = prob.dirichlet_device()
    assert float((u[mask.bool()] - ubc[mask.bool()]).abs().max()) == 0.0


@pytest.mark.gpu
def test_trained_network_effect_on_heldout(pkg, cuda):
    """What the committed trained network does on held-out SIMP cantilevers
    (seeds disjoint from training), measured against the zero start.

    Asserted, from measurements of this network:
    - the raw prediction's relative displacement error ||u* - d|| / ||u*||
      is below 0.1 (the zero start's is 1): the network has learned the
      displacement field to a few per cent;
    - the Galerkin-scaled start's energy-norm error ||u* - u0||_K / ||u*||_K
      is below 1 (the zero start's is 1);
    - to the same absolute residual (1e-8 of the zero-start residual) the
      learned start takes at most 5 % more Krylov iterations than the zero
      start, on the FP64 path and on the mixed path (FP32 CG inside FP64
      refinement).
    Not asserted, because it does not hold: a gain at rel.res 1e-8.  The
    raw prediction's strain is noisy (its energy-norm error is above 1), so
    the Galerkin factor shrinks it to an energy-norm error of about 0.9,
    and CG, which removes the smooth error no later than the rest, gains
    about nothing at 1e-8 (measured 1110 vs 1108 iterations on the FP64
    path).  This is the measured ceiling of a coarse-grid (2h) prediction
    of this high-contrast field."""
    import os
    ws = _ws()
    path = os.path.join(os.path.dirname(ws.__file__), "weights", "warmstart_simp60.pt")
    net, meta = ws.load(path, cuda)
    pred, raw = ws.Predictor(net), ws.Predictor(net, galerkin=False)
    prob = ws.cantilever_problem()
    g = torch.Generator().manual_seed(424242)
    lin = {"cg": {"precond": "block_jacobi", "rtol": "adaptive", "atol": 0.0, "maxiter": 50000}}
    l2, energy = [], []
    iters = {f"{p}_{a}": [] for p in ("fp64", "mixed") for a in ("zero", "learned")}
    for _ in range(6):
        rho = ws.random_density(g)
        prob.set_patch(float(torch.randint(0, ws.NZ - 2, (1,), generator=g).item()))
        prob.set_params(ws.cell_rho_to_torch(rho, cuda))
        ref = pkg.solver(prob, {"newton": {"rel_tol": 1e-10, "tol": 1e-30, "linear": lin}})[0].reshape(-1)
        K = prob.A  # FP64 eliminated tangent of the linear problem (assembled by the solve)
        e = ref - raw(prob)
        l2.append((e.norm() / ref.norm()).item())
        e = ref - pred(prob)
        energy.append((torch.dot(e, K.matvec(e)) / torch.dot(ref, K.matvec(ref))).sqrt().item())
        refine = {"cg": dict(lin["cg"], reliable_delta=0.0)}
        for prec, plin in (("fp64", lin), ("mixed", refine)):
            for arm, start in (("zero", None), ("learned", pred)):
                (_,), info = pkg.solver(prob, {"newton": {"rel_tol": 1e-8, "tol": 1e-30, "linear": plin,
                                                           "precision": prec, "rel_tol_reference": "zero",
                                                           "warm_start": start, "return_info": True}})
                iters[f"{prec}_{arm}"].append(sum(info["krylov_iters"]))
    print(f"raw prediction L2 error {np.round(l2, 4)}; Galerkin start energy-norm error {np.round(energy, 4)}; "
          f"krylov {iters}")
    assert max(l2) < 0.1
    assert max(energy) < 1.0
    for prec in ("fp64", "mixed"):
        assert sum(iters[f"{prec}_learned"]) <= 1.05 * sum(iters[f"{prec}_zero"]), iters
