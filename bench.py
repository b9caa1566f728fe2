"""Benchmark of the HEX8 assemble-and-solve path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--n N]

Default workload (one step): the 50^3 compressible Neo-Hookean cube
(397,953 dofs, E=10, nu=0.3), x=0 clamped, x=1 face rotated 30 degrees about
the x-axis in 5 load steps, Newton to ||R||/||R0|| <= 1e-8 at every step --
solved with the headline path (HEADLINE_PRECISION / HEADLINE_LINEAR: FP64
residual, FP32 tangent, FP64 CG over an FP32 multigrid V-cycle).  The same
workload on the plain FP64 path and other variants is timed in the same run.
One JSON line on stdout (rank 0).

``--impl reference`` times the reference's method on the host cores: the
FP64 C++/OpenMP restatement in oracle/fem_cpu.cpp (the reference itself
needs JAX, basix and PETSc, which are not installed), one load step of the
same twist per step, every load step solved in full.

Under torchrun (N>1) each rank solves its own replica of the workload (the
path does not shard: replicas only); the time is the max over ranks.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

import numpy as np
import torch

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from __graft_entry__ import load_package  # noqa: E402

METRIC = "time-to-solve @rel.res 1e-8: mixed+learned vs plain on B200; assembly DoF/s"


# ---------------------------------------------------------------------------
# workloads (shapes and values of the benchmark configurations)
# ---------------------------------------------------------------------------

def _left(p):
    return np.isclose(p[0], 0.0, atol=1e-5)


def _right(p):
    return np.isclose(p[0], 1.0, atol=1e-5)


def _zero(p):
    return 0.0 * p[0]


def rotation_bc(theta):
    """x=0 clamped; x=1: u_x=0, (y,z) rotated by theta about (y,z)=(0.5,0.5).
    The faces' location functions are defined once, as a user script would;
    only the value functions change with the load step."""
    c, s = math.cos(theta), math.sin(theta)

    def uy(p):
        return 0.5 + (p[1] - 0.5) * c - (p[2] - 0.5) * s - p[1]

    def uz(p):
        return 0.5 + (p[1] - 0.5) * s + (p[2] - 0.5) * c - p[2]

    return [[_left] * 3 + [_right] * 3, [0, 1, 2] * 2, [_zero, _zero, _zero, _zero, uy, uz]]


def nh_problem(pkg, n=50, E=10.0, nu=0.3):
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])

    class HyperElasticity(pkg.Problem):
        def get_tensor_map(self):
            return pkg.NeoHookean(E, nu)

    return HyperElasticity(mesh, vec=3, dim=3, dirichlet_bc_info=rotation_bc(0.0))


# the headline solver: mixed precision (FP64 residual, FP32 tangent) with CG
# in FP64 over an FP32 geometric-multigrid V-cycle, Eisenstat-Walker forcing,
# coarse operators shared by up to 4 Newton solves of one twist
HEADLINE_PRECISION = "mixed"
HEADLINE_LINEAR = {"cg": {"precond": "gmg", "rtol": "adaptive", "atol": 0.0, "maxiter": 2000, "mg_lag": 4}}


def nh_solve(pkg, prob, precision, steps=5, total_deg=30.0, linear=None, extrapolate=True):
    """The load-stepped solve; returns (sol, per-step infos).  Each call is
    an independent solve: multigrid coarse operators kept from an earlier
    call are not reused (its first Newton solve forms them afresh)."""
    linear = linear or {"cg": {"precond": "block_jacobi", "rtol": 1e-10, "atol": 1e-10, "maxiter": 20000}}
    pkg.reset_multigrid(prob)
    infos, prev, prev2 = [], None, None
    for k in range(1, steps + 1):
        prob.fes[0].update_Dirichlet_boundary_conditions(rotation_bc(math.radians(total_deg * k / steps)))
        guess = None
        if prev is not None:
            guess = prev if (prev2 is None or not extrapolate) else 2.0 * prev - prev2
        opts = {"newton": {"rel_tol": 1e-8, "tol": 1e-12, "precision": precision, "linear": linear,
                           "initial_guess": guess, "return_info": True}}
        (sol,), info = pkg.solver(prob, opts)
        infos.append(info)
        prev2, prev = prev, sol.reshape(-1).clone()
    return sol, infos


def element_problem(pkg, ele, n):
    """The Neo-Hookean twist on an n^3 box of another element type."""
    import importlib
    gm = importlib.import_module("jax_fem_b200.generate_mesh")
    m = gm.box_mesh_gmsh(n, n, n, 1.0, 1.0, 1.0, None, ele)
    mesh = pkg.Mesh(m.points, m.cells_dict[gm.get_meshio_cell_type(ele)], ele)

    class HyperElasticity(pkg.Problem):
        def get_tensor_map(self):
            return pkg.NeoHookean(10.0, 0.3)

    return HyperElasticity(mesh, vec=3, dim=3, ele_type=ele, dirichlet_bc_info=rotation_bc(0.0))


# element type -> box divisions: 51^3 nodes (397,953 dofs, the HEX8 50^3
# node count) for TET4, TET10 and HEX27; HEX20 has no face or cell nodes
ELEMENT_BOXES = (("TET4", 50), ("TET10", 25), ("HEX27", 25), ("HEX20", 25))


def element_bench(pkg, device):
    """General-element kernel: Neo-Hookean assembly (FP64 residual with the
    FP64 or FP32 tangent) and the 5-step twist solved in mixed precision,
    with block-Jacobi CG (adaptive forcing) and with the multigrid
    preconditioner (the lattice hierarchy for TET4 boxes, p-multigrid to the
    corner-node lattice for the quadratic types)."""
    out = {}
    for ele, n in ELEMENT_BOXES:
        prob = element_problem(pkg, ele, n)
        dv = prob.dev()
        nd = dv.ndofs
        u = torch.zeros(nd, dtype=torch.float64, device=device)
        res = torch.empty_like(u)
        A64, A32 = dv.new_matrix(torch.float64), dv.new_matrix(torch.float32)
        t64 = time_kernel(lambda: prob.assemble(u, res=res, vals=A64.vals), reps=5)
        t32 = time_kernel(lambda: prob.assemble(u, res=res, vals=A32.vals, fp32=True), reps=5)
        nen, nq = dv.nen, prob.fes[0].num_quads
        # cells: connectivity + node coordinates + u; the tangent values once; the residual
        asm_bytes = dv.num_cells * nen * (4 + 3 * 8 + 3 * 8) + dv.nnzb * 9 * 8 + nd * 8
        del A64, A32
        lin = {"cg": {"precond": "block_jacobi", "rtol": "adaptive", "atol": 0.0, "maxiter": 20000}}
        nh_solve(pkg, prob, "mixed", linear=lin)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, infos = nh_solve(pkg, prob, "mixed", linear=lin)
        e1.record()
        torch.cuda.synchronize()
        hbm, _ = peaks()
        # multigrid: the lattice hierarchy (TET4 boxes), p-multigrid to the corner lattice (quadratic cells)
        lin_mg = {"cg": {"precond": "gmg", "rtol": "adaptive", "atol": 0.0, "mg_lag": 4}}
        nh_solve(pkg, prob, "mixed", linear=lin_mg)
        torch.cuda.synchronize()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record()
        _, infos_mg = nh_solve(pkg, prob, "mixed", linear=lin_mg)
        e3.record()
        torch.cuda.synchronize()
        gmg = {"twist_solve_s": round(e2.elapsed_time(e3) * 1e-3, 4),
               "newton_iters": sum(i["newton_iters"] for i in infos_mg),
               "krylov_iters": sum(sum(i["krylov_iters"]) for i in infos_mg)}
        out[ele] = {"cells": dv.num_cells, "dofs": nd, "nodes_per_cell": nen, "quad_points": nq, "nnzb": dv.nnzb,
                    "assembly_us": {"fp64": round(t64 * 1e6, 1), "fp32": round(t32 * 1e6, 1)},
                    "assembly_dofs_per_s": {"fp64": round(nd / t64), "fp32": round(nd / t32)},
                    "assembly_hbm_frac_fp64": round(asm_bytes / t64 / 1e9 / hbm, 3),
                    "twist_solve_s": round(e0.elapsed_time(e1) * 1e-3, 4),
                    "newton_iters": sum(i["newton_iters"] for i in infos),
                    "krylov_iters": sum(sum(i["krylov_iters"]) for i in infos)}
        out[ele]["multigrid_mixed"] = gmg
        del prob, dv
        torch.cuda.empty_cache()
    return out


def amg_bench(pkg, device, n=12):
    """precond='amg' (smoothed-aggregation AMG, hierarchy formed on the host)
    on a mesh where the lattice multigrid cannot run: the Neo-Hookean twist
    on an n^3 TET10 box whose nodes are randomly renumbered, FP64, against
    block-Jacobi CG.  Reports the solve time and, for AMG, the host setup
    time inside it (wall clock, included in the solve time)."""
    import importlib
    gm = importlib.import_module("jax_fem_b200.generate_mesh")
    m = gm.box_mesh_gmsh(n, n, n, 1.0, 1.0, 1.0, None, "TET10")
    cells = m.cells_dict[gm.get_meshio_cell_type("TET10")]
    perm = np.random.default_rng(3).permutation(len(m.points))
    inv = np.argsort(perm)
    mesh = pkg.Mesh(m.points[perm], inv[cells], "TET10")

    class HyperElasticity(pkg.Problem):
        def get_tensor_map(self):
            return pkg.NeoHookean(10.0, 0.3)

    out = {"workload": f"neo-hookean twist, {n}^3 TET10 box, nodes randomly renumbered (no lattice), FP64"}
    for name, pc in (("amg", "amg"), ("block_jacobi", "block_jacobi")):
        prob = HyperElasticity(mesh, vec=3, dim=3, ele_type="TET10", dirichlet_bc_info=rotation_bc(0.0))
        lin = {"cg": {"precond": pc, "rtol": "adaptive", "atol": 0.0, "maxiter": 20000}}
        nh_solve(pkg, prob, "fp64", linear=lin)  # warm-up
        mgc = prob.dev().__dict__.get("_mg", {}).get("amg")
        s0 = getattr(mgc, "setup_seconds", 0.0)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, infos = nh_solve(pkg, prob, "fp64", linear=lin)
        torch.cuda.synchronize()
        r = {"twist_solve_s": round(time.perf_counter() - t0, 4), "newton_iters": sum(i["newton_iters"] for i in infos),
             "krylov_iters": sum(sum(i["krylov_iters"]) for i in infos), "dofs": prob.num_total_dofs_all_vars}
        if mgc is not None:
            r["host_setup_s"] = round(mgc.setup_seconds - s0, 4)
            r["levels"] = len(mgc.levels) + 1
        out[name] = r
    return out


def _nh_universal(E=10.0, nu=0.3):
    """The compressible Neo-Hookean weak form written as a torch universal
    kernel (the reference's form of a user-written weak form)."""
    mu = E / (2.0 * (1.0 + nu))
    kappa = E / (3.0 * (1.0 - 2.0 * nu))

    def kernel(sol, x, sg, jxw, vg):
        F = torch.einsum("ai,qaj->qij", sol.reshape(-1, 3), sg) + torch.eye(3, dtype=sol.dtype, device=sol.device)
        J = torch.linalg.det(F)
        H = torch.linalg.inv(F).transpose(1, 2)
        I1 = torch.einsum("qij,qij->q", F, F)
        m = mu * J ** (-2.0 / 3.0)
        P = m[:, None, None] * (F - (I1 / 3.0)[:, None, None] * H) + (kappa * J * (J - 1.0))[:, None, None] * H
        return torch.einsum("qij,qaj->ai", P, vg[:, :, 0, :]).reshape(-1)

    return kernel


def cell_path_bench(pkg, device, n=30):
    """Cost of the cell-kernel path: the Neo-Hookean twist on an n^3 HEX8
    box with the weak form as a torch universal kernel (vmap of jacfwd, then
    the CUDA scatter into a scalar CSR tangent), against the registered
    NeoHookean CUDA kernel on the same box."""
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])

    class Universal(pkg.Problem):
        def get_universal_kernel(self):
            return _nh_universal()

    class Law(pkg.Problem):
        def get_tensor_map(self):
            return pkg.NeoHookean(10.0, 0.3)

    out = {"workload": f"neo-hookean twist, {n}^3 HEX8 box, weak form as a torch universal kernel"}
    for name, cls in (("cell_path", Universal), ("law_kernel", Law)):
        prob = cls(mesh, vec=3, dim=3, dirichlet_bc_info=rotation_bc(0.0))
        dv = prob.dev()
        u = torch.zeros(dv.ndofs, dtype=torch.float64, device=device)
        res = torch.empty_like(u)
        A = dv.new_matrix(torch.float64)
        t = time_kernel(lambda: prob.assemble(u, res=res, vals=A.vals), reps=5)
        lin = {"bicgstab": {"precond": "jacobi", "rtol": "adaptive", "atol": 0.0, "maxiter": 20000}}
        nh_solve(pkg, prob, "fp64", linear=lin)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, infos = nh_solve(pkg, prob, "fp64", linear=lin)
        e1.record()
        torch.cuda.synchronize()
        out[name] = {"dofs": dv.ndofs, "assembly_ms": round(t * 1e3, 3),
                     "twist_solve_s": round(e0.elapsed_time(e1) * 1e-3, 4),
                     "newton_iters": sum(i["newton_iters"] for i in infos),
                     "krylov_iters": sum(sum(i["krylov_iters"]) for i in infos)}
        del prob, dv, A
        torch.cuda.empty_cache()
    return out


def j2_run(pkg, n=40, increments=10, precision="fp64", linear=None):
    """40^3 J2 cube with hardening: u_x(x=1) ramped to 0.02 over the increments,
    Newton to 1e-8 per increment, state committed after each."""
    m = pkg.box_mesh(n, n, n, 1.0, 1.0, 1.0)
    mesh = pkg.Mesh(m.points, m.cells_dict["hexahedron"])
    C = len(mesh.cells)
    left = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    right = lambda p: np.isclose(p[0], 1.0, atol=1e-5)  # noqa: E731
    bc = [[left] * 3 + [right], [0, 1, 2, 0], [lambda p: 0.0 * p[0]] * 4]

    class J2(pkg.Problem):
        def get_tensor_map(self):
            return pkg.J2Plasticity(70e3, 0.3, 250.0, 700.0)

    prob = J2(mesh, vec=3, dim=3, dirichlet_bc_info=bc)
    dev = prob.dev().device
    z = lambda *sh: torch.zeros(*sh, dtype=torch.float64, device=dev)  # noqa: E731
    prob.internal_vars = [z(C, 8, 3, 3), z(C, 8, 3, 3), z(C, 8)]
    linear = linear or {"cg": {"precond": "block_jacobi", "rtol": 1e-10, "atol": 0.0, "maxiter": 20000}}
    sol, newton, krylov = None, 0, 0
    for k in range(1, increments + 1):
        bc[2][-1] = (lambda v: (lambda p: v + 0.0 * p[0]))(0.02 * k / increments)
        prob.fes[0].update_Dirichlet_boundary_conditions(bc)
        (sol,), info = pkg.solver(prob, {"newton": {"rel_tol": 1e-8, "tol": 1e-14, "precision": precision,
                                                    "linear": linear, "initial_guess": sol,
                                                    "return_info": True}})
        prob.update_j2_state(sol)
        newton += info["newton_iters"]
        krylov += sum(info["krylov_iters"])
    return sol, newton, krylov


# ---------------------------------------------------------------------------
# measurement helpers
# ---------------------------------------------------------------------------

class ClockSampler:
    """nvidia-smi sampling of SM clocks / throttle reasons during a region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"clocks_{os.getpid()}.csv")

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(buf):
    buf.add_(1.0)  # writes 256 MB > 126 MB L2


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def bf16_peak():
    """Dense BF16 TFLOP/s for a kernel timed alone (burst figure)."""
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["bf16_tflops"]), "measured"
    except (OSError, KeyError, ValueError):
        return 1590.0, "fallback"


def conv_bench(pkg, device):
    """Throughput of the tensor-core kernels of the warm-start network
    (tcgen05, BF16 operands, FP32 accumulation in TMEM): the 3x3x3 forward
    convolution at every U-Net layer shape of a 16-sample training batch,
    at one large layer (128 -> 128 channels on 16 x 32^3 voxels), and the
    weight-gradient GEMM at the largest U-Net layer and at the large layer.
    CUDA events around 20 back-to-back launches after 3 warm-up ones."""
    import importlib
    ws = importlib.import_module("jax_fem_b200.warmstart")
    nat = pkg._native
    lib = nat.lib()
    peak, kind = bf16_peak()
    g = torch.Generator(device=device).manual_seed(0)
    B = 16
    dims = {1: (ws.CD, ws.CH, ws.CW), 2: (ws.CD // 2, ws.CH // 2, ws.CW // 2),
            3: (ws.CD // 4, ws.CH // 4, ws.CW // 4), 4: (ws.CD // 8, ws.CH // 8, ws.CW // 8)}
    level = {"e1": 1, "e2": 2, "e3": 3, "e4": 4, "d3": 3, "d2": 2, "d1": 1, "ou": 1}
    shapes = [(name, B, *dims[level[name[:2]]], cin, cout) for name, cin, cout in ws.WarmStartNet.LAYERS]
    shapes.append(("large_128x128", B, 32, 32, 32, 128, 128))
    out = {"peak_tflops": peak, "peak_kind": kind, "fwd": {}, "wgrad": {}}
    for name, N, D, H, W, cin, cout in shapes:
        x = torch.randn(N, D, H, W, cin, generator=g, device=device).to(torch.bfloat16)
        w = (0.05 * torch.randn(cout, 27, cin, generator=g, device=device)).to(torch.bfloat16)
        b = torch.zeros(cout, dtype=torch.float32, device=device)
        y = torch.empty(N, D, H, W, cout, dtype=torch.bfloat16, device=device)

        def fwd():
            nat.check(lib.fem_conv3d_fwd_bf16(nat.ptr(x), nat.ptr(w), nat.ptr(b), nat.ptr(y), N, D, H, W, cin,
                                              cout, 1, nat.stream_ptr()), "conv3d_fwd")

        t = time_kernel(fwd)
        V = N * D * H * W
        fl = 2.0 * V * 27 * cin * cout
        out["fwd"][name] = {"shape": [N, D, H, W, cin, cout], "us": round(t * 1e6, 2),
                            "tflops": round(fl / t / 1e12, 2), "frac": round(fl / t / 1e12 / peak, 4)}
    for name, N, D, H, W, cin, cout in (("e1b", B, ws.CD, ws.CH, ws.CW, 16, 16),
                                        ("large_128x128", 4, 32, 32, 32, 128, 128)):
        V = N * D * H * W
        M = 27 * cin
        col = torch.randn(M, V, generator=g, device=device).to(torch.bfloat16)
        dzt = torch.randn(cout, V, generator=g, device=device).to(torch.bfloat16)
        dwt = torch.zeros(M, cout, dtype=torch.float32, device=device)
        mtiles = (M + 127) // 128
        split = int(max(1, min(max(1, V // 64), math.ceil(2 * 148 / mtiles))))

        def wgrad():
            nat.check(lib.fem_gemm_bf16_tn_f32(nat.ptr(col), nat.ptr(dzt), nat.ptr(dwt), M, cout, V, cout, split,
                                               nat.stream_ptr()), "wgrad")

        t = time_kernel(wgrad)
        fl = 2.0 * M * cout * V
        out["wgrad"][name] = {"M": M, "N": cout, "K": V, "split_k": split, "us": round(t * 1e6, 2),
                              "tflops": round(fl / t / 1e12, 2), "frac": round(fl / t / 1e12 / peak, 4)}
        del col, dzt, dwt
    err = nat._c.c_int(0)
    nat.check(lib.fem_tc_error(nat._c.byref(err), 1), "tc_error")
    out["tc_error_flag"] = err.value
    try:
        meta = torch.load(os.path.join(ROOT, "jax-fem_b200", "weights", "warmstart_simp60.pt"),
                          map_location="cpu", weights_only=False).get("meta", {})
        if meta.get("train_s") is not None and meta.get("epochs"):
            out["committed_network_training"] = {"epochs": meta["epochs"], "train_s": round(meta["train_s"], 1),
                                                 "s_per_epoch": round(meta["train_s"] / meta["epochs"], 2),
                                                 "n_train": meta.get("n_train")}
    except Exception:  # noqa: BLE001 - optional context only
        pass
    return out


def time_kernel(fn, reps=20):
    """Average duration of fn() with CUDA events on the current stream."""
    st = torch.cuda.current_stream()
    for _ in range(3):
        fn()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(st)
    for _ in range(reps):
        fn()
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps * 1e-3


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def reduce_max(x, world, device):
    """Max of a per-rank time over the replicas (the whole-job time): an
    all-reduce of one scalar, the bench's only collective."""
    if world == 1:
        return x
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def run_ours(args, rank, world, device):
    pkg = load_package()
    nat = pkg._native
    prob = nh_problem(pkg, n=args.n)
    ndofs = prob.num_total_dofs_all_vars
    dv = prob.dev()
    l2 = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)

    def timed(precision, K, W, linear):
        for _ in range(W):
            nh_solve(pkg, prob, precision, linear=linear)
        torch.cuda.synchronize()
        times, infos = [], None
        for _ in range(K):
            flush_l2(l2)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            _, infos = nh_solve(pkg, prob, precision, linear=linear)
            e1.record()
            torch.cuda.synchronize()
            times.append(e0.elapsed_time(e1) * 1e-3)
        return times, infos

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        return reduce_max(x, world, device)

    tight = {"cg": {"precond": "block_jacobi", "rtol": 1e-10, "atol": 1e-10, "maxiter": 20000}}
    adaptive = {"cg": {"precond": "block_jacobi", "rtol": "adaptive", "atol": 0.0, "maxiter": 20000}}
    refine = {"cg": dict(adaptive["cg"], reliable_delta=0.0)}
    refm = {"jax_solver": {}}  # the reference's default linear solver: BiCGSTAB + Jacobi, tol = atol = 1e-10
    # multigrid: coarse operators shared by up to 4 Newton solves (re-formed
    # sooner when convergence slows); the finest level takes every tangent
    gmg = HEADLINE_LINEAR
    variants = {  # name -> (precision, linear options)
        "reference_method_fp64": ("fp64", refm),  # the reference's exact Newton + linear settings on the GPU
        "plain_fp64": ("fp64", tight),            # tight linear solves, CG + 3x3 block-Jacobi
        "plain_fp64_adaptive": ("fp64", adaptive),
        "mixed_tight": ("mixed", tight),
        "mixed_refinement": ("mixed", refine),    # FP32 CG restarted inside FP64 iterative refinement
        "mixed": ("mixed", adaptive),             # FP32 tangent/Krylov with reliable updates
        "plain_fp64_gmg": ("fp64", gmg),          # FP64 CG + FP64 multigrid V-cycle
        "mixed_gmg": (HEADLINE_PRECISION, gmg),   # headline: FP64 CG + FP32 multigrid V-cycle
    }
    HEAD = "mixed_gmg"
    results = {}
    sampler = ClockSampler(torch.cuda.current_device())
    for name, (prec, lin) in variants.items():
        barrier()
        if name == HEAD:
            l0 = nat.launch_count()
            sampler.start()
        times, infos = timed(prec, args.steps, args.warmup, lin)
        if name == HEAD:
            clocks = sampler.stop()
            launches = (nat.launch_count() - l0) * args.steps // (args.steps + args.warmup)
        barrier()
        results[name] = (max_over_ranks(statistics.mean(times)), infos)
    t_mixed = results[HEAD][0]
    t_plain = results["plain_fp64"][0]
    mixed_infos, plain_infos = results[HEAD][1], results["plain_fp64"][1]

    # e2e through the public API with host buffers: the step's inputs (node
    # coordinates and Dirichlet values) come from pinned host memory, the
    # solution goes back to pinned host memory.
    pts_h = torch.from_numpy(prob.mesh.points.copy()).pin_memory()
    sol_h = torch.empty(ndofs, dtype=torch.float64).pin_memory()
    e2e = []
    for i in range(args.warmup + args.steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        dv.points.copy_(pts_h, non_blocking=True)
        sol, _ = nh_solve(pkg, prob, variants[HEAD][0], linear=variants[HEAD][1])
        sol_h.copy_(sol.reshape(-1), non_blocking=True)
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e.append(time.perf_counter() - t0)
    bc_bytes = ndofs * (8 + 1)  # Dirichlet values + mask, uploaded at each of the 5 load steps
    h2d = pts_h.numel() * 8 + 5 * bc_bytes
    t_e2e = max_over_ranks(statistics.mean(e2e))

    # dominant kernel roofline: FP32 block-CSR SpMV on the converged tangent
    A32 = prob.A32
    x32 = torch.randn(ndofs, dtype=torch.float32, device=device)
    y32 = torch.empty_like(x32)

    def spmv32():
        nat.check(nat.lib().fem_bsr_spmv_f32(3, A32.n_brows, nat.ptr(A32.row_ptr), nat.ptr(A32.col_idx),
                                             nat.ptr(A32.vals), nat.ptr(x32), nat.ptr(y32),
                                             nat.stream_ptr()), "spmv")

    t_spmv = time_kernel(spmv32)
    nnzb = dv.nnzb
    spmv_bytes = nnzb * 9 * 4 + nnzb * 4 + (dv.num_nodes + 1) * 4 + 2 * ndofs * 4
    hbm, peak_kind = peaks()

    # assembly throughput, DoF/s: FP64 residual with the FP64 or the FP32
    # tangent (the plain and the mixed Newton passes)
    sol_last = torch.zeros(ndofs, dtype=torch.float64, device=device)
    res = torch.empty(ndofs, dtype=torch.float64, device=device)
    A64 = dv.new_matrix(torch.float64)
    t_asm64 = time_kernel(lambda: prob.assemble(sol_last, res=res, vals=A64.vals), reps=10)
    t_asm32 = time_kernel(lambda: prob.assemble(sol_last, res=res, vals=A32.vals, fp32=True), reps=10)
    asm_bytes64 = dv.num_cells * (32 + 8 * 3 * 8 + 24 * 8 + 256) + nnzb * 9 * 8 + ndofs * 8
    asm_bytes32 = dv.num_cells * (32 + 8 * 3 * 8 + 24 * 8 + 256) + nnzb * 9 * 4 + ndofs * 8

    # SIMP 60x30x30 with the committed learned warm start (held-out samples)
    simp = None
    try:
        import importlib
        ws = importlib.import_module("jax_fem_b200.warmstart")
        wpath = os.path.join(ROOT, "jax-fem_b200", "weights", "warmstart_simp60.pt")
        if os.path.exists(wpath):
            net, _ = ws.load(wpath, device)
            sprob = ws.cantilever_problem()
            warmstart_eval(pkg, ws, sprob, net, 1, seed=77)  # warm-up
            rows = warmstart_eval(pkg, ws, sprob, net, args.simp_samples, seed=999_000,
                                  arms=[(pr, st) for pr in ("fp64", "mixed", "fp64_gmg", "mixed_gmg")
                                        for st in ("zero", "learned")])
            simp = {"workload": "SIMP cantilever 60x30x30 (175,863 dofs), seeded Gaussian random density, "
                                "load patch position uniform in z; rel.res 1e-8 of the zero-start residual; "
                                "fp64/mixed = block-Jacobi CG (mixed: FP32 tangent, FP32 CG restarted inside FP64 "
                                "refinement); *_gmg = FP64 CG with a multigrid V-cycle (FP32 in mixed_gmg)",
                    "samples": args.simp_samples, "arms": summarize_eval(rows)}
    except Exception as e:  # noqa: BLE001 - report, do not lose the headline line
        simp = {"error": str(e)[:200]}
    # J2 40^3, 10 increments, plain vs mixed
    j2 = {}
    for arm, prec, rt, pc in (("fp64", "fp64", 1e-10, "block_jacobi"), ("fp64_adaptive", "fp64", "adaptive", "block_jacobi"),
                              ("mixed", "mixed", "adaptive", "block_jacobi"), ("fp64_gmg", "fp64", "adaptive", "gmg"),
                              ("mixed_gmg", "mixed", "adaptive", "gmg")):
        lin_j2 = {"cg": {"precond": pc, "rtol": rt, "atol": 0.0, "maxiter": 20000}}
        j2_run(pkg, 40, 10, prec, lin_j2)  # warm-up
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        _, jn, jk = j2_run(pkg, 40, 10, prec, lin_j2)
        e1.record()
        torch.cuda.synchronize()
        j2[arm] = {"s": round(e0.elapsed_time(e1) * 1e-3, 4), "newton": jn, "krylov": jk}
    elements = cell_path = amg = None
    if not args.no_elements:
        try:
            elements = element_bench(pkg, device)
        except Exception as e:  # noqa: BLE001 - report, do not lose the headline line
            elements = {"error": str(e)[:300]}
        try:
            cell_path = cell_path_bench(pkg, device)
        except Exception as e:  # noqa: BLE001 - report, do not lose the headline line
            cell_path = {"error": str(e)[:300]}
        try:
            amg = amg_bench(pkg, device)
        except Exception as e:  # noqa: BLE001 - report, do not lose the headline line
            amg = {"error": str(e)[:300]}
    try:
        tc = conv_bench(pkg, device)
    except Exception as e:  # noqa: BLE001 - report, do not lose the headline line
        tc = {"error": str(e)[:300]}
    newton = {k: sum(i["newton_iters"] for i in v[1]) for k, v in results.items()}
    krylov = {k: sum(sum(i["krylov_iters"]) for i in v[1]) for k, v in results.items()}
    out = {
        "metric": METRIC,
        "value": round(t_mixed, 6),
        "unit": "s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_mixed * 1e3, 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64 residual, CG vectors and reductions; f32 tangent values and multigrid V-cycle",
        "data": "synthetic",
        "config": {"workload": f"neo-hookean {args.n}^3 HEX8, 30 deg twist in 5 load steps, "
                               "Newton rel.res 1e-8", "dofs": ndofs, "cells": dv.num_cells,
                   "precision": "mixed", "krylov": "cg (f64 vectors, f32 tangent) preconditioned by a geometric multigrid v-cycle (f32)",
                   "l2": "flushed (256 MB write) between timed steps", "parallelism": f"replicas x{world}",
                   "learned_warm_start": "not in value: the trained network gains nothing at rel.res 1e-8 "
                                         "(simp60_learned_warm_start), and no network is trained for this "
                                         "twist; value is the mixed-precision multigrid solve alone",
                   "multigrid_state": "reset before every timed solve (each pays its own coarse setups)"},
        "plain_fp64_s": round(t_plain, 6),
        "speedup_vs_plain_fp64": round(t_plain / t_mixed, 3),
        "speedup_mixed_vs_fp64_same_method": {
            "gmg": round(results["plain_fp64_gmg"][0] / results["mixed_gmg"][0], 3),
            "block_jacobi_adaptive": round(results["plain_fp64_adaptive"][0] / results["mixed"][0], 3)},
        "variants_s": {k: round(v[0], 6) for k, v in results.items()},
        "variants_note": "reference_method_fp64 = the reference's default BiCGSTAB + Jacobi (tol = atol = 1e-10) in "
                         "FP64 on the GPU; plain_fp64 = tight (1e-10) CG + 3x3 block-Jacobi solves in FP64; "
                         "*_adaptive/mixed* = Eisenstat-Walker forcing; mixed = FP32 tangent and FP32 CG "
                         "iterations with reliable updates (FP64 solution, true residual, reductions); "
                         "mixed_tight = the same to the 1e-10 linear tolerance; mixed_refinement = FP32 CG "
                         "restarted inside FP64 iterative refinement; *_gmg = CG preconditioned by a geometric "
                         "multigrid V-cycle (FP64 CG; plain_fp64_gmg: FP64 tangent and V-cycle; mixed_gmg: FP32 "
                         "tangent values and V-cycle; coarse operators shared by up to 4 Newton solves, mg_lag 4); "
                         "value = mixed_gmg",
        "solves_per_s": round(world / t_mixed, 4),
        "newton_iters": newton,
        "krylov_iters": krylov,
        "assembly_dofs_per_s": {"fp64_residual_tangent": round(ndofs / t_asm64),
                                "fp64_residual_fp32_tangent": round(ndofs / t_asm32)},
        "assembly_us": {"fp64": round(t_asm64 * 1e6, 1), "fp32": round(t_asm32 * 1e6, 1)},
        "assembly_hbm_frac": {"fp64": round(asm_bytes64 / t_asm64 / 1e9 / hbm, 3),
                              "fp32": round(asm_bytes32 / t_asm32 / 1e9 / hbm, 3)},
        "roofline": {"kernel": "fem_bsr_spmv_f32 (block-CSR 3x3, FP32 values) on the converged 50^3 tangent: "
                               "the row kernel that the headline V-cycle's smoothing and residual steps "
                               "(cheb_step/cheb_resid/mg_residual) run with fused epilogues",
                     "bound": "hbm", "achieved": round(spmv_bytes / t_spmv / 1e9, 1), "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(spmv_bytes / t_spmv / 1e9 / hbm, 4),
                     "traffic": 143.9e6, "traffic_note": "ncu dram__bytes_read+write of this kernel at this size",
                     "algorithmic_bytes": spmv_bytes, "us_per_launch": round(t_spmv * 1e6, 2)},
        "simp60_learned_warm_start": simp,
        "j2_40_10_increments": j2,
        "other_elements_neo_hookean_twist": elements,
        "cell_kernel_path": cell_path,
        "tensor_core_conv": tc,
        "amg_renumbered_tet10": amg,
        "e2e": {"value": round(t_e2e, 6), "unit": "s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(ndofs * 8)},
        "gpu_launches": int(launches),
        "clocks": clocks,
    }
    return out


# ---------------------------------------------------------------------------
# CPU baseline: the reference's method restated in C++ / OpenMP (oracle/)
# ---------------------------------------------------------------------------

def host_threads():
    """Host cores this process may run on (its CPU affinity)."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover - non-Linux
        return os.cpu_count() or 1


class CPUTwist:
    """The Neo-Hookean twist on the host cores, solved by the reference's
    method (fem_cpu.cpp: forward-mode cell Jacobians, COO sum into CSR,
    zeroRows, BiCGSTAB + Jacobi at tol = atol = 1e-10, Newton to rel.res 1e-8
    with tol 1e-12), one load step per call, in order: load step 1 starts
    from zero, later ones from the same extrapolated guess the GPU arm's
    nh_solve uses (2 u_{k-1} - u_{k-2}).  After load step 5 the next call
    starts a new solve."""

    def __init__(self, n, threads, steps=5, total_deg=30.0):
        from oracle import fem_cpu as fc
        fc.build()
        self.fc, self.n, self.steps, self.total_deg = fc, n, steps, total_deg
        self.prob = fc.CPUProblem(n, fc.LAW_NEO_HOOKEAN, 10.0, 0.3, threads=threads)
        self.k, self.prev, self.prev2 = 0, None, None

    def step(self):
        """Solve the next load step; returns (load step 1..5, seconds, stats)."""
        fc = self.fc
        k = self.k % self.steps + 1
        if k == 1:
            self.prev = self.prev2 = None
        t0 = time.perf_counter()
        if self.prev is None:
            u = np.zeros(self.prob.ndofs)
        else:
            u = self.prev.copy() if self.prev2 is None else 2.0 * self.prev - self.prev2
        self.prob.set_dirichlet(*fc.box_dirichlet(self.n, "twist", math.radians(self.total_deg * k / self.steps)))
        st = self.prob.newton(u, rel_tol=1e-8, tol=1e-12, method=fc.METHOD_BICGSTAB, lin_tol=1e-10,
                              lin_atol=1e-10, lin_maxiter=10000)
        dt = time.perf_counter() - t0
        self.prev2, self.prev = self.prev, u
        self.k += 1
        return k, dt, st


def _cpu_sample_text(n, threads, what):
    return (f"oracle/fem_cpu.cpp (the reference's method restated in C++/OpenMP, FP64, {threads} threads): "
            f"{what} of the Neo-Hookean {n}^3 HEX8 twist (30 deg in 5 load steps), each load step a full Newton "
            f"solve to rel.res 1e-8 with forward-mode cell Jacobians, COO sum + zeroRows and BiCGSTAB + Jacobi "
            f"at tol = atol = 1e-10")


def cpu_baseline(n):
    """One whole solve (the 5 load steps) of the headline workload on the
    host cores, timed: the time-to-solve of the reference's method on CPU."""
    threads = host_threads()
    tw = CPUTwist(n, threads)
    t, tot = 0.0, {"newton": 0, "krylov": 0}
    for _ in range(tw.steps):
        _, dt, st = tw.step()
        t += dt
        tot["newton"] += st["newton"]
        tot["krylov"] += st["krylov"]
    return {"value": round(t, 3), "unit": "s", "cores": threads, "kind": "port",
            "sample": _cpu_sample_text(n, threads, "one whole solve (all 5 load steps, timed in full)"),
            "newton_iters": tot["newton"], "krylov_iters": tot["krylov"]}


def run_reference(args, rank, world):
    """The reference arm: the reference's method on the host cores (the
    reference itself needs JAX, basix and PETSc, which this image lacks).
    One step = one load step of the twist, solved in full, in the order of
    the load history; warm-up steps run the first load steps.  value = the
    time-to-solve of the whole twist: the mean time of each of the 5 load
    steps over the timed steps, summed (a load step not among the timed
    steps takes its warm-up time, or, with fewer than 5 steps in all, the
    time of a solve of it run after the timed steps)."""
    if rank != 0:
        return None
    threads = host_threads()
    tw = CPUTwist(args.n, threads)
    per_k = {k: [] for k in range(1, tw.steps + 1)}
    warm_k = {}
    for _ in range(args.warmup):
        k, dt, _ = tw.step()
        warm_k.setdefault(k, dt)
    step_s, newton, krylov = [], 0, 0
    for _ in range(args.steps):
        k, dt, st = tw.step()
        per_k[k].append(dt)
        step_s.append(dt)
        newton += st["newton"]
        krylov += st["krylov"]
    # A load step not among the timed steps takes its warm-up time; one
    # neither timed nor warmed up (steps + warmup < 5) is solved now, in the
    # order of the history, and its measured time is used (at most 5 more).
    extra_k = {}
    for _ in range(tw.steps):
        if all(per_k[k] or k in warm_k or k in extra_k for k in per_k):
            break
        k, dt, _ = tw.step()
        extra_k.setdefault(k, dt)
    missing = {k: ("warm-up" if k in warm_k else "after the timed steps") for k, t in per_k.items() if not t}
    v = sum(statistics.mean(per_k[k]) if per_k[k] else warm_k.get(k, extra_k.get(k)) for k in per_k)
    sample = _cpu_sample_text(args.n, threads, f"{args.steps} timed load steps after {args.warmup} warm-up ones")
    cb = {"value": round(v, 3), "unit": "s", "cores": threads, "kind": "port", "sample": sample}
    return {"metric": METRIC, "value": round(v, 3), "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(statistics.mean(step_s) * 1e3, 1),
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "impl": "reference",
            "config": {"workload": f"neo-hookean {args.n}^3 HEX8, 30 deg twist in 5 load steps, Newton rel.res 1e-8",
                       "precision": "fp64 (the reference's method on the host cores)",
                       "step": "one load step of the twist, solved in full; value = the 5 load steps' mean "
                               "times summed",
                       "load_step_s": {k: round(statistics.mean(t), 3) for k, t in per_k.items() if t},
                       "load_steps_not_timed_as_steps": missing,
                       "newton_iters_timed": newton, "krylov_iters_timed": krylov},
            "cpu_baseline": cb,
            "e2e": {"value": round(v, 3), "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_asm_only(args, device):
    """Assembly times of the HEX8 kernel (CUDA events, 20 launches after 3
    warm-up ones) at a twisted state of the n^3 Neo-Hookean cube: FP64
    residual with the FP64 / FP32 tangent, and the residual alone."""
    pkg = load_package()
    prob = nh_problem(pkg, n=args.n)
    dv = prob.dev()
    prob.fes[0].update_Dirichlet_boundary_conditions(rotation_bc(math.radians(6.0)))
    mask, vals = prob.dirichlet_device()
    u = torch.where(mask.bool(), vals, torch.zeros_like(vals))
    res = torch.empty_like(u)
    A64, A32 = dv.new_matrix(torch.float64), dv.new_matrix(torch.float32)
    hbm, kind = peaks()
    t64 = time_kernel(lambda: prob.assemble(u, res=res, vals=A64.vals))
    t32 = time_kernel(lambda: prob.assemble(u, res=res, vals=A32.vals, fp32=True))
    tr = time_kernel(lambda: prob.assemble(u, res=res))
    nd = dv.ndofs
    b64 = dv.num_cells * (32 + 8 * 3 * 8 + 24 * 8 + 256) + dv.nnzb * 9 * 8 + nd * 8
    b32 = dv.num_cells * (32 + 8 * 3 * 8 + 24 * 8 + 256) + dv.nnzb * 9 * 4 + nd * 8
    print(json.dumps({"n": args.n, "cells": dv.num_cells, "us": {"fp64": round(t64 * 1e6, 1),
                      "fp32": round(t32 * 1e6, 1), "residual_only": round(tr * 1e6, 1)},
                      "hbm_frac": {"fp64": round(b64 / t64 / 1e9 / hbm, 4), "fp32": round(b32 / t32 / 1e9 / hbm, 4)},
                      "peak_kind": kind}), flush=True)


def run_mg_only(args, device):
    """Multigrid times on the n^3 Neo-Hookean tangent at a twisted state
    (CUDA events, 20 calls after 3 warm-up ones): a full setup of the FP32
    hierarchy from the FP32 tangent, a fine-only setup, one V-cycle launched
    directly and replayed from a CUDA graph."""
    import importlib
    pkg = load_package()
    mgm = importlib.import_module("jax_fem_b200.multigrid")
    prob = nh_problem(pkg, n=args.n)
    dv = prob.dev()
    prob.fes[0].update_Dirichlet_boundary_conditions(rotation_bc(math.radians(6.0)))
    mask, vals = prob.dirichlet_device()
    u = torch.where(mask.bool(), vals, torch.zeros_like(vals))
    A32 = dv.new_matrix(torch.float32)
    prob.assemble(u, res=torch.empty_like(u), vals=A32.vals, fp32=True)
    M = mgm.Multigrid(dv, prob.mesh.points, prob.mesh.cells, fp32=True, nu_fine=1)
    t_full = time_kernel(lambda: M.setup(A32))
    t_fine = time_kernel(lambda: M.setup(A32, fine_only=True))
    r = torch.randn(dv.ndofs, device=device)
    z = torch.empty_like(r)
    t_v = time_kernel(lambda: M.vcycle(r, z, nu=2, coarse_steps=8, ratio=25.0))
    # the same V-cycle replayed from a CUDA graph (as inside the solve graph)
    s = torch.cuda.Stream(device=device)
    s.wait_stream(torch.cuda.current_stream(device))
    with torch.cuda.stream(s):
        M.vcycle(r, z, nu=2, coarse_steps=8, ratio=25.0)
    torch.cuda.current_stream(device).wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        M.vcycle(r, z, nu=2, coarse_steps=8, ratio=25.0)
    t_g = time_kernel(g.replay)
    print(json.dumps({"n": args.n, "levels": M.nlevels, "us": {"full_setup": round(t_full * 1e6, 1),
                      "fine_setup": round(t_fine * 1e6, 1), "vcycle": round(t_v * 1e6, 1),
                      "vcycle_graph": round(t_g * 1e6, 1)},
                      "half_fine": M.half_fine}), flush=True)


def run_profile_element(args, device):
    """For ncu: the general-element kernel on one element type at its bench
    size (ELEMENT_BOXES), Neo-Hookean at a twisted state: FP64 assembly x2,
    then FP64-residual/FP32-tangent assembly x2."""
    pkg = load_package()
    nat = pkg._native
    n = dict(ELEMENT_BOXES)[args.profile_element]
    prob = element_problem(pkg, args.profile_element, n)
    dv = prob.dev()
    prob.fes[0].update_Dirichlet_boundary_conditions(rotation_bc(math.radians(6.0)))
    mask, vals = prob.dirichlet_device()
    u = torch.where(mask.bool(), vals, torch.zeros_like(vals))
    res = torch.empty_like(u)
    A64, A32 = dv.new_matrix(torch.float64), dv.new_matrix(torch.float32)
    for _ in range(2):
        prob.assemble(u, res=res, vals=A64.vals)
    for _ in range(2):
        prob.assemble(u, res=res, vals=A32.vals, fp32=True)
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.profile_element, "cells": dv.num_cells, "dofs": dv.ndofs, "nnzb": dv.nnzb,
                      "launches": nat.launch_count()}))


def run_profile(args, device):
    """A short fixed sequence of the hot kernels at the bench size, for ncu:
    FP64 assembly and the FP64-residual/FP32-tangent assembly (x2 each),
    FP32/FP64 SpMV (x3 each), one mixed solve with block-Jacobi CG and one
    with the multigrid-preconditioned CG (the headline's linear solver)."""
    pkg = load_package()
    nat = pkg._native
    prob = nh_problem(pkg, n=args.n)
    dv = prob.dev()
    n = prob.num_total_dofs_all_vars
    prob.fes[0].update_Dirichlet_boundary_conditions(rotation_bc(math.radians(6.0)))
    u = torch.zeros(n, dtype=torch.float64, device=device)
    res = torch.empty_like(u)
    A64, A32 = dv.new_matrix(torch.float64), dv.new_matrix(torch.float32)
    for _ in range(2):
        prob.assemble(u, res=res, vals=A64.vals)
    for _ in range(2):
        prob.assemble(u, res=res, vals=A32.vals, fp32=True)
    x64 = torch.randn(n, dtype=torch.float64, device=device)
    x32 = x64.float()
    for _ in range(3):
        A32.matvec(x32)
    for _ in range(3):
        A64.matvec(x64)
    nh_solve(pkg, prob, "mixed", steps=1, total_deg=6.0,
             linear={"cg": {"precond": "block_jacobi", "rtol": "adaptive", "atol": 0.0}})
    nh_solve(pkg, prob, "mixed", steps=1, total_deg=6.0,
             linear={"cg": {"precond": "gmg", "rtol": "adaptive", "atol": 0.0, "mg_lag": 4}})
    torch.cuda.synchronize()
    print(json.dumps({"profile": "done", "launches": nat.launch_count()}))


def warmstart_eval(pkg, ws, prob, net, n, seed, log=None, arms=None):
    """Held-out SIMP solves from zero and from the network's prediction, on
    the plain FP64 and the mixed path, all stopping at the same absolute
    residual (rel.res 1e-8 of the zero-start residual, adaptive forcing).
    Each arm is solved twice per sample and the second solve timed.
    Returns per-sample Krylov iterations and times per arm."""
    linear = {"cg": {"precond": "block_jacobi", "rtol": "adaptive", "atol": 0.0, "maxiter": 50000}}
    # FP32 CG restarted inside FP64 refinement: on this high-contrast problem
    # it is the faster of the two mixed CG forms (reliable updates stall)
    linear_mixed = {"cg": dict(linear["cg"], reliable_delta=0.0)}
    linear_gmg = {"cg": {"precond": "gmg", "rtol": "adaptive", "atol": 0.0, "maxiter": 2000}}
    preds = {"zero": None, "learned": ws.Predictor(net, galerkin=True),
             "learned_raw": ws.Predictor(net, galerkin=False)}
    arms = arms or [(p, s) for p in ("fp64", "mixed") for s in ("zero", "learned", "learned_raw")]
    lin_of = {"fp64": ("fp64", linear), "mixed": ("mixed", linear_mixed),
              "fp64_gmg": ("fp64", linear_gmg), "mixed_gmg": ("mixed", linear_gmg)}
    g = torch.Generator().manual_seed(seed)
    dev = prob.dev().device
    rows = []
    for i in range(n):
        rho = ws.random_density(g)
        z0 = float(torch.randint(0, ws.NZ - 3 + 1, (1,), generator=g).item())
        prob.set_patch(z0)
        prob.set_params(ws.cell_rho_to_torch(rho, dev))
        r = {}
        for arm, start in arms:
            prec, lin = lin_of[arm]
            opts = {"newton": {"rel_tol": 1e-8, "tol": 1e-14, "precision": prec, "linear": lin,
                               "rel_tol_reference": "zero", "return_info": True,
                               "warm_start": preds[start]}}
            # the first solve after a new density / load patch pays one-off
            # host work (load vectors, graph captures); time the second
            pkg.solver(prob, opts)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            (sol,), info = pkg.solver(prob, opts)
            e1.record()
            torch.cuda.synchronize()
            r[f"{arm}_{start}"] = {"krylov": sum(info["krylov_iters"]), "newton": info["newton_iters"],
                                    "s": e0.elapsed_time(e1) * 1e-3}
        rows.append(r)
        if log and (i + 1) % 20 == 0:
            log(f"  eval {i + 1}/{n}")
    return rows


def summarize_eval(rows):
    out = {}
    for arm in rows[0]:
        out[arm] = {"krylov_mean": float(np.mean([r[arm]["krylov"] for r in rows])),
                    "newton_mean": float(np.mean([r[arm]["newton"] for r in rows])),
                    "s_mean": float(np.mean([r[arm]["s"] for r in rows]))}
    return out


def run_warmstart_train(args, device):
    """Generate (rho, u) pairs with the solver, train the warm-start network on
    the tensor-core kernels, evaluate on held-out samples, save the weights."""
    pkg = load_package()
    import importlib
    ws = importlib.import_module("jax_fem_b200.warmstart")
    prob = ws.cantilever_problem()
    t0 = time.time()
    train_data = ws.generate(prob, args.ws_train, seed=1000)
    t_gen = time.time() - t0
    print(f"generated {args.ws_train} training samples in {t_gen:.1f} s", flush=True)
    net = ws.WarmStartNet(seed=0)
    t0 = time.time()
    hist = ws.train(net, train_data, epochs=args.ws_epochs, batch=16, lr=args.ws_lr, device=device)
    torch.cuda.synchronize()
    t_train = time.time() - t0
    print(f"trained {args.ws_epochs} epochs in {t_train:.1f} s", flush=True)
    rows = warmstart_eval(pkg, ws, prob, net, args.ws_test, seed=999_000, log=print)
    meta = {"n_train": args.ws_train, "n_test": args.ws_test, "epochs": args.ws_epochs, "lr": args.ws_lr,
            "loss_history": hist, "gen_s": t_gen, "train_s": t_train, "heldout": summarize_eval(rows),
            "u_scale": float(net.u_scale.item())}
    if args.ws_out:
        ws.save(net, args.ws_out, meta)
    print(json.dumps({k: v for k, v in meta.items() if k != "loss_history"}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=50)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--simp-samples", type=int, default=12)
    ap.add_argument("--no-elements", action="store_true", help="skip the TET4/TET10/HEX20/HEX27 measurements")
    ap.add_argument("--elements-only", action="store_true",
                    help="only the TET4/TET10/HEX20/HEX27 and cell-kernel-path measurements")
    ap.add_argument("--profile", action="store_true", help="short kernel sequence for ncu captures")
    ap.add_argument("--asm-only", action="store_true", help="only the HEX8 assembly times")
    ap.add_argument("--mg-only", action="store_true", help="only the multigrid setup and V-cycle times")
    ap.add_argument("--conv-only", action="store_true",
                    help="only the tensor-core convolution / weight-gradient throughput")
    ap.add_argument("--profile-element", default="", choices=["", "TET4", "TET10", "HEX20", "HEX27"],
                    help="general-element assembly sequence for ncu captures")
    ap.add_argument("--warmstart-train", action="store_true",
                    help="generate SIMP (rho, u) pairs, train the warm-start network, evaluate, save")
    ap.add_argument("--ws-train", type=int, default=2000)
    ap.add_argument("--ws-test", type=int, default=200)
    ap.add_argument("--ws-epochs", type=int, default=30)
    ap.add_argument("--ws-lr", type=float, default=2e-3)
    ap.add_argument("--ws-out", default="")
    ap.add_argument("--warmstart-eval", default="", help="evaluate a saved warm-start model on held-out samples")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
        if out is not None:
            print(json.dumps(out), flush=True)
        return
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                             device_id=device)
    if args.profile:
        run_profile(args, device)
        return
    if args.profile_element:
        run_profile_element(args, device)
        return
    if args.asm_only:
        run_asm_only(args, device)
        return
    if args.mg_only:
        run_mg_only(args, device)
        return
    if args.conv_only:
        print(json.dumps({"tensor_core_conv": conv_bench(load_package(), device)}), flush=True)
        return
    if args.elements_only:
        pkg = load_package()
        print(json.dumps({"other_elements_neo_hookean_twist": element_bench(pkg, device),
                          "cell_kernel_path": cell_path_bench(pkg, device),
                          "amg_renumbered_tet10": amg_bench(pkg, device)}), flush=True)
        return
    if args.warmstart_train:
        run_warmstart_train(args, device)
        return
    if args.warmstart_eval:
        import importlib
        pkg = load_package()
        ws = importlib.import_module("jax_fem_b200.warmstart")
        net, meta = ws.load(args.warmstart_eval, device)
        rows = warmstart_eval(pkg, ws, ws.cantilever_problem(), net, args.ws_test, seed=999_000)
        print(json.dumps({"heldout": summarize_eval(rows), "n_test": args.ws_test}), flush=True)
        return
    out = run_ours(args, rank, world, device)
    if rank == 0:
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(args.n)
        print(json.dumps(out), flush=True)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
