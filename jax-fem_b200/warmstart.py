"""Learned warm start for the SIMP cantilever (60 x 30 x 30 HEX8 cells).

A 3D convolutional encoder-decoder maps the density field rho and the load
patch to a displacement field that seeds Newton/CG.  The exact FP64 Newton
residual still decides convergence: the converged answer is always the solver's, the
network only changes where the iteration starts (``solver_options
['newton']['warm_start']``); with no network the start is zero.

Network (all convolutions 3x3x3, padding 1, BF16 weights/activations, FP32
accumulation on the tensor cores through libjaxfem_b200's tcgen05 kernels):
  input   32 x 16 x 16 coarse grid (2x2x2 cell blocks), 16 channels:
          rho, E(rho)/E0, load indicator, domain mask, 12 zero channels
  encoder 16 -> 32 -> 64 -> 128 channels, two convs (+ReLU) per level,
          2x average pooling between levels (4 levels)
  decoder nearest 2x upsampling, conv to the skip's width (+ReLU), additive
          skip, conv (+ReLU); a last conv (no ReLU) gives 3 used channels
  output  displacement / scale at the coarse nodes (fine nodes with even
          indices), prolonged trilinearly to the 61 x 31 x 31 mesh nodes.
Forward and backward of every convolution run on the project's kernels
(conv3d forward, the same kernel with flipped weights for the input
gradient, im2col + split-K GEMM for the weight gradient); pooling,
upsampling, skips and the optimiser step are PyTorch tensor ops.

Training data: (rho, u) pairs solved by this package on seeded Gaussian
random fields (correlation length 4 cells) mapped to [0.01, 1] by a sigmoid,
with the load patch position drawn uniformly along z.
"""
import math
import time

import numpy as np
import torch
import torch.nn.functional as F

from . import _native as nat
from .generate_mesh import Mesh, box_mesh
from .laws import SIMPElastic
from .problem import Problem
from .solver import solver

NX, NY, NZ = 60, 30, 30
CD, CH, CW = 32, 16, 16          # coarse network grid (x, y, z)
IN_CH = 16
E0, EMIN, NU, PENAL = 70e3, 70.0, 0.3, 3.0


# ---------------------------------------------------------------------------
# the SIMP cantilever and its random inputs
# ---------------------------------------------------------------------------

def gaussian_random_field(shape, corr_len, generator):
    """Zero-mean, unit-variance Gaussian random field with a Gaussian
    correlation function of length ``corr_len`` cells: white noise convolved
    (FFT, periodic) with a Gaussian kernel of std corr_len / sqrt(2)."""
    noise = torch.randn(shape, generator=generator, dtype=torch.float64)
    sigma = corr_len / math.sqrt(2.0)
    freqs = [torch.fft.fftfreq(n, dtype=torch.float64) for n in shape]
    k2 = sum(f.reshape([-1 if i == d else 1 for i in range(len(shape))]) ** 2 for d, f in enumerate(freqs))
    filt = torch.exp(-2.0 * math.pi ** 2 * sigma ** 2 * k2)
    g = torch.fft.ifftn(torch.fft.fftn(noise) * filt).real
    g = g - g.mean()
    return g / g.std()


def random_density(generator, corr_len=4.0):
    """rho = 0.01 + 0.99 sigmoid(g) per cell, shape (60, 30, 30)."""
    g = gaussian_random_field((NX, NY, NZ), corr_len, generator)
    return 0.01 + 0.99 * torch.sigmoid(g)


def patch_location(z0, width=3.0):
    """Loaded faces: x = 60 and z0 <= z <= z0 + width."""
    def loc(p):
        return np.isclose(p[0], float(NX), atol=1e-5) & (p[2] >= z0 - 1e-5) & (p[2] <= z0 + width + 1e-5)
    return loc


class SIMPCantilever(Problem):
    """60x30x30 cantilever clamped at x=0, unit downward traction on a patch of
    the x=60 face (surface_map = -t = (0,0,1)); density per cell via set_params."""

    def get_tensor_map(self):
        return SIMPElastic(E0, EMIN, NU, PENAL)

    def get_surface_maps(self):
        return [lambda u, x: np.array([0.0, 0.0, 1.0])]

    def set_params(self, params):
        C = self.num_cells
        self.internal_vars = [params.reshape(C, 1, 1).expand(C, 8, 1)]

    def set_patch(self, z0):
        self.location_fns = [patch_location(z0)]
        self.boundary_inds_list = self.fes[0].get_boundary_conditions_inds(self.location_fns)
        self._fext = None
        if hasattr(self, "_surface_loads"):
            del self._surface_loads


def cantilever_problem(z0=0.0):
    m = box_mesh(NX, NY, NZ, float(NX), float(NY), float(NZ))
    mesh = Mesh(m.points, m.cells_dict["hexahedron"])
    fixed = lambda p: np.isclose(p[0], 0.0, atol=1e-5)  # noqa: E731
    zero = lambda p: 0.0 * p[0]  # noqa: E731
    bc = [[fixed] * 3, [0, 1, 2], [zero] * 3]
    return SIMPCantilever(mesh, vec=3, dim=3, dirichlet_bc_info=bc, location_fns=[patch_location(z0)])


def cell_rho_to_torch(rho, device):
    """(60,30,30) cell field in box_mesh cell order (x slowest) -> (C,) f64."""
    return rho.reshape(-1).to(device=device, dtype=torch.float64)


# ---------------------------------------------------------------------------
# tensor-core convolution with autograd
# ---------------------------------------------------------------------------

def _conv_fwd(x, wb, b, relu):
    N, D, H, W, Cin = x.shape
    Cout = wb.shape[0]
    y = torch.empty(N, D, H, W, Cout, dtype=torch.bfloat16, device=x.device)
    nat.check(nat.lib().fem_conv3d_fwd_bf16(nat.ptr(x), nat.ptr(wb), nat.ptr(b), nat.ptr(y), N, D, H, W, Cin,
                                            Cout, int(relu), nat.stream_ptr()), "conv3d_fwd")
    return y


class ConvTC(torch.autograd.Function):
    """3x3x3 convolution (+bias, optional fused ReLU) on the tensor cores.

    x: (N,D,H,W,Cin) bf16 NDHWC; w: (Cout,27,Cin) f32 master weights;
    b: (Cout,) f32.  Returns bf16 NDHWC."""

    @staticmethod
    def forward(ctx, x, w, b, relu):
        x = x.contiguous()
        wb = w.detach().to(torch.bfloat16).contiguous()
        y = _conv_fwd(x, wb, b.detach().contiguous(), relu)
        ctx.save_for_backward(x, wb, y)
        ctx.relu = relu
        return y

    @staticmethod
    def backward(ctx, dy):
        x, wb, y = ctx.saved_tensors
        N, D, H, W, Cin = x.shape
        Cout = wb.shape[0]
        st = nat.stream_ptr()
        lib = nat.lib()
        dy = dy.to(torch.bfloat16).contiguous()
        if ctx.relu:
            dz = torch.empty_like(dy)
            nat.check(lib.fem_relu_mask_bf16(nat.ptr(dy), nat.ptr(y), nat.ptr(dz), dy.numel(), st), "relu_mask")
        else:
            dz = dy
        dx = None
        if ctx.needs_input_grad[0]:
            wt = torch.empty(Cin, 27, Cout, dtype=torch.bfloat16, device=x.device)
            nat.check(lib.fem_conv3d_flip_weights_bf16(nat.ptr(wb), nat.ptr(wt), Cout, Cin, st), "flip")
            dx = _conv_fwd(dz, wt, None, False)
        V = N * D * H * W
        col = torch.empty(27 * Cin, V, dtype=torch.bfloat16, device=x.device)
        nat.check(lib.fem_conv3d_im2col_t_bf16(nat.ptr(x), nat.ptr(col), N, D, H, W, Cin, st), "im2col")
        dzt = torch.empty(Cout, V, dtype=torch.bfloat16, device=x.device)
        nat.check(lib.fem_transpose_bf16(nat.ptr(dz), nat.ptr(dzt), V, Cout, st), "transpose")
        dwt = torch.zeros(27 * Cin, Cout, dtype=torch.float32, device=x.device)
        mtiles = (27 * Cin + 127) // 128
        kchunks = max(1, V // 64)
        split = int(max(1, min(kchunks, math.ceil(2 * 148 / mtiles))))
        nat.check(lib.fem_gemm_bf16_tn_f32(nat.ptr(col), nat.ptr(dzt), nat.ptr(dwt), 27 * Cin, Cout, V, Cout,
                                           split, st), "wgrad")
        dw = dwt.view(27, Cin, Cout).permute(2, 0, 1).contiguous()
        db = dz.float().reshape(-1, Cout).sum(0)
        return dx, dw, db, None


def pool2(x):
    N, D, H, W, C = x.shape
    return x.float().reshape(N, D // 2, 2, H // 2, 2, W // 2, 2, C).mean(dim=(2, 4, 6)).to(torch.bfloat16)


def up2(x):
    N, D, H, W, C = x.shape
    return x[:, :, None, :, None, :, None, :].expand(N, D, 2, H, 2, W, 2, C).reshape(N, 2 * D, 2 * H, 2 * W, C)


class WarmStartNet(torch.nn.Module):
    """4-level 3D U-Net (16-128 channels) on the tensor-core convolution."""

    LAYERS = [("e1a", IN_CH, 16), ("e1b", 16, 16), ("e2a", 16, 32), ("e2b", 32, 32), ("e3a", 32, 64),
              ("e3b", 64, 64), ("e4a", 64, 128), ("e4b", 128, 128), ("d3a", 128, 64), ("d3b", 64, 64),
              ("d2a", 64, 32), ("d2b", 32, 32), ("d1a", 32, 16), ("d1b", 16, 16), ("out", 16, 16)]

    def __init__(self, seed=0):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.w = torch.nn.ParameterDict()
        self.b = torch.nn.ParameterDict()
        for name, cin, cout in self.LAYERS:
            std = math.sqrt(2.0 / (27 * cin))
            self.w[name] = torch.nn.Parameter(torch.randn(cout, 27, cin, generator=g) * std)
            self.b[name] = torch.nn.Parameter(torch.zeros(cout))
        self.register_buffer("u_scale", torch.ones(1))

    def conv(self, name, x, relu=True):
        return ConvTC.apply(x, self.w[name], self.b[name], relu)

    def forward(self, x):
        e1 = self.conv("e1b", self.conv("e1a", x))
        e2 = self.conv("e2b", self.conv("e2a", pool2(e1)))
        e3 = self.conv("e3b", self.conv("e3a", pool2(e2)))
        e4 = self.conv("e4b", self.conv("e4a", pool2(e3)))
        d3 = self.conv("d3b", self.conv("d3a", up2(e4)) + e3)
        d2 = self.conv("d2b", self.conv("d2a", up2(d3)) + e2)
        d1 = self.conv("d1b", self.conv("d1a", up2(d2)) + e1)
        return self.conv("out", d1, relu=False)


# ---------------------------------------------------------------------------
# features and targets on the coarse grid
# ---------------------------------------------------------------------------

def features(rho, load_nodes, device):
    """rho (B,60,30,30) cells, load_nodes (B,61,31,31) nodal traction
    magnitude -> (B,32,16,16,16) bf16 network input."""
    B = rho.shape[0]
    x = torch.zeros(B, CD, CH, CW, IN_CH, dtype=torch.float32, device=device)
    r = rho.to(device=device, dtype=torch.float32)
    rc = r.reshape(B, NX // 2, 2, NY // 2, 2, NZ // 2, 2).mean(dim=(2, 4, 6))
    ec = (EMIN + (E0 - EMIN) * r ** PENAL).reshape(B, NX // 2, 2, NY // 2, 2, NZ // 2, 2).mean(dim=(2, 4, 6)) / E0
    x[:, :NX // 2, :NY // 2, :NZ // 2, 0] = rc
    x[:, :NX // 2, :NY // 2, :NZ // 2, 1] = ec
    ln = load_nodes.to(device=device, dtype=torch.float32)
    lc = torch.zeros(B, NX // 2, NY // 2, NZ // 2, device=device)
    ii = torch.clamp(torch.arange(NX + 1, device=device) // 2, max=NX // 2 - 1)
    jj = torch.clamp(torch.arange(NY + 1, device=device) // 2, max=NY // 2 - 1)
    kk = torch.clamp(torch.arange(NZ + 1, device=device) // 2, max=NZ // 2 - 1)
    idx = ((ii[:, None, None] * (NY // 2) + jj[None, :, None]) * (NZ // 2) + kk[None, None, :]).reshape(-1)
    lc.view(B, -1).index_add_(1, idx, ln.reshape(B, -1))
    x[:, :NX // 2, :NY // 2, :NZ // 2, 2] = lc / lc.amax(dim=(1, 2, 3), keepdim=True).clamp_min(1e-30)
    x[:, :NX // 2, :NY // 2, :NZ // 2, 3] = 1.0
    return x.to(torch.bfloat16).contiguous()


def coarse_target(u_nodes):
    """Fine nodal displacement (B, 61*31*31*3) -> (B,32,16,16,3) at even nodes."""
    B = u_nodes.shape[0]
    u = u_nodes.reshape(B, NX + 1, NY + 1, NZ + 1, 3)[:, ::2, ::2, ::2, :]  # (B,31,16,16,3)
    out = torch.zeros(B, CD, CH, CW, 3, dtype=u.dtype, device=u.device)
    out[:, : NX // 2 + 1] = u
    return out


def prolong(uc):
    """(B,32,16,16,3) coarse-node displacement -> (B, 61*31*31*3) fine nodes."""
    B = uc.shape[0]
    c = uc[:, : NX // 2 + 1].permute(0, 4, 1, 2, 3).float()  # (B,3,31,16,16)
    f = F.interpolate(c, size=(NX + 1, NY + 1, NZ + 1), mode="trilinear", align_corners=True)
    return f.permute(0, 2, 3, 4, 1).reshape(B, -1)


def load_nodes_of(problem):
    f = problem.surface_load_vectors()[0].reshape(NX + 1, NY + 1, NZ + 1, 3)
    return f.norm(dim=-1)


# ---------------------------------------------------------------------------
# data generation, training, prediction
# ---------------------------------------------------------------------------

GEN_SOLVE = {"newton": {"rel_tol": 1e-8, "tol": 1e-14, "precision": "fp64",
                        "linear": {"cg": {"precond": "block_jacobi", "rtol": 1e-10, "atol": 0.0,
                                          "maxiter": 50000}}}}


def generate(problem, n, seed, log_every=100):
    """n solver-generated samples: dict of rho (n,60,30,30) f32, z0 (n,),
    load (n,61,31,31) f32, target (n,32,16,16,3) f32."""
    g = torch.Generator().manual_seed(seed)
    dev = problem.dev().device
    rhos, z0s, loads, targets = [], [], [], []
    t0 = time.time()
    for i in range(n):
        rho = random_density(g)
        z0 = float(torch.randint(0, NZ - 3 + 1, (1,), generator=g).item())
        problem.set_patch(z0)
        problem.set_params(cell_rho_to_torch(rho, dev))
        sol = solver(problem, GEN_SOLVE)[0].reshape(1, -1)
        rhos.append(rho.float())
        z0s.append(z0)
        loads.append(load_nodes_of(problem).float().cpu())
        targets.append(coarse_target(sol).float().cpu())
        if log_every and (i + 1) % log_every == 0:
            print(f"  generated {i + 1}/{n} ({time.time() - t0:.1f} s)", flush=True)
    return {"rho": torch.stack(rhos), "z0": torch.tensor(z0s), "load": torch.stack(loads),
            "target": torch.cat(targets)}


def train(net, data, epochs=30, batch=16, lr=2e-3, device=None, log=print):
    """Adam on the MSE of scaled coarse displacements; returns loss history."""
    device = device or torch.device("cuda", torch.cuda.current_device())
    net.to(device)
    n = data["rho"].shape[0]
    scale = data["target"].pow(2).mean().sqrt().item()
    net.u_scale.fill_(scale)
    x_all = features(data["rho"], data["load"], device)
    y_all = (data["target"] / scale).to(device)
    opt = torch.optim.Adam(net.parameters(), lr=lr)
    sched = torch.optim.lr_scheduler.CosineAnnealingLR(opt, T_max=epochs * (n // batch))
    g = torch.Generator().manual_seed(1)
    hist = []
    for ep in range(epochs):
        perm = torch.randperm(n, generator=g)
        tot = 0.0
        for s in range(0, n - batch + 1, batch):
            idx = perm[s:s + batch].to(device)
            out = net(x_all[idx])[..., :3].float()
            loss = F.mse_loss(out, y_all[idx])
            opt.zero_grad(set_to_none=True)
            loss.backward()
            opt.step()
            sched.step()
            tot += loss.item()
        hist.append(tot / (n // batch))
        if log:
            log(f"  epoch {ep + 1}/{epochs}: loss {hist[-1]:.4e}")
    return hist


class Predictor:
    """``warm_start`` callable for the solver: network prediction of the
    displacement of a SIMPCantilever at its current density and load patch.

    With ``galerkin=True`` (default) the prediction d (free dofs) is rescaled
    by the energy-optimal factor alpha = -(f.d + d.K u_b) / (d.K d) of the
    linear problem (K the Dirichlet-eliminated tangent, f the external load,
    u_b the prescribed values): one tangent assembly and one SpMV remove the
    network's error in the overall magnitude of the field."""

    def __init__(self, net, galerkin=True):
        self.net = net.eval()
        self.galerkin = galerkin
        self.calls = 0
        self.last_alpha = None
        self._A = None

    @torch.no_grad()
    def __call__(self, problem):
        dev = problem.dev().device
        rho = problem.internal_vars[0].reshape(problem.num_cells, -1)[:, 0].reshape(1, NX, NY, NZ)
        x = features(rho.float(), load_nodes_of(problem).reshape(1, NX + 1, NY + 1, NZ + 1), dev)
        pad = 8 - 1  # the 4x2x2 level tiles 8 samples per 128-voxel brick
        xb = torch.cat([x, x.new_zeros((pad,) + x.shape[1:])])
        uc = self.net(xb)[:1, ..., :3].float() * self.net.u_scale
        d = prolong(uc).reshape(-1).to(torch.float64)
        mask, ubc = problem.dirichlet_device()
        mb = mask.bool()
        d = torch.where(mb, torch.zeros_like(d), d)
        if self.galerkin:
            if self._A is None or self._A.vals.numel() != problem.dev().nnzb * 9:
                self._A = problem.dev().new_matrix(torch.float64)
            zero = torch.zeros_like(d)
            lift = torch.empty_like(d)
            ub = torch.where(mb, ubc, zero)
            problem.assemble(zero, vals=self._A.vals, lift=lift, dvec=ub)
            f = problem.external_load()
            Kd = self._A.matvec(d)
            dKd = float(torch.dot(d, Kd))
            if dKd > 0:
                alpha = -float(torch.dot(torch.where(mb, zero, f), d) + torch.dot(d, torch.where(mb, zero, lift))) / dKd
                self.last_alpha = alpha
                d = alpha * d
        self.calls += 1
        return torch.where(mb, ubc, d)


def save(net, path, meta=None):
    """Weights in BF16 (what the tensor-core kernels consume), buffers as-is."""
    state = {}
    for k, v in net.state_dict().items():
        v = v.detach().cpu()
        state[k] = v.to(torch.bfloat16) if k.startswith(("w.", "b.")) else v
    torch.save({"state": state, "meta": meta or {}}, path)


def load(path, device=None):
    ck = torch.load(path, map_location="cpu", weights_only=False)
    net = WarmStartNet()
    net.load_state_dict({k: v.float() if v.dtype == torch.bfloat16 else v for k, v in ck["state"].items()})
    if device is not None:
        net.to(device)
    return net, ck.get("meta", {})
