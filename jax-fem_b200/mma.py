"""Topology-optimisation outer loop: the Method of Moving Asymptotes (MMA)
driving the solver, with the reference's density-sensitivity filter.

Mirrors ``optimize`` and the filter helpers of the reference's mma.py
(``compute_filter_kd_tree`` mma.py:27-57, ``applySensitivityFilter`` :59-62,
``applyDensityFilter`` :64-65, ``optimize`` :415-528): same arguments, the
same filter (cells' centroids, radius 1.5 average element sizes, weights
max(rmin - distance, 0) over the 20 nearest design cells, sensitivities
filtered, densities not), the same MMA settings (bounds [0, 1], a0 = 1,
a = 0, c = 1e4, d = 0, the caller's move limit).

The MMA step itself is written here from Svanberg's method: K. Svanberg,
"The method of moving asymptotes - a new method for structural
optimization", IJNME 24 (1987) 359-373, with the asymptote, move-limit and
approximation rules and the primal-dual interior-point subproblem solver of
his "MMA and GCMMA - two methods for nonlinear optimization" (KTH, 2007).
Everything runs as torch tensor operations on the device of the design
variables (the GPU in a topology-optimisation loop), float64.
"""
import time
import warnings

import numpy as np
import torch

# MMA constants (Svanberg 2007, section 3)
_ASYINIT, _ASYINCR, _ASYDECR, _ALBEFA, _RAA0 = 0.5, 1.2, 0.7, 0.1, 1e-5


# ---- the MMA subproblem --------------------------------------------------------

def _approximation(x, xold1, xold2, low, upp, k, xmin, xmax, df0, fval, dfdx, move):
    """Asymptotes, bounds alpha/beta and the convex separable approximation
    p0, q0, P, Q, b at x (iteration k >= 1)."""
    span = xmax - xmin
    if k <= 2:
        low = x - _ASYINIT * span
        upp = x + _ASYINIT * span
    else:
        trend = (x - xold1) * (xold1 - xold2)
        factor = torch.where(trend > 0, torch.full_like(x, _ASYINCR),
                             torch.where(trend < 0, torch.full_like(x, _ASYDECR), torch.ones_like(x)))
        low = x - factor * (xold1 - low)
        upp = x + factor * (upp - xold1)
        low = torch.minimum(torch.maximum(low, x - 10.0 * span), x - 0.01 * span)
        upp = torch.maximum(torch.minimum(upp, x + 10.0 * span), x + 0.01 * span)
    alpha = torch.maximum(torch.maximum(low + _ALBEFA * (x - low), x - move * span), xmin)
    beta = torch.minimum(torch.minimum(upp - _ALBEFA * (upp - x), x + move * span), xmax)
    ux2, xl2 = (upp - x) ** 2, (x - low) ** 2
    reg = _RAA0 / torch.clamp(span, min=1e-5)
    pos, neg = torch.clamp(df0, min=0), torch.clamp(-df0, min=0)
    p0 = (1.001 * pos + 0.001 * neg + reg) * ux2
    q0 = (0.001 * pos + 1.001 * neg + reg) * xl2
    pos, neg = torch.clamp(dfdx, min=0), torch.clamp(-dfdx, min=0)
    P = (1.001 * pos + 0.001 * neg + reg) * ux2
    Q = (0.001 * pos + 1.001 * neg + reg) * xl2
    b = P @ (1.0 / (upp - x)) + Q @ (1.0 / (x - low)) - fval
    return low, upp, alpha, beta, p0, q0, P, Q, b


def subsolve(low, upp, alpha, beta, p0, q0, P, Q, a0, a, b, c, d, epsimin=1e-7, max_newton=500):
    """Primal-dual Newton solution of the MMA subproblem

        min  sum_j p0_j/(u_j - x_j) + q0_j/(x_j - l_j) + a0 z + sum_i (c_i y_i + d_i y_i^2 / 2)
        s.t. sum_j P_ij/(u_j - x_j) + Q_ij/(x_j - l_j) - a_i z - y_i <= b_i,
             alpha <= x <= beta, y >= 0, z >= 0,

    following the relaxed KKT conditions down to epsilon = epsimin (Svanberg
    2007, section 5).  The Newton system is reduced to (m+1) x (m+1) in the
    constraint multipliers and z.  Returns (x, y, z, lam, kkt) with kkt the
    infinity norm of the final relaxed-KKT residual."""
    n, m = p0.numel(), b.numel()
    dt, dev = p0.dtype, p0.device
    one_m = torch.ones(m, dtype=dt, device=dev)
    x = 0.5 * (alpha + beta)
    y, z, lam, s = one_m.clone(), torch.ones((), dtype=dt, device=dev), one_m.clone(), one_m.clone()
    xsi = torch.clamp(1.0 / (x - alpha), min=1.0)
    eta = torch.clamp(1.0 / (beta - x), min=1.0)
    mu = torch.clamp(0.5 * c, min=1.0)
    zet = torch.ones((), dtype=dt, device=dev)

    def residual(x, y, z, lam, xsi, eta, mu, zet, s, eps):
        ux1, xl1 = upp - x, x - low
        plam, qlam = p0 + P.t() @ lam, q0 + Q.t() @ lam
        gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
        parts = [plam / ux1 ** 2 - qlam / xl1 ** 2 - xsi + eta,
                 c + d * y - mu - lam,
                 (a0 - zet - a @ lam).reshape(1),
                 gvec - a * z - y + s - b,
                 xsi * (x - alpha) - eps, eta * (beta - x) - eps,
                 mu * y - eps, (zet * z - eps).reshape(1), lam * s - eps]
        r = torch.cat(parts)
        return torch.linalg.vector_norm(r), torch.linalg.vector_norm(r, ord=float("inf"))

    eps = 1.0
    kkt = float("inf")
    while eps > 0.99 * epsimin:
        rnorm, rmax = residual(x, y, z, lam, xsi, eta, mu, zet, s, eps)
        for _ in range(max_newton):
            if float(rmax) <= 0.9 * eps:
                break
            ux1, xl1 = upp - x, x - low
            plam, qlam = p0 + P.t() @ lam, q0 + Q.t() @ lam
            gvec = P @ (1.0 / ux1) + Q @ (1.0 / xl1)
            GG = P / ux1 ** 2 - Q / xl1 ** 2                      # d gvec / dx  (m, n)
            dpsidx = plam / ux1 ** 2 - qlam / xl1 ** 2
            delx = dpsidx - eps / (x - alpha) + eps / (beta - x)
            dely = c + d * y - lam - eps / y
            delz = a0 - a @ lam - eps / z
            dellam = gvec - a * z - y - b + eps / lam
            Dx = 2.0 * plam / ux1 ** 3 + 2.0 * qlam / xl1 ** 3 + xsi / (x - alpha) + eta / (beta - x)
            Dy = d + mu / y
            Dly = s / lam + 1.0 / Dy
            rhs_lam = dellam + dely / Dy - GG @ (delx / Dx)
            A = torch.diag(Dly) + (GG / Dx) @ GG.t()
            K = torch.zeros((m + 1, m + 1), dtype=dt, device=dev)
            K[:m, :m] = A
            K[:m, m] = a
            K[m, :m] = a
            K[m, m] = -zet / z
            sol = torch.linalg.solve(K, torch.cat([rhs_lam, delz.reshape(1)]))
            dlam, dz = sol[:m], sol[m]
            dx = -(delx + GG.t() @ dlam) / Dx
            dy = (dlam - dely) / Dy
            dxsi = eps / (x - alpha) - xsi - xsi * dx / (x - alpha)
            deta = eps / (beta - x) - eta + eta * dx / (beta - x)
            dmu = eps / y - mu - mu * dy / y
            dzet = eps / z - zet - zet * dz / z
            ds = eps / lam - s - s * dlam / lam
            # largest step keeping every positive quantity positive (1.01 margin)
            ratios = torch.cat([(-1.01 * dy / y), (-1.01 * dz / z).reshape(1), -1.01 * dlam / lam,
                                -1.01 * dxsi / xsi, -1.01 * deta / eta, -1.01 * dmu / mu,
                                (-1.01 * dzet / zet).reshape(1), -1.01 * ds / s,
                                -1.01 * dx / (x - alpha), 1.01 * dx / (beta - x)])
            step = 1.0 / max(1.0, float(ratios.max()))
            # backtrack until the relaxed-KKT residual decreases
            for _ in range(50):
                cand = (x + step * dx, y + step * dy, z + step * dz, lam + step * dlam, xsi + step * dxsi,
                        eta + step * deta, mu + step * dmu, zet + step * dzet, s + step * ds)
                rn, rm = residual(*cand, eps)
                if float(rn) < float(rnorm):
                    break
                step *= 0.5
            x, y, z, lam, xsi, eta, mu, zet, s = cand
            rnorm, rmax = rn, rm
        kkt = float(rmax)
        eps *= 0.1
    return x, y, z, lam, kkt


class MMA:
    """State of an MMA run: the last two iterates and the asymptotes."""

    def __init__(self, xmin, xmax, move, a0=1.0, a=None, c=None, d=None, num_constraints=1):
        self.xmin, self.xmax, self.move = xmin, xmax, float(move)
        m, dt, dev = num_constraints, xmin.dtype, xmin.device
        self.a0 = float(a0)
        self.a = torch.zeros(m, dtype=dt, device=dev) if a is None else torch.as_tensor(a, dtype=dt, device=dev)
        self.c = torch.full((m,), 1e4, dtype=dt, device=dev) if c is None else torch.as_tensor(c, dtype=dt, device=dev)
        self.d = torch.zeros(m, dtype=dt, device=dev) if d is None else torch.as_tensor(d, dtype=dt, device=dev)
        self.k = 0
        self.xold1 = self.xold2 = None
        self.low = self.upp = None
        self.last_kkt = None

    def step(self, x, f0, df0, fval, dfdx):
        """One MMA iteration from x given f0, its gradient, the constraint
        values fval (m,) and their gradients dfdx (m, n); returns the new x."""
        self.k += 1
        if self.xold1 is None:
            self.xold1, self.xold2 = x.clone(), x.clone()
        low, upp, alpha, beta, p0, q0, P, Q, b = _approximation(
            x, self.xold1, self.xold2, self.low, self.upp, self.k, self.xmin, self.xmax, df0, fval, dfdx, self.move)
        self.low, self.upp = low, upp
        xnew, _, _, _, self.last_kkt = subsolve(low, upp, alpha, beta, p0, q0, P, Q, self.a0, self.a, b, self.c,
                                                self.d)
        self.xold2, self.xold1 = self.xold1, x.clone()
        return xnew


# ---- filter and the optimisation loop ---------------------------------------------

def compute_filter_kd_tree(fe):
    """(H, Hs) over the design cells ``fe.flex_inds`` (all cells when the
    attribute is absent): H[i, j] = max(rmin -
    |c_i - c_j|, 0) for the 20 nearest centroids c_j of c_i, rmin = 1.5 x the
    average element size; Hs its row sums.  H is a torch sparse CSR matrix
    (host), Hs a (n, 1) tensor."""
    from scipy.spatial import cKDTree
    import scipy.sparse as sp
    flex = np.asarray(getattr(fe, "flex_inds", np.arange(len(fe.cells)))).reshape(-1)
    centroids = fe.points[fe.cells].mean(axis=1)[flex]
    avg_size = (fe.JxW().sum() / len(fe.cells)) ** (1.0 / fe.dim)
    rmin = 1.5 * avg_size
    k = min(20, len(flex))
    dd, ii = cKDTree(centroids).query(centroids, k)
    dd, ii = dd.reshape(len(flex), k), ii.reshape(len(flex), k)
    rows = np.repeat(np.arange(len(flex)), k)
    Hsp = sp.csr_array((np.maximum(rmin - dd, 0.0).reshape(-1), (rows, ii.reshape(-1))),
                       shape=(len(flex), len(flex)))
    Hsp.sum_duplicates()
    Hsp.sort_indices()
    with warnings.catch_warnings():  # torch flags its CSR tensors as beta
        warnings.simplefilter("ignore", UserWarning)
        H = torch.sparse_csr_tensor(torch.from_numpy(Hsp.indptr.astype(np.int64)),
                                    torch.from_numpy(Hsp.indices.astype(np.int64)),
                                    torch.from_numpy(Hsp.data.astype(np.float64)), size=Hsp.shape,
                                    check_invariants=True)
    Hs = torch.from_numpy(np.asarray(Hsp.sum(axis=1)).reshape(-1, 1).astype(np.float64))
    return H, Hs


def applySensitivityFilter(ft, rho, dJ, dvc):  # noqa: N802 - the reference's name
    """dJ <- H (rho dJ / max(1e-3, rho) / Hs), and the same for each
    constraint gradient in dvc (m, n, 1)."""
    H, Hs = ft["H"], ft["Hs"]
    w = rho / torch.clamp(rho, min=1e-3) / Hs
    dJ = H @ (w * dJ)
    dvc = torch.stack([H @ (w * g) for g in dvc])
    return dJ, dvc


def applyDensityFilter(ft, rho):  # noqa: N802 - the reference's name
    return ft["H"] @ rho / ft["Hs"]


def optimize(fe, rho_ini, optimizationParams, objectiveHandle, consHandle, numConstraints,  # noqa: N803
             density_filtering=False, sensitivity_filtering=True, device=None):
    """Topology optimisation by MMA (the reference's mma.optimize).

    rho_ini (n, 1) over ``fe.flex_inds``; optimizationParams {'maxIters',
    'movelimit'}; ``J, dJ = objectiveHandle(rho)`` and ``vc, dvc =
    consHandle(rho, iteration)`` (vc (m,), dvc (m, n, 1) or (m, n)), numpy
    or torch.  Returns the final rho (n, 1), of rho_ini's type.  Per-iteration
    values are kept in ``optimize.history`` (J, constraint values, MMA's
    final relaxed-KKT residual, the MMA step's wall time)."""
    as_numpy = not isinstance(rho_ini, torch.Tensor)
    if device is None:
        device = rho_ini.device if isinstance(rho_ini, torch.Tensor) else (
            torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else torch.device("cpu"))
    rho = torch.as_tensor(np.asarray(rho_ini) if as_numpy else rho_ini, dtype=torch.float64, device=device)
    rho = rho.reshape(-1, 1).clone()
    n, m = rho.shape[0], int(numConstraints)
    ft = _to_device_filter(compute_filter_kd_tree(fe), device)
    mma = MMA(torch.zeros(n, dtype=torch.float64, device=device), torch.ones(n, dtype=torch.float64, device=device),
              optimizationParams["movelimit"], a0=1.0, num_constraints=m)
    history = []

    def give(t):
        return t.detach().cpu().numpy().reshape(rho_ini.shape) if as_numpy else t.reshape(rho_ini.shape)

    for loop in range(1, int(optimizationParams["maxIters"]) + 1):
        rho_phys = applyDensityFilter(ft, rho) if density_filtering else rho
        J, dJ = objectiveHandle(give(rho_phys))
        vc, dvc = consHandle(give(rho_phys), loop)
        J = float(J)
        dJ = torch.as_tensor(np.asarray(dJ) if not isinstance(dJ, torch.Tensor) else dJ,
                             dtype=torch.float64, device=device).reshape(n, 1)
        vc = torch.as_tensor(np.asarray(vc) if not isinstance(vc, torch.Tensor) else vc,
                             dtype=torch.float64, device=device).reshape(m)
        dvc = torch.as_tensor(np.asarray(dvc) if not isinstance(dvc, torch.Tensor) else dvc,
                              dtype=torch.float64, device=device).reshape(m, n, 1)
        if sensitivity_filtering:
            dJ, dvc = applySensitivityFilter(ft, rho, dJ, dvc)
        t0 = time.perf_counter()
        x = mma.step(rho.reshape(-1), J, dJ.reshape(-1), vc, dvc.reshape(m, n))
        rho = x.reshape(n, 1)
        history.append({"iter": loop, "J": J, "constraints": vc.cpu().tolist(), "kkt": mma.last_kkt,
                        "mma_s": time.perf_counter() - t0})
    optimize.history = history
    return give(rho)


def _to_device_filter(ft, device):
    H, Hs = ft
    return {"H": H.to(device), "Hs": Hs.to(device)}
