"""Smoothed-aggregation algebraic multigrid: the multigrid preconditioner for
meshes that are not box lattices.

The reference's optional AMGX path (solver.py:136-259) preconditions its
Krylov solve with an algebraic multigrid that needs no mesh structure.  This
is its counterpart here, ``precond='amg'`` (and the reference's
``amgx_solver`` key): a smoothed-aggregation hierarchy (Vanek, Mandel and
Brezina, Computing 56, 1996) built on the host from the Dirichlet-eliminated
tangent and applied on the device as a V-cycle inside FP64 CG.

Setup (host, numpy / scipy):

- unknowns are grouped into nodes (the mesh's nodes on the finest level,
  the previous level's aggregates below); nodes i and j are strongly
  connected when ||A_ij||_F >= theta sqrt(||A_ii||_F ||A_jj||_F);
  Dirichlet-eliminated unknowns take no part;
- aggregation in three passes: a node with all its strong neighbours still
  free forms an aggregate with them; remaining nodes join a neighbouring
  aggregate; what is left forms aggregates with its free neighbours;
- the tentative prolongator T orthonormalises the near null space on each
  aggregate (QR, rank-revealing by the diagonal of R): rigid-body modes
  (translations and rotations about the mesh's centre) when vec equals the
  dimension, constants per component otherwise; R is the next level's near
  null space;
- P = (I - omega D^-1 A) T with omega = 4 / (3 rho(D^-1 A)) and the coarse
  operator P^T A P (symmetrised); levels are added until the coarsest has
  at most ``coarse_size`` unknowns, whose inverse is formed densely.

Apply (device): the finest operator is the problem's own block-CSR matrix;
every coarser operator and every transfer is a scalar CSR matrix applied by
the library's block-CSR product (``fem_bsr_spmv_f64``).  Each level smooths
with Chebyshev polynomials in the Jacobi-scaled operator on
[lmax/ratio, lmax], the same polynomial before and after the coarse
correction, so the V-cycle is symmetric.  The aggregates and T are kept
across Newton steps: a full setup re-forms P, the coarse operators and the
smoothers' scaling from the new tangent; a fine-only setup refreshes the
finest level's scaling only.
"""
import math

import numpy as np
import scipy.sparse as sp
import torch

from . import _native as nat


class _CSR:
    """A scalar CSR matrix on the device (y = M x), from a scipy matrix or a
    torch sparse CSR tensor."""

    def __init__(self, M, device):
        if isinstance(M, torch.Tensor):
            self.shape = tuple(M.shape)
            self.n_brows = M.shape[0]
            self.row_ptr = M.crow_indices().to(device=device, dtype=torch.int32).contiguous()
            self.col_idx = M.col_indices().to(device=device, dtype=torch.int32).contiguous()
            self.vals = M.values().to(device=device, dtype=torch.float64).contiguous()
            return
        M = sp.csr_matrix(M)
        M.sort_indices()
        self.shape = M.shape
        self.n_brows = M.shape[0]
        self.row_ptr = torch.from_numpy(M.indptr.astype(np.int32)).to(device)
        self.col_idx = torch.from_numpy(M.indices.astype(np.int32)).to(device)
        self.vals = torch.from_numpy(M.data.astype(np.float64)).to(device)

    def apply(self, x, y):
        nat.check(nat.lib().fem_bsr_spmv_f64(1, self.n_brows, nat.ptr(self.row_ptr), nat.ptr(self.col_idx),
                                             nat.ptr(self.vals), nat.ptr(x), nat.ptr(y), nat.stream_ptr()),
                  "amg product")
        return y


def strength(A, dof_node, n_nodes, theta):
    """Strong connections between nodes (CSR pattern, no diagonal) from the
    block Frobenius norms of A; unknowns with dof_node < 0 are left out."""
    keep = dof_node >= 0
    rows = np.flatnonzero(keep)
    N = sp.csr_matrix((np.ones(len(rows)), (rows, dof_node[keep])), shape=(A.shape[0], n_nodes))
    A2 = sp.csr_matrix(A).multiply(sp.csr_matrix(A)).tocsr()
    S = (N.T @ A2 @ N).tocoo()
    S.data = np.sqrt(S.data)
    d = np.zeros(n_nodes)
    on = S.row == S.col
    d[S.row[on]] = S.data[on]
    strong = (~on) & (S.data >= theta * np.sqrt(d[S.row] * d[S.col]))
    out = sp.csr_matrix((np.ones(strong.sum()), (S.row[strong], S.col[strong])), shape=(n_nodes, n_nodes))
    out.sort_indices()
    return out


def aggregate(S):
    """Aggregate number of every node (-1: none) and the aggregate count."""
    n = S.shape[0]
    ptr, idx = S.indptr, S.indices
    agg = np.full(n, -1, dtype=np.int64)
    na = 0
    for i in range(n):  # pass 1: a node and all its strong neighbours
        nb = idx[ptr[i]:ptr[i + 1]]
        if agg[i] < 0 and len(nb) and (agg[nb] < 0).all():
            agg[i] = na
            agg[nb] = na
            na += 1
    first = agg.copy()
    for i in range(n):  # pass 2: join a neighbouring aggregate of pass 1
        if first[i] < 0:
            cand = first[idx[ptr[i]:ptr[i + 1]]]
            cand = cand[cand >= 0]
            if len(cand):
                agg[i] = cand[0]
    for i in range(n):  # pass 3: the rest, with their free neighbours
        nb = idx[ptr[i]:ptr[i + 1]]
        if agg[i] < 0 and len(nb):
            agg[nb[agg[nb] < 0]] = na
            agg[i] = na
            na += 1
    return agg, na


def tentative(agg, na, dof_node, B):
    """(T, coarse near null space, coarse dof -> aggregate): per aggregate the
    Q factor of its unknowns' rows of B, columns kept while |R_jj| stays
    above 1e-10 of the largest."""
    n, m = B.shape
    d_agg = np.where(dof_node >= 0, agg[np.maximum(dof_node, 0)], -1)
    order = np.argsort(d_agg, kind="stable")
    bounds = np.searchsorted(d_agg[order], np.arange(na + 1))
    rows, cols, vals, Bc, owner = [], [], [], [], []
    nc = 0
    for a in range(na):
        dofs = order[bounds[a]:bounds[a + 1]]
        if len(dofs) == 0:
            continue
        Q, R = np.linalg.qr(B[dofs])
        dr = np.abs(np.diag(R))
        r = int(np.sum(dr > 1e-10 * max(dr.max(), 1e-300)))
        if r == 0:
            continue
        rows.append(np.repeat(dofs, r))
        cols.append(np.tile(nc + np.arange(r), len(dofs)))
        vals.append(Q[:, :r].reshape(-1))
        Bc.append(R[:r])
        owner.append(np.full(r, a))
        nc += r
    T = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, nc))
    return T, np.vstack(Bc), np.concatenate(owner)


def near_null_space(points, vec, free):
    """Rigid-body modes of node-major unknowns (vec == dim of points), or
    constants per component; rows of eliminated unknowns zeroed."""
    n_nodes, dim = points.shape
    if vec == dim and dim in (2, 3):
        x = points - points.mean(axis=0)
        x = x / max(np.abs(x).max(), 1e-300)
        cols = [np.eye(dim)[c][None, :].repeat(n_nodes, 0) for c in range(dim)]
        rots = [(0, 1), (1, 2), (2, 0)] if dim == 3 else [(0, 1)]
        for i, j in rots:
            r = np.zeros((n_nodes, dim))
            r[:, i], r[:, j] = -x[:, j], x[:, i]
            cols.append(r)
        B = np.stack([c.reshape(-1) for c in cols], axis=1)
    else:
        B = np.zeros((n_nodes * vec, vec))
        for c in range(vec):
            B[c::vec, c] = 1.0
    return B * free[:, None]


def spectral_radius(A, dinv, iters=15, seed=0):
    """Largest eigenvalue of D^-1 A by power iteration (host)."""
    x = np.random.default_rng(seed).random(A.shape[0])
    lam = 1.0
    for _ in range(iters):
        x /= np.linalg.norm(x)
        y = dinv * (A @ x)
        lam = float(x @ y)
        x = y
    return lam


def _t_csr(M, device):
    """scipy CSR -> torch sparse CSR (FP64, int64 indices) on device."""
    M = sp.csr_matrix(M)
    M.sort_indices()
    return torch.sparse_csr_tensor(torch.from_numpy(M.indptr.astype(np.int64)),
                                   torch.from_numpy(M.indices.astype(np.int64)),
                                   torch.from_numpy(M.data.astype(np.float64)), size=M.shape).to(device)


def _t_scipy(M):
    """torch sparse CSR -> scipy CSR (host copy)."""
    return sp.csr_matrix((M.values().cpu().numpy(), M.col_indices().cpu().numpy(), M.crow_indices().cpu().numpy()),
                         shape=tuple(M.shape))


def _t_diag(M):
    """Diagonal of a square torch sparse CSR matrix (dense vector)."""
    crow, col, val = M.crow_indices(), M.col_indices(), M.values()
    rows = torch.repeat_interleave(torch.arange(M.shape[0], device=val.device), crow[1:] - crow[:-1])
    d = torch.zeros(M.shape[0], dtype=val.dtype, device=val.device)
    on = rows == col
    d.index_add_(0, rows[on], val[on])
    return d


def _t_scale_rows(M, s):
    """diag(s) M for a torch sparse CSR matrix (same pattern)."""
    crow, col, val = M.crow_indices(), M.col_indices(), M.values()
    rows = torch.repeat_interleave(torch.arange(M.shape[0], device=val.device), crow[1:] - crow[:-1])
    return torch.sparse_csr_tensor(crow, col, val * s[rows], size=M.shape)


def _t_transpose(M):
    return M.t().to_sparse_csr()


def _t_spectral_radius(A, dinv, iters=15, seed=0):
    """Largest eigenvalue of D^-1 A by power iteration (A torch sparse CSR)."""
    g = torch.Generator(device=dinv.device).manual_seed(seed)
    x = torch.rand(A.shape[0], 1, dtype=torch.float64, device=dinv.device, generator=g)
    lam = torch.ones((), dtype=torch.float64, device=dinv.device)
    for _ in range(iters):
        x = x / x.norm()
        y = dinv[:, None] * (A @ x)
        lam = (x * y).sum()
        x = y
    return float(lam)


def galerkin_t(A, T):
    """(P, P^T A P) with P = (I - omega D^-1 A) T, omega = 4 / (3 rho(D^-1 A)),
    as sparse products on the operators' device (torch sparse CSR, FP64);
    the coarse operator symmetrised."""
    d = _t_diag(A)
    dinv = torch.where(d != 0, 1.0 / torch.where(d != 0, d, torch.ones_like(d)), torch.zeros_like(d))
    omega = 4.0 / (3.0 * _t_spectral_radius(A, dinv))
    AT = torch.sparse.mm(A, T)
    P = torch.add(T, _t_scale_rows(AT, omega * dinv), alpha=-1.0)
    Ac = torch.sparse.mm(_t_transpose(P), torch.sparse.mm(A, P))
    Ac = torch.add(Ac, _t_transpose(Ac)) * 0.5
    return P, Ac


class AMG:
    """Smoothed-aggregation AMG preconditioned CG for one problem (see the
    module docstring).  Interface of the multigrid objects of solver.mg_solve."""

    def __init__(self, problem, max_levels=10, coarse_size=500, theta=0.08, nu_fine=0):
        if problem.num_vars != 1:
            raise NotImplementedError("precond 'amg' needs a problem of one variable")
        self.problem = problem
        fe = problem.fes[0]
        self.node_vec, self.points = fe.vec, fe.points
        self.max_levels, self.coarse_size, self.theta = int(max_levels), int(coarse_size), float(theta)
        self.nu_fine = int(nu_fine)  # smoothing steps on the finest level (0: nu, as on the others)
        self.device = problem.dev().device
        self.T = None
        self.lmax = None
        self.first_rate = self.last_rate = None
        self.solves_on_coarse = 0
        self.setup_for = None

    # ---- setup -------------------------------------------------------------------
    def _fine_csr(self, A):
        """The fine operator as a torch sparse CSR matrix on its device: the
        block-CSR values gathered into scalar CSR order (the gather index is
        built once from the pattern)."""
        vec = A.vec
        if getattr(self, "_fine_map", None) is None:
            rp = A.row_ptr.cpu().numpy().astype(np.int64)
            ci = A.col_idx.cpu().numpy().astype(np.int64)
            nb = len(rp) - 1
            cnt = np.diff(rp)
            # entries in the order (block row b, component i, block k, component c):
            # scalar row r = vec b + i holds blocks k of block row b, columns vec ci[k] + c
            per_row = np.repeat(cnt, vec)  # blocks per scalar row
            crow = np.zeros(nb * vec + 1, dtype=np.int64)
            crow[1:] = np.cumsum(per_row * vec)
            r_k = np.repeat(np.arange(nb * vec), per_row)
            starts = np.concatenate([[0], np.cumsum(per_row)[:-1]]).astype(np.int64)
            t = np.arange(len(r_k)) - np.repeat(starts, per_row)
            b_of, i_of = r_k // vec, r_k % vec
            k = rp[b_of] + t
            k_rep, i_rep = np.repeat(k, vec), np.repeat(i_of, vec)
            c_rep = np.tile(np.arange(vec), len(k))
            col = ci[k_rep] * vec + c_rep
            gather = k_rep * vec * vec + i_rep * vec + c_rep
            dev = A.vals.device
            self._fine_map = (torch.from_numpy(crow).to(dev), torch.from_numpy(col).to(dev),
                              torch.from_numpy(gather).to(dev), (nb * vec, nb * vec))
        crow, col, gather, shape = self._fine_map
        return torch.sparse_csr_tensor(crow, col, A.vals.to(torch.float64)[gather], size=shape)

    def _hierarchy(self, A, Ah):
        """Aggregates and tentative prolongators of every level (first
        setup), with the Galerkin products of each level (needed for the
        next level's strength of connection) on A's device; returns the
        (P, coarse operator) torch pairs it formed.  Ah: host copy of A."""
        mask, _ = self.problem.dirichlet_device()
        free = (mask.cpu().numpy() == 0).astype(np.float64)
        vec = self.node_vec
        dof_node = np.where(free > 0, np.arange(Ah.shape[0]) // vec, -1)
        n_nodes = Ah.shape[0] // vec
        B = near_null_space(self.points, vec, free)
        self.T, self._Td, self.free = [], [], free
        Al, Al_h = A, Ah
        formed = []
        for _ in range(self.max_levels - 1):
            if Al_h.shape[0] <= self.coarse_size:
                break
            agg, na = aggregate(strength(Al_h, dof_node, n_nodes, self.theta))
            if na == 0:
                break
            T, B, owner = tentative(agg, na, dof_node, B)
            if T.shape[1] >= Al_h.shape[0]:
                break
            self.T.append(T)
            self._Td.append(_t_csr(T, A.values().device))
            formed.append(galerkin_t(Al, self._Td[-1]))
            Al = formed[-1][1]
            Al_h = _t_scipy(Al)
            dof_node, n_nodes = owner, na
        return formed

    def setup(self, A, fine_only=False):
        import time
        t0 = time.perf_counter()
        self._setup(A, fine_only)
        self.setup_seconds = getattr(self, "setup_seconds", 0.0) + time.perf_counter() - t0
        self.full_setups = getattr(self, "full_setups", 0) + (0 if fine_only else 1)
        self._setups = getattr(self, "_setups", 0) + 1  # the captured CG iteration reads this setup's buffers

    def _setup(self, A, fine_only=False):
        if A.vals.dtype != torch.float64:
            raise TypeError("AMG works on the FP64 fine operator")
        vec = A.vec
        blocks = A.vals.view(-1, vec, vec)[A.diag.long()]
        self.dinv0 = (1.0 / torch.diagonal(blocks, dim1=1, dim2=2).reshape(-1)).contiguous()
        if not fine_only or self.lmax is None:
            self.lmax = 1.1 * self._power(A)
        if not fine_only or self.T is None:
            Ad = self._fine_csr(A)
            formed = self._hierarchy(Ad, sp.csr_matrix(A.to_scipy())) if self.T is None else None
            self.levels = []  # (A_l on the device, D_l^-1, lmax_l) for l >= 1
            self.P, self.R = [], []
            Al = Ad
            for k, Td in enumerate(self._Td):
                P, Al = formed[k] if formed is not None else galerkin_t(Al, Td)
                self.P.append(_CSR(P, self.device))
                self.R.append(_CSR(_t_transpose(P), self.device))
                d = _t_diag(Al)
                dinv = torch.where(d != 0, 1.0 / torch.where(d != 0, d, torch.ones_like(d)), torch.zeros_like(d))
                self.levels.append((_CSR(Al, self.device), dinv.to(self.device),
                                    1.1 * _t_spectral_radius(Al, dinv)))
            Ad_dense = Al.to_dense()
            try:
                inv = torch.linalg.inv(Ad_dense)
            except RuntimeError:
                inv = torch.linalg.pinv(Ad_dense)
            self.coarse_inv = inv.to(self.device).contiguous()
            self.solves_on_coarse = 0
        self.setup_for = A

    def _power(self, A):
        """Largest eigenvalue of D^-1 A on the finest level (device power iteration)."""
        g = torch.Generator(device=A.vals.device).manual_seed(0)
        x = torch.rand(A.n_brows * A.vec, dtype=torch.float64, device=A.vals.device, generator=g)
        y = torch.empty_like(x)
        lam = torch.ones((), dtype=torch.float64, device=x.device)
        for _ in range(12):
            x /= x.norm()
            A.matvec(x, y)
            z = self.dinv0 * y
            lam = x.dot(z)
            x = z
        return float(lam)

    # ---- V-cycle -----------------------------------------------------------------
    @staticmethod
    def _chebyshev(matvec, dinv, lmax, b, z, nu, ratio, zero_start=False):
        """nu Chebyshev steps for A z = b in the Jacobi-scaled operator (z in place)."""
        lmin = lmax / ratio
        theta, delta = 0.5 * (lmax + lmin), 0.5 * (lmax - lmin)
        sigma = theta / delta
        rho = 1.0 / sigma
        r = b.clone() if zero_start else b - matvec(z)
        d = dinv * r / theta
        for k in range(nu):
            z += d
            if k == nu - 1:
                break
            r -= matvec(d)
            rho_new = 1.0 / (2.0 * sigma - rho)
            d = rho_new * rho * d + (2.0 * rho_new / delta) * (dinv * r)
            rho = rho_new
        return z

    def _vcycle(self, level, A, b, nu, ratio):
        """z ~ A_level^-1 b (a new tensor)."""
        if level == len(self.levels):
            return self.coarse_inv @ b
        if level == 0:
            matvec = lambda v: A.matvec(v.contiguous())  # noqa: E731
            dinv, lmax = self.dinv0, self.lmax
        else:
            Al, dinv, lmax = self.levels[level - 1]
            matvec = lambda v: Al.apply(v.contiguous(), torch.empty(Al.n_brows, dtype=v.dtype,  # noqa: E731
                                                                    device=v.device))
        nu_l = self.nu_fine if (level == 0 and self.nu_fine > 0) else nu
        z = torch.zeros_like(b)
        self._chebyshev(matvec, dinv, lmax, b, z, nu_l, ratio, zero_start=True)
        r = (b - matvec(z)).contiguous()
        R, P = self.R[level], self.P[level]
        rc = R.apply(r, torch.empty(R.n_brows, dtype=b.dtype, device=b.device))
        zc = self._vcycle(level + 1, A, rc, nu, ratio).contiguous()
        z += P.apply(zc, torch.empty(P.n_brows, dtype=b.dtype, device=b.device))
        return self._chebyshev(matvec, dinv, lmax, b, z, nu_l, ratio)

    def apply(self, A, r, nu=2, ratio=30.0):
        return self._vcycle(0, A, r.contiguous(), nu, ratio)

    # ---- outer CG ----------------------------------------------------------------
    def _cg_step(self, A, nu, ratio):
        """One CG iteration on the persistent state (self._cg), scalars on the
        device: q = A p, the curvature check, x += alpha p, r -= alpha q, then
        the V-cycle's z and the next direction."""
        c = self._cg
        A.matvec(c["p"], c["q"])
        pq = c["p"].dot(c["q"])
        ok = pq > 0
        c["bad"] |= ~ok
        alpha = torch.where(ok, c["rz"] / torch.where(ok, pq, 1.0), c["zero"])
        c["x"].add_(alpha * c["p"])
        c["r"].sub_(alpha * c["q"])
        z = self.apply(A, c["r"], nu, ratio)
        rz_new = c["r"].dot(z)
        c["p"].mul_(rz_new / c["rz"]).add_(z)
        c["rz"].copy_(rz_new)

    def solve(self, A, b, x, rtol, atol=0.0, maxiter=1000, nu=2, coarse_steps=None, ratio=30.0, check_every=4,
              max_restarts=3, strict=True):
        """Preconditioned CG on A x = b (x: initial guess, in place).

        The scalars stay on the device; the recursive residual is read every
        ``check_every`` iterations.  When it meets max(rtol ||b||, atol) the
        true residual b - A x is formed, and when that misses the target CG
        restarts from it (at most ``max_restarts`` times), as the native CG
        of krylov.cu does.  A step whose curvature p.Ap is not positive
        leaves x and r unchanged and ends the solve with FEM_ERR_BREAKDOWN at
        the next check (the operator is not positive definite: the Newton
        loop then retries with BiCGSTAB); ``maxiter`` iterations without
        convergence end it with FEM_ERR_NOT_CONVERGED, unless ``strict`` is
        False: the reference's AMGX call returns its last iterate whatever
        the residual (solver.py:200-209), and so does this solve then.  On
        the GPU one iteration (operator product, updates and the whole
        V-cycle) is captured as a CUDA graph after it has run once eagerly,
        and replayed; a new setup is captured anew.
        Returns (iterations, relative true residual)."""
        bn = float(b.norm())
        target = max(rtol * bn, atol)
        n, dev = b.numel(), b.device
        if getattr(self, "_cg", None) is None or self._cg["x"].numel() != n or self._cg["x"].device != dev:
            e = lambda: torch.empty(n, dtype=b.dtype, device=dev)  # noqa: E731
            self._cg = {"x": e(), "r": e(), "p": e(), "q": e(), "rz": torch.empty((), dtype=b.dtype, device=dev),
                        "bad": torch.zeros((), dtype=torch.bool, device=dev),
                        "zero": torch.zeros((), dtype=b.dtype, device=dev)}
            self._graph = None
        c = self._cg
        c["x"].copy_(x)
        key = (getattr(self, "_setups", 0), A.vals.data_ptr(), int(nu), float(ratio))
        use_graph = b.is_cuda and _graphs_enabled()
        total = 0
        for restart in range(max_restarts + 1):
            A.matvec(c["x"], c["q"])
            torch.sub(b, c["q"], out=c["r"])
            rn = float(c["r"].norm())
            if not math.isfinite(rn):
                raise nat.FEMNativeError(nat.FEM_ERR_NONFINITE, "AMG-CG: non-finite residual")
            if rn <= target:
                x.copy_(c["x"])
                return total, rn / bn if bn > 0 else rn
            if restart == max_restarts or total >= maxiter:
                break
            z = self.apply(A, c["r"], nu, ratio)
            c["p"].copy_(z)
            c["rz"].copy_(c["r"].dot(z))
            c["bad"].fill_(False)
            met = False
            while total < maxiter:
                total += 1
                if use_graph and self._graph is not None and self._graph_key == key:
                    self._graph.replay()
                else:
                    self._cg_step(A, nu, ratio)
                    if use_graph:
                        g = torch.cuda.CUDAGraph()
                        with torch.cuda.graph(g):
                            self._cg_step(A, nu, ratio)
                        self._graph, self._graph_key = g, key
                if total % check_every == 0 or total == maxiter:
                    if bool(c["bad"]):
                        raise nat.FEMNativeError(nat.FEM_ERR_BREAKDOWN,
                                                 "AMG-CG: the operator is not positive definite")
                    rn = float(c["r"].norm())
                    if not math.isfinite(rn):
                        raise nat.FEMNativeError(nat.FEM_ERR_NONFINITE, "AMG-CG: non-finite residual")
                    if rn <= target:
                        met = True
                        break
            if not met:
                break
        x.copy_(c["x"])
        if not strict:
            A.matvec(x, c["q"])
            rn = float((b - c["q"]).norm())
            return total, rn / bn if bn > 0 else rn
        raise nat.FEMNativeError(nat.FEM_ERR_NOT_CONVERGED,
                                 f"AMG-CG: relative residual {rn / bn if bn > 0 else rn:.3e} after {total} iterations "
                                 f"(target {target / bn if bn > 0 else target:.3e})")


def _graphs_enabled():
    import os
    return os.environ.get("FEM_AMG_GRAPHS", "1") != "0"
