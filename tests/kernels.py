"""Weak-form kernels for the cell-kernel path tests, written once over an
array namespace so that the product runs them as torch code on the GPU and
the oracle as numpy code (complex-step safe) on the CPU.  Signatures are the
reference's (problem.py:189-340)."""


def linear_elastic_universal(xp, E, nu):
    """The linear-elasticity weak form as a universal kernel (one variable, vec 3)."""
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))

    def kernel(sol, x, sg, jxw, vg, *iv):
        n = sg.shape[1]
        u = sol.reshape(n, 3)
        ug = xp.einsum("ai,qaj->qij", u, sg)
        eps = 0.5 * (ug + xp.swapaxes(ug, 1, 2))
        tr = xp.einsum("qii->q", eps)
        sig = 2.0 * mu * eps + lam * tr[:, None, None] * eye3(xp, sol)
        return xp.einsum("qij,qaj->ai", sig, vg[:, :, 0, :]).reshape(-1)

    return kernel


def eye3(xp, like):
    """3x3 identity of the namespace, dtype and device of ``like``."""
    if hasattr(like, "device"):
        return xp.eye(3, dtype=like.dtype, device=like.device)
    return xp.eye(3)


def neo_hookean_universal(xp, E, nu):
    """The compressible Neo-Hookean weak form (hyperelastic3d_common.py:152-169)
    as a universal kernel: P = mu J^-2/3 (F - I1/3 F^-T) + kappa J (J-1) F^-T."""
    mu = E / (2.0 * (1.0 + nu))
    kappa = E / (3.0 * (1.0 - 2.0 * nu))

    def kernel(sol, x, sg, jxw, vg, *iv):
        n = sg.shape[1]
        u = sol.reshape(n, 3)
        F = xp.einsum("ai,qaj->qij", u, sg) + eye3(xp, sol)
        J = xp.linalg.det(F)
        Finv_T = xp.swapaxes(xp.linalg.inv(F), 1, 2)
        I1 = xp.einsum("qij,qij->q", F, F)
        m = mu * J ** (-2.0 / 3.0)
        P = m[:, None, None] * (F - (I1 / 3.0)[:, None, None] * Finv_T) + (kappa * J * (J - 1.0))[:, None, None] * Finv_T
        return xp.einsum("qij,qaj->ai", P, vg[:, :, 0, :]).reshape(-1)

    return kernel


def svk_tensor_map(xp, E, nu):
    """Saint Venant-Kirchhoff tensor map with a per-point stiffness scale:
    P = s F (lambda tr(E) I + 2 mu E), E = (F^T F - I)/2."""
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))

    def tensor_map(u_grad, s):
        I = eye3(xp, u_grad)  # noqa: E741
        F = u_grad + I
        Eg = 0.5 * (F.T @ F - I)
        S = lam * xp.trace(Eg) * I + 2.0 * mu * Eg
        return s * (F @ S)

    return tensor_map


def thermoelastic_universal(xp, nu_nodes, NT, E, nu, beta, k, f):
    """Two variables: u (vec 3, nu_nodes per cell) and T (vec 1, the shape
    values NT (nq, nT) at the quadrature points).  u: div sigma = 0 with
    sigma = lambda tr(eps) I + 2 mu eps - beta T I; T: -div(k c grad T) = f,
    c a per-cell conductivity scale (internal variable, one value per cell)."""
    mu = E / (2.0 * (1.0 + nu))
    lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))

    def kernel(sol, x, sg, jxw, vg, c):
        n3 = nu_nodes * 3
        u = sol[:n3].reshape(nu_nodes, 3)
        T = sol[n3:]
        ug = xp.einsum("ai,qaj->qij", u, sg[:, :nu_nodes, :])
        eps = 0.5 * (ug + xp.swapaxes(ug, 1, 2))
        Tq = xp.einsum("a,qa->q", T, NT)
        tr = xp.einsum("qii->q", eps)
        sig = 2.0 * mu * eps + (lam * tr - beta * Tq)[:, None, None] * eye3(xp, sol)
        ru = xp.einsum("qij,qaj->ai", sig, vg[:, :nu_nodes, 0, :]).reshape(-1)
        gT = xp.einsum("a,qaj->qj", T, sg[:, nu_nodes:, :])
        rT = k * c * xp.einsum("qj,qaj->a", gT, vg[:, nu_nodes:, 0, :]) - f * xp.einsum("qa,q->a", NT, jxw[1])
        return xp.concatenate([ru, rT])

    return kernel


def robin_surface(xp, nu_nodes, h, T_inf):
    """Surface universal kernel: h (T - T_inf) w on the selected faces, for
    the second variable (T)."""

    def kernel(sol, x, fsv, fsg, nanson):
        n3 = nu_nodes * 3
        T = sol[n3:]
        NT = fsv[:, nu_nodes:]
        Tq = xp.einsum("a,qa->q", T, NT)
        rT = h * xp.einsum("q,qa,q->a", Tq - T_inf, NT, nanson[1])
        return xp.concatenate([0.0 * sol[:n3], rT])

    return kernel
