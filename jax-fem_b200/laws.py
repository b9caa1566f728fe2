"""Registered constitutive laws: what ``get_tensor_map`` returns here.

The reference's ``get_tensor_map`` returns a JAX-traceable callable that the
framework differentiates with jacfwd (problem.py:262-266, 283-285).  This
implementation has no tracer and no CPU fallback, so each supported law is a
descriptor naming a hand-written CUDA kernel with its exact tangent:

================  ==========================================  ===================
descriptor        stress                                     internal_vars
================  ==========================================  ===================
Laplace()         P = grad u                                 -
LinearElastic     sigma = lmbda tr(eps) I + 2 mu eps          -
SIMPElastic       LinearElastic with E = Emin+(E0-Emin)t^p    [theta (C,Q[,1])]
NeoHookean        P = dpsi/dF (compressible Neo-Hookean)      [] or [scale (C,Q)]
J2Plasticity      radial return + linear iso. hardening       [sigma_old, eps_old(, alpha_old)]
================  ==========================================  ===================

``as_law`` also accepts a plain callable when it is recognisably the
identity (the Poisson test's ``lambda x: x``) or a linear isotropic elastic
stress; anything else raises ``NotImplementedError``.

Each law also has a torch form (``torch_map``) for the cell-kernel path;
on 2D problems the elastic and inelastic laws act in plane strain through
``plane_strain``.
"""
import numpy as np

from . import _native as nat


class Law:
    law_id = None
    vec = 3

    def params(self):
        return []

    def torch_map(self):
        """The law as a torch tensor map ``P(u_grad, *ivars at a point)`` for
        the cell-kernel path (problem.py:189-214 form), where the CUDA
        kernels do not apply (several variables, universal kernels,
        u-dependent loads)."""
        raise NotImplementedError(f"{type(self).__name__} has no torch form for the cell-kernel path")


class Laplace(Law):
    """Tensor map P = grad u (the linear Poisson test, test_linear_poisson.py:15-17)."""
    law_id = nat.LAW_LAPLACE
    vec = None  # any vec

    def torch_map(self):
        return lambda u_grad, *ivars: u_grad


class LinearElastic(Law):
    """Isotropic linear elasticity (test_linear_elasticity_cube.py:16-25)."""
    law_id = nat.LAW_LINEAR

    def __init__(self, E, nu):
        self.E, self.nu = float(E), float(nu)

    def params(self):
        return [self.E, self.nu]

    def torch_map(self):
        return _elastic_map(self.E, self.nu)


def _elastic_map(E, nu):
    mu = E / (2.0 * (1.0 + nu))
    lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))

    def stress(u_grad, scale=None):
        import torch
        eps = 0.5 * (u_grad + u_grad.transpose(-1, -2))
        sig = lm * torch.diagonal(eps, dim1=-2, dim2=-1).sum(-1)[..., None, None] * torch.eye(
            3, dtype=u_grad.dtype, device=u_grad.device) + 2.0 * mu * eps
        return sig if scale is None else scale * sig

    return stress


class SIMPElastic(Law):
    """SIMP-penalised linear elasticity (top_opt/fem_model.py:67-80 in the reference)."""
    law_id = nat.LAW_SIMP

    def __init__(self, E0=70e3, Emin=70.0, nu=0.3, penal=3.0):
        self.E0, self.Emin, self.nu, self.penal = float(E0), float(Emin), float(nu), float(penal)

    def params(self):
        return [self.E0, self.Emin, self.nu, self.penal]

    def torch_map(self):
        unit = _elastic_map(1.0, self.nu)
        E0, Emin, p = self.E0, self.Emin, self.penal

        def stress(u_grad, theta):
            return unit(u_grad, (Emin + (E0 - Emin) * theta.reshape(()) ** p))

        return stress


class NeoHookean(Law):
    """psi = mu/2 (J^-2/3 I1 - 3) + kappa/2 (J-1)^2, P = dpsi/dF
    (test_hyper_elasticity.py:17-33; scalability/hyperelastic3d_common.py:152-202)."""
    law_id = nat.LAW_NEO_HOOKEAN

    def __init__(self, E, nu):
        self.E, self.nu = float(E), float(nu)

    def params(self):
        return [self.E, self.nu]

    def torch_map(self):
        mu = self.E / (2.0 * (1.0 + self.nu))
        kappa = self.E / (3.0 * (1.0 - 2.0 * self.nu))

        def stress(u_grad, scale=None):
            import torch
            F = u_grad + torch.eye(3, dtype=u_grad.dtype, device=u_grad.device)
            # cofactor matrix (J F^-T) and J by cofactor expansion
            c0 = torch.linalg.cross(F[1], F[2])
            c1 = torch.linalg.cross(F[2], F[0])
            c2 = torch.linalg.cross(F[0], F[1])
            cof = torch.stack([c0, c1, c2])
            J = (F[0] * c0).sum()
            H = cof / J
            I1 = (F * F).sum()
            P = mu * J ** (-2.0 / 3.0) * (F - I1 / 3.0 * H) + kappa * J * (J - 1.0) * H
            return P if scale is None else scale.reshape(()) * P

        return stress


class J2Plasticity(Law):
    """Small-strain J2 radial return (test_plasticity.py:42-64) with linear
    isotropic hardening modulus H (H=0 is the reference's perfect plasticity)."""
    law_id = nat.LAW_J2

    def __init__(self, E, nu, sigma_y, H=0.0):
        self.E, self.nu, self.sigma_y, self.H = float(E), float(nu), float(sigma_y), float(H)

    def params(self):
        return [self.E, self.nu, self.sigma_y, self.H]

    def torch_state(self):
        """The radial return in torch form: (u_grad (3,3), sigma_old,
        eps_old, alpha_old) at one point -> (sigma, eps, alpha), the state a
        converged increment commits.  The plastic branch is chosen with
        torch.where and the deviatoric norm's square root is guarded at
        zero, so forward-mode derivatives stay finite on both branches."""
        E, nu, sy0, Hh = self.E, self.nu, self.sigma_y, self.H
        mu = E / (2.0 * (1.0 + nu))
        lm = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu))

        def state(u_grad, sigma_old, eps_old, alpha_old=None):
            import torch
            I = torch.eye(3, dtype=u_grad.dtype, device=u_grad.device)  # noqa: E741
            eps = 0.5 * (u_grad + u_grad.T)
            de = eps - eps_old.reshape(3, 3)
            st = lm * torch.trace(de) * I + 2.0 * mu * de + sigma_old.reshape(3, 3)
            s = st - torch.trace(st) / 3.0 * I
            ss = 1.5 * (s * s).sum()
            pos = ss > 0.0
            q = torch.where(pos, torch.sqrt(torch.where(pos, ss, torch.ones_like(ss))), torch.zeros_like(ss))
            a = alpha_old.reshape(()) if alpha_old is not None else torch.zeros_like(ss)
            f = q - (sy0 + Hh * a)
            dg = torch.where(f > 0.0, f, torch.zeros_like(f)) / (3.0 * mu + Hh)
            qs = torch.where(pos, q, torch.ones_like(q))
            sigma = st - torch.where(pos, 3.0 * mu * dg / qs, torch.zeros_like(q)) * s
            return sigma, eps, a + dg

        return state

    def torch_map(self):
        """The stress of ``torch_state`` as a tensor map of (u_grad,
        sigma_old, eps_old, alpha_old)."""
        state = self.torch_state()

        def stress(u_grad, sigma_old, eps_old, alpha_old=None):
            return state(u_grad, sigma_old, eps_old, alpha_old)[0]

        return stress


def plane_strain(tensor_map):
    """A 3D tensor map on a 2D problem: the in-plane gradient (vec, 2) is
    the upper-left block of a 3x3 gradient (no out-of-plane displacement or
    variation) and the in-plane block of the 3D stress is returned, so the
    2D weak form is the 3D one restricted to in-plane fields."""
    import torch

    def tm2(u_grad, *ivars):
        v, d = u_grad.shape[-2:]
        g = torch.nn.functional.pad(u_grad, (0, 3 - d, 0, 3 - v))
        return tensor_map(g, *ivars)[..., :v, :d]

    return tm2


def _probe(fn, vec, dim, rng):
    x = rng.standard_normal((vec, dim))
    return x, np.asarray(fn(x), dtype=np.float64)


def as_law(obj, vec, dim=3):
    """Turn what ``get_tensor_map`` returned into a registered law."""
    if isinstance(obj, Law):
        if obj.vec is not None and obj.vec != vec:
            raise NotImplementedError(f"{type(obj).__name__} needs vec={obj.vec}, problem has vec={vec}")
        return obj
    if not callable(obj):
        raise NotImplementedError(f"get_tensor_map returned {type(obj)}; expected a law descriptor")
    try:
        nargs = obj.__code__.co_argcount
    except AttributeError:
        nargs = 1
    if nargs != 1:
        raise NotImplementedError(
            "tensor maps with internal variables must be registered laws "
            "(SIMPElastic, NeoHookean, J2Plasticity)")
    rng = np.random.default_rng(1234)
    try:
        samples = [_probe(obj, vec, dim, rng) for _ in range(4)]
    except Exception as e:  # noqa: BLE001 - any failure means "not recognisable"
        raise NotImplementedError(f"cannot evaluate tensor map on numpy input: {e}") from e
    if all(y.shape == x.shape and np.allclose(y, x, rtol=1e-13, atol=1e-13) for x, y in samples):
        return Laplace()
    if vec == 3 and dim == 3:
        # linear isotropic elasticity: sigma(eps) = lmbda tr I + 2 mu eps
        e11 = np.zeros((3, 3))
        e11[0, 0] = 1.0
        s = np.asarray(obj(e11), dtype=np.float64)
        lmbda = s[1, 1]
        mu = 0.5 * (s[0, 0] - lmbda)
        if mu > 0:
            E = mu * (3 * lmbda + 2 * mu) / (lmbda + mu)
            nu = lmbda / (2 * (lmbda + mu))
            cand = LinearElastic(E, nu)
            ok = True
            for x, y in samples:
                eps = 0.5 * (x + x.T)
                ref = lmbda * np.trace(eps) * np.eye(3) + 2 * mu * eps
                ok &= y.shape == (3, 3) and np.allclose(y, ref, rtol=1e-11, atol=1e-9 * abs(mu))
            if ok:
                return cand
    raise NotImplementedError(
        "unrecognised tensor map: return a registered law (Laplace, LinearElastic, "
        "SIMPElastic, NeoHookean, J2Plasticity) from get_tensor_map")
