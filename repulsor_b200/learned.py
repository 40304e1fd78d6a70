"""Learned per-cluster preconditioner for TangentPointMetric0.Solve.

The network (16 -> 64 -> 64 -> 3, GELU, BF16 weights with FP32 accumulation) lives on
the device and is trained there by the library's own forward/backward/Adam kernels
(``rpb_mlp_*`` in include/repulsor_b200.h), either by the unrolled-CG loss
(``train_unrolled``: the energy functional after K preconditioned CG iterations,
differentiated through the CG recurrences) or on (residual, solve-correction) pairs that
plain CG solves of the metric produce (``train``):

    for a right-hand side b with exact solution x* = A^{-1} b (a tight plain CG solve)
    and a CG iterate x_k, the pair is r_k = b - A x_k and e_k = x* - x_k, so that
    A e_k = r_k.

``Solve(..., precond=PRECOND_LEARNED)`` then runs flexible CG with z = M(r); when the
residual stops decreasing it switches to the reference preconditioner
(MultiplyPreconditioner) for the rest of the solve.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _capi
from ._capi import PRECOND_NONE, RepulsorError, check, dptr, fptr

__all__ = ["LearnedPreconditioner", "training_pairs", "train", "unrolled_sensitivities", "train_unrolled",
           "slow_residual", "NPARAM_OUTPUT_OFFSET"]

# offset of the output layer (W3, b3) in the parameter vector: W1 64x16, b1 64, W2 64x64, b2 64
NPARAM_OUTPUT_OFFSET = 64 * 16 + 64 + 64 * 64 + 64


class LearnedPreconditioner:
    """One MLP on a CUDA device; attach it to meshes with ``attach``."""

    def __init__(self, seed: int = 0, device: int = 0, params=None):
        lib = _capi.load()
        h = ctypes.c_void_p()
        check(lib.rpb_mlp_create(int(device), ctypes.c_uint64(seed), ctypes.byref(h)), "rpb_mlp_create")
        self._h = h
        self.device = device
        if params is not None:
            self.set_params(params)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _capi is not None and _capi._lib is not None:
            _capi._lib.rpb_mlp_destroy(h)
            self._h = None

    @staticmethod
    def param_count() -> int:
        return _capi.load().rpb_mlp_param_count()

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.param_count(), np.float32)
        check(_capi.load().rpb_mlp_get_params(self._h, fptr(out)), "rpb_mlp_get_params")
        return out

    def set_params(self, params):
        params = np.ascontiguousarray(params, dtype=np.float32)
        if params.size != self.param_count():
            raise RepulsorError(_capi.RPB_EINVAL, f"expected {self.param_count()} parameters, got {params.size}")
        check(_capi.load().rpb_mlp_set_params(self._h, fptr(params)), "rpb_mlp_set_params")

    def save(self, path):
        np.save(path, self.get_params())

    @classmethod
    def load(cls, path, device: int = 0):
        return cls(device=device, params=np.load(path))

    def eval(self, F, dO=None):
        """MLP outputs O (n x 3) for features F (n x 16); with dO also d(sum dO*O)/dparams."""
        F = np.ascontiguousarray(F, dtype=np.float32)
        n = F.shape[0]
        O = np.zeros((n, 3), np.float32)
        grad = None
        if dO is not None:
            dO = np.ascontiguousarray(dO, dtype=np.float32)
            grad = np.zeros(self.param_count(), np.float32)
        check(_capi.load().rpb_mlp_eval(self._h, fptr(F), n, None if dO is None else fptr(dO), fptr(O),
                                        None if grad is None else fptr(grad)), "rpb_mlp_eval")
        return O if dO is None else (O, grad)

    def attach(self, M):
        check(_capi.load().rpb_mesh_set_learned(M._h, self._h), "rpb_mesh_set_learned")
        M._learned = self          # keep the network alive while the mesh uses it

    @staticmethod
    def detach(M):
        check(_capi.load().rpb_mesh_set_learned(M._h, None), "rpb_mesh_set_learned")
        M._learned = None

    def apply(self, M, R):
        """z = M(R) on mesh M (attaches the network to M)."""
        self.attach(M)
        R = np.ascontiguousarray(R, dtype=np.float64)
        Z = np.zeros_like(R)
        check(_capi.load().rpb_tpm0_learned_apply(M._h, dptr(R), dptr(Z)), "rpb_tpm0_learned_apply")
        return Z

    def apply_pair(self, M, R, Y):
        """(M(R), M_R(Y)): the application to R and, with the gains it gave, to Y."""
        self.attach(M)
        R = np.ascontiguousarray(R, dtype=np.float64)
        Y = np.ascontiguousarray(Y, dtype=np.float64)
        Z, ZY = np.zeros_like(R), np.zeros_like(R)
        check(_capi.load().rpb_tpm0_learned_apply_pair(M._h, dptr(R), dptr(Y), dptr(Z), dptr(ZY)),
              "rpb_tpm0_learned_apply_pair")
        return Z, ZY

    def train_step_sens(self, M, R, G, lr=1e-3, reg=0.0, want_grad=False):
        """One Adam step (none for lr <= 0) on sum_k G[k] . M(R[k]) over the pairs of mesh M;
        returns that objective before the step (and its gradient with want_grad)."""
        R = np.ascontiguousarray(R, dtype=np.float64)
        G = np.ascontiguousarray(G, dtype=np.float64)
        if R.ndim == 2:
            R, G = R[None], G[None]
        obj = ctypes.c_double()
        grad = np.zeros(self.param_count(), np.float32) if want_grad else None
        check(_capi.load().rpb_mlp_train_step_sens(self._h, M._h, dptr(R), dptr(G), R.shape[0], float(lr), float(reg),
                                                   ctypes.byref(obj), None if grad is None else fptr(grad)),
              "rpb_mlp_train_step_sens")
        return (obj.value, grad) if want_grad else obj.value

    def train_step(self, M, metric, R, E, lr=1e-3, want_grad=False, reg=0.0):
        """One Adam step (none for lr <= 0) on the pairs (R[k], E[k]) of mesh M and the
        metric's exponents; returns the loss before the step (and its gradient with
        want_grad)."""
        R = np.ascontiguousarray(R, dtype=np.float64)
        E = np.ascontiguousarray(E, dtype=np.float64)
        if R.ndim == 2:
            R, E = R[None], E[None]
        loss = ctypes.c_double()
        grad = np.zeros(self.param_count(), np.float32) if want_grad else None
        check(_capi.load().rpb_mlp_train_step(self._h, M._h, metric.q, metric.p, dptr(R), dptr(E), R.shape[0], float(lr),
                                              float(reg), ctypes.byref(loss), None if grad is None else fptr(grad)),
              "rpb_mlp_train_step")
        return (loss.value, grad) if want_grad else loss.value


def training_pairs(M, metric, n_rhs=4, checkpoints=(0, 4, 16, 48, 128), seed=0, exact_tol=1e-9,
                   exact_max_iter=20000, smooth=0):
    """(R, E) pairs from plain CG solves of metric on mesh M.

    For each of n_rhs seeded right-hand sides b (column means removed, optionally
    smoothed by `smooth` passes of vertex averaging over the simplices), x* is solved
    by plain CG to exact_tol; every checkpoint k gives the CG iterate x_k after k
    iterations and the pair (b - A x_k, x* - x_k)."""
    from . import meshes

    V = M.VertexCoordinates()
    nV = V.shape[0]
    Rs, Es = [], []
    for j in range(n_rhs):
        b = meshes.random_rhs(nV, seed=seed + j, project=True)
        for _ in range(smooth):
            b = _smooth(M, b)
        xs = metric.Solve(M, 1.0, b, max_iter=exact_max_iter, tolerance=exact_tol, precond=PRECOND_NONE,
                          strict=False)
        for k in checkpoints:
            if k == 0:
                xk = np.zeros_like(b)
            else:
                xk = metric.Solve(M, 1.0, b, max_iter=k, tolerance=1e-30, precond=PRECOND_NONE, strict=False)
            r = b - metric.MultiplyMetric(M, 1.0, xk)
            Rs.append(r)
            Es.append(xs - xk)
    return np.stack(Rs), np.stack(Es)


def _smooth(M, b):
    S = M._S if hasattr(M, "_S") else None
    if S is None:
        return b
    acc = np.zeros_like(b)
    cnt = np.zeros(b.shape[0])
    for l in range(S.shape[1]):
        np.add.at(acc, S[:, l], b[S].mean(1))
        np.add.at(cnt, S[:, l], 1.0)
    out = acc / np.maximum(cnt, 1.0)[:, None]
    return out - out.mean(0)


def train(net: LearnedPreconditioner, metric, data, epochs=200, lr=1e-3, batch=4, seed=0, log=None, reg=1.0):
    """Adam over the (mesh, R, E) sets in `data`, `batch` pairs per step, with the gain
    penalty reg * mean(o^2). Returns the loss history (one mean per epoch, penalty excluded)."""
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        losses = []
        for M, R, E in data:
            order = rng.permutation(R.shape[0])
            for s in range(0, len(order), batch):
                idx = order[s:s + batch]
                losses.append(net.train_step(M, metric, R[idx], E[idx], lr=lr, reg=reg))
        hist.append(float(np.mean(losses)))
        if log is not None:
            log(ep, hist[-1])
    return hist


def _cdot(a, b):
    return np.einsum("ij,ij->j", a, b)


def unrolled_sensitivities(net, M, metric, b, steps=30, loss="energy", hybrid=False, weight=None):
    """The loss of `steps` iterations of preconditioned CG with z = M(r) from x = 0, one CG
    per column, and its sensitivities to the preconditioner outputs, dL/dz_k, by the adjoint
    of the CG recurrences

        q_k = A p_k,  alpha_k = g_k / (p_k . q_k),  x_k+1 = x_k + alpha_k p_k,  r_k+1 = r_k - alpha_k q_k,
        z_k+1 = M(r_k+1),  g_k+1 = r_k+1 . z_k+1,  beta_k = g_k+1 / g_k,  p_k+1 = z_k+1 + beta_k p_k,

    run backwards; through z = M(r) the adjoint takes the application with the gains of
    that r held fixed (apply_pair). loss = "energy": L = -sum_c log(-phi_c(x_K)) with
    phi(x) = x.Ax/2 - b.x = -x.(b + r)/2, the functional CG minimizes (phi(x_K) - phi(x*) is
    half the squared A-norm of the error); loss = "residual": L = sum_c log(|r_K,c|^2 / |b_c|^2).
    hybrid: the preconditioner is z = P_ref r + w M(r) (RPB_PRECOND_HYBRID), P_ref the
    reference preconditioner (linear, symmetric) and w = (b, P_ref b) / (8 (b, M b)) (or
    `weight`) fixed for the solve; its adjoint adds P_ref to the frozen application.
    Returns (L, R, G): the residuals r_0 .. r_K-1 the preconditioner was applied to and the
    sensitivities of L to the network's outputs M(r_k), for train_step_sens."""
    b = np.ascontiguousarray(b, dtype=np.float64)
    A = lambda X: metric.MultiplyMetric(M, 1.0, X)
    w = 1.0
    if hybrid:
        Pref = lambda X: metric.MultiplyPreconditioner(M, 1.0, X)
        w = weight if weight is not None else 0.125 * float(np.sum(b * Pref(b))) / float(np.sum(b * net.apply(M, b)))
        apply = lambda X: Pref(X) + w * net.apply(M, X)
    else:
        apply = lambda X: net.apply(M, X)
    r, z, p, q = [b], [apply(b)], [], []
    p.append(z[0])
    g = [_cdot(r[0], z[0])]
    alpha, beta, delta = [], [], []
    x = np.zeros_like(b)
    for k in range(steps):
        qk = A(p[k])
        dk = _cdot(p[k], qk)
        ak = g[k] / dk
        x = x + ak * p[k]
        rk1 = r[k] - ak * qk
        q.append(qk); delta.append(dk); alpha.append(ak); r.append(rk1)
        if k + 1 < steps:
            zk1 = apply(rk1)
            gk1 = _cdot(rk1, zk1)
            bk = gk1 / g[k]
            z.append(zk1); g.append(gk1); beta.append(bk)
            p.append(zk1 + bk * p[k])
    if loss == "energy":
        phi = -0.5 * _cdot(x, b + r[steps])
        value = float(-np.sum(np.log(-phi)))
        xbar = r[steps] / phi                 # dL/dphi = -1/phi, dphi/dx = A x - b = -r
        rbar = np.zeros_like(b)
    elif loss == "residual":
        nb2, nr2 = _cdot(b, b), _cdot(r[steps], r[steps])
        value = float(np.sum(np.log(nr2 / nb2)))
        xbar = np.zeros_like(b)
        rbar = 2.0 * r[steps] / nr2
    else:
        raise ValueError("loss must be 'energy' or 'residual'")
    zbar = [np.zeros_like(b) for _ in range(steps)]
    pbar_next = np.zeros_like(b)
    for k in reversed(range(steps)):
        pbar = np.zeros_like(b)
        if k + 1 < steps:
            # p_k+1 = z_k+1 + beta_k p_k; beta_k = g_k+1 / g_k; g_k+1 = r_k+1 . z_k+1
            zbar[k + 1] += pbar_next
            bbar = _cdot(pbar_next, p[k])
            pbar += beta[k] * pbar_next
            gbar1 = bbar / g[k]
            gbar_k = -bbar * g[k + 1] / g[k] ** 2
            rbar = rbar + gbar1 * z[k + 1]
            zbar[k + 1] += gbar1 * r[k + 1]
            # z_k+1 = M(r_k+1) (+ P_ref r_k+1), gains held fixed
            _, mz = net.apply_pair(M, r[k + 1], zbar[k + 1])
            rbar = rbar + (Pref(zbar[k + 1]) + w * mz if hybrid else mz)
        else:
            gbar_k = np.zeros(b.shape[1])
        # x_k+1 = x_k + alpha_k p_k; r_k+1 = r_k - alpha_k q_k; alpha_k = g_k / delta_k;
        # delta_k = p_k . q_k; q_k = A p_k
        abar = _cdot(xbar, p[k]) - _cdot(rbar, q[k])
        pbar += alpha[k] * xbar
        qbar = -alpha[k] * rbar
        gbar_k = gbar_k + abar / delta[k]
        dbar = -abar * g[k] / delta[k] ** 2
        pbar += dbar * q[k]
        qbar = qbar + dbar * p[k]
        pbar += A(qbar)
        # g_k = r_k . z_k
        rbar = rbar + gbar_k * z[k]
        zbar[k] += gbar_k * r[k]
        pbar_next = pbar
    zbar[0] += pbar_next            # p_0 = z_0
    return value, np.stack(r[:steps]), w * np.stack(zbar)


def slow_residual(net, M, metric, b, iterations):
    """The residual b - A x after `iterations` flexible-CG steps from x = 0 with the
    preconditioner `net`, scaled to unit norm. Its error lies in the modes that the
    preconditioned solve resolves last, which set the iteration count to a tight tolerance;
    as a training right-hand side it points the unrolled loss at them."""
    from ._capi import PRECOND_LEARNED

    net.attach(M)
    b = np.ascontiguousarray(b, dtype=np.float64)
    X = metric.Solve(M, 1.0, b, max_iter=iterations, tolerance=1e-30, precond=PRECOND_LEARNED, strict=False)
    r = b - metric.MultiplyMetric(M, 1.0, X)
    r -= r.mean(axis=0)
    return r / np.linalg.norm(r)


def train_unrolled(net, metric, meshes_rhs, epochs=1, lr=1e-3, steps=30, reg=1e-3, seed=0, log=None, loss="energy",
                   hybrid=False):
    """Adam on the unrolled-CG loss: for every (mesh, right-hand side) pair in meshes_rhs,
    the sensitivities of `steps` preconditioned CG iterations with the current network (as
    the whole preconditioner, or with hybrid as the learned part of z = P_ref r + w M(r)),
    then one step on them. Returns the mean loss per epoch (the loss of the network each
    pair was visited with)."""
    rng = np.random.default_rng(seed)
    hist = []
    for ep in range(epochs):
        losses = []
        for i in rng.permutation(len(meshes_rhs)):
            M, b = meshes_rhs[i]
            value, R, G = unrolled_sensitivities(net, M, metric, b, steps, loss, hybrid)
            net.train_step_sens(M, R, G, lr=lr, reg=reg)
            losses.append(value)
        hist.append(float(np.mean(losses)))
        if log is not None:
            log(ep, hist[-1])
    return hist
