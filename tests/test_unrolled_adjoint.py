"""The adjoint of the unrolled preconditioned CG (repulsor_b200.learned.unrolled_sensitivities)
against finite differences, on the CPU with small dense stand-ins for the metric and the
preconditioner, for both losses (the CG energy functional and the residual norm): for a
linear preconditioner M_t = M0 + t M1 the derivative of the loss is
dL/dt = sum_k G_k . M1 r_k, where G_k are the returned sensitivities; likewise for the
hybrid preconditioner P_ref + w M_t with the weight w held fixed."""
import numpy as np
import pytest

from repulsor_b200.learned import unrolled_sensitivities


class _Dense:
    def __init__(self, Mat):
        self.Mat = Mat

    def apply(self, M, R):
        return self.Mat @ R

    def apply_pair(self, M, R, Y):
        return self.Mat @ R, self.Mat @ Y


class _Metric:
    def __init__(self, A, P=None):
        self.A, self.P = A, P

    def MultiplyMetric(self, M, alpha, X):
        return alpha * (self.A @ X)

    def MultiplyPreconditioner(self, M, alpha, X):
        return alpha * (self.P @ X)


def _spd(n, rng, cond):
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * np.geomspace(1.0, cond, n)) @ Q.T


@pytest.mark.parametrize("loss", ["energy", "residual"])
def test_unrolled_cg_sensitivities_match_finite_differences(loss):
    rng = np.random.default_rng(0)
    n = 40
    A = _spd(n, rng, 1e3)
    M0 = _spd(n, rng, 10.0)
    S = rng.standard_normal((n, n))
    M1 = 0.1 * (S + S.T)
    b = rng.standard_normal((n, 3))
    metric = _Metric(A)
    for steps in (1, 5, 12):
        value, R, G = unrolled_sensitivities(_Dense(M0), None, metric, b, steps, loss)
        assert R.shape == (steps, n, 3) and G.shape == (steps, n, 3)
        analytic = float(sum(np.sum(G[k] * (M1 @ R[k])) for k in range(steps)))
        h = 1e-4      # smaller steps lose digits to the rounding CG amplifies
        lp, _, _ = unrolled_sensitivities(_Dense(M0 + h * M1), None, metric, b, steps, loss)
        lm, _, _ = unrolled_sensitivities(_Dense(M0 - h * M1), None, metric, b, steps, loss)
        fd = (lp - lm) / (2 * h)
        assert abs(analytic - fd) <= 1e-5 * max(1.0, abs(fd)), (steps, analytic, fd)


@pytest.mark.parametrize("loss", ["energy", "residual"])
def test_hybrid_sensitivities_match_finite_differences(loss):
    rng = np.random.default_rng(1)
    n = 40
    A = _spd(n, rng, 1e3)
    P = _spd(n, rng, 30.0) * 1e-2
    M0 = _spd(n, rng, 10.0)
    S = rng.standard_normal((n, n))
    M1 = 0.1 * (S + S.T)
    b = rng.standard_normal((n, 3))
    metric = _Metric(A, P)
    w = 0.37
    for steps in (1, 6):
        value, R, G = unrolled_sensitivities(_Dense(M0), None, metric, b, steps, loss, hybrid=True, weight=w)
        analytic = float(sum(np.sum(G[k] * (M1 @ R[k])) for k in range(steps)))
        h = 1e-4
        lp, _, _ = unrolled_sensitivities(_Dense(M0 + h * M1), None, metric, b, steps, loss, hybrid=True, weight=w)
        lm, _, _ = unrolled_sensitivities(_Dense(M0 - h * M1), None, metric, b, steps, loss, hybrid=True, weight=w)
        fd = (lp - lm) / (2 * h)
        assert abs(analytic - fd) <= 1e-5 * max(1.0, abs(fd)), (steps, analytic, fd)
