"""Test infrastructure: numpy restatement of GPRat's FP64 GP-regression path.

This is the checker, never the product.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg import it.
It is pinned against the reference's golden file (data/data_1024/output.json)
and against the reference's own CPU code compiled from source
(``oracle/_ref``; see ``tests/test_oracle.py``).

Each function cites the reference code it restates (paths relative to the
reference project root).  Dense matrices replace the reference's tiles; the
arithmetic is the same FP64 algebra, so results agree to rounding.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence, Tuple

import numpy as np
import scipy.linalg as sla

LOG_2PI = math.log(2.0 * math.pi)


# --------------------------------------------------------------------------
# Inputs
def feature_matrix(series: np.ndarray, n_rows: int, n_reg: int) -> np.ndarray:
    """Row i is series[i : i + n_reg] (sliding window).

    core/src/cpu/gp_algorithms.cpp:22-26 reads input[i_global + k] for
    k < n_regressors, so the series must hold >= n_rows + n_reg - 1 values."""
    series = np.asarray(series, dtype=np.float64)
    if series.size < n_rows + n_reg - 1:
        raise ValueError("input series too short for the sliding window")
    idx = np.arange(n_rows)[:, None] + np.arange(n_reg)[None, :]
    return series[idx]


def load_data(path: str, n_samples: int, offset: int) -> np.ndarray:
    """utils::load_data (core/src/utils_c.cpp:54-81): `offset` leading zeros,
    then n_samples values read with %lf."""
    vals = np.loadtxt(path, dtype=np.float64, max_rows=n_samples)
    out = np.zeros(n_samples + offset)
    out[offset:] = vals[:n_samples]
    return out


def compute_test_tiles(n_test: int, n_tiles: int, n_tile_size: int) -> Tuple[int, int]:
    """utils::compute_test_tiles (core/src/utils_c.cpp:34-52)."""
    if n_test % n_tile_size > 0:
        return n_tiles, n_test // n_tiles
    return n_test // n_tile_size, n_tile_size


# --------------------------------------------------------------------------
# Covariance assembly
def sq_dist(xa: np.ndarray, xb: np.ndarray) -> np.ndarray:
    """sum_k (xa_ik - xb_jk)^2, summed in k order like
    compute_covariance_function (core/src/cpu/gp_algorithms.cpp:19-26)."""
    d = np.zeros((xa.shape[0], xb.shape[0]))
    for k in range(xa.shape[1]):
        diff = xa[:, k][:, None] - xb[:, k][None, :]
        d += diff * diff
    return d


def se_kernel(xa, xb, lengthscale: float, vertical_lengthscale: float) -> np.ndarray:
    """k = v * exp(-0.5 / l^2 * r^2) (core/src/cpu/gp_algorithms.cpp:27)."""
    return vertical_lengthscale * np.exp(-0.5 / (lengthscale * lengthscale) * sq_dist(xa, xb))


def covariance(x_train, n, n_reg, hyper) -> np.ndarray:
    """Full K with noise on the diagonal (gen_tile_covariance,
    core/src/cpu/gp_algorithms.cpp:30-62)."""
    X = feature_matrix(x_train, n, n_reg)
    K = se_kernel(X, X, hyper[0], hyper[1])
    K[np.diag_indices(n)] += hyper[2]
    return K


# --------------------------------------------------------------------------
# Pipelines (core/src/cpu/gp_functions.cpp)
class OracleGP:
    """Dense restatement of gprat::GP's CPU pipelines."""

    def __init__(self, x, y, n_tiles: int, n_tile_size: int, n_reg: int = 8,
                 kernel_params: Sequence[float] = (1.0, 1.0, 0.1),
                 trainable: Sequence[bool] = (True, True, True)):
        self.x = np.asarray(x, dtype=np.float64).copy()
        self.y = np.asarray(y, dtype=np.float64).copy()
        self.n_tiles, self.n_tile_size, self.n_reg = int(n_tiles), int(n_tile_size), int(n_reg)
        self.n = self.n_tiles * self.n_tile_size
        self.hyper = [float(v) for v in kernel_params]
        self.trainable = [bool(t) for t in trainable]
        self.m_T = [0.0, 0.0, 0.0]
        self.w_T = [0.0, 0.0, 0.0]

    # -- factorisation -----------------------------------------------------
    def _factor(self):
        K = covariance(self.x, self.n, self.n_reg, self.hyper)
        L = np.linalg.cholesky(K)
        return K, L

    def _alpha(self, L):
        """forward_solve_tiled + backward_solve_tiled
        (core/src/cpu/tiled_algorithms.cpp:61-115)."""
        z = sla.solve_triangular(L, self.y[: self.n], lower=True)
        return sla.solve_triangular(L, z, lower=True, trans="T")

    def cholesky(self) -> List[Optional[np.ndarray]]:
        """cpu::cholesky (core/src/cpu/gp_functions.cpp:18-78).  Lower tiles
        only; diagonal tiles keep K's strict upper triangle, because LAPACKE
        dpotrf2('L') leaves it untouched (core/src/cpu/adapter_cblas_fp64.cpp:19)."""
        K, L = self._factor()
        T, nt = self.n_tile_size, self.n_tiles
        out: List[Optional[np.ndarray]] = []
        for i in range(nt):
            for j in range(nt):
                if j > i:
                    out.append(None)
                    continue
                tile = L[i * T:(i + 1) * T, j * T:(j + 1) * T].copy()
                if i == j:
                    Kt = K[i * T:(i + 1) * T, j * T:(j + 1) * T]
                    iu = np.triu_indices(T, 1)
                    tile[iu] = Kt[iu]
                out.append(tile.reshape(-1))
        return out

    def _cross(self, x_test, m):
        Xs = feature_matrix(x_test, m, self.n_reg)
        X = feature_matrix(self.x, self.n, self.n_reg)
        return se_kernel(Xs, X, self.hyper[0], self.hyper[1])

    def predict(self, x_test, m_tiles: int, m_tile_size: int) -> np.ndarray:
        """cpu::predict (core/src/cpu/gp_functions.cpp:81-216)."""
        m = m_tiles * m_tile_size
        _, L = self._factor()
        alpha = self._alpha(L)
        return self._cross(x_test, m) @ alpha

    def predict_with_uncertainty(self, x_test, m_tiles: int, m_tile_size: int):
        """cpu::predict_with_uncertainty (core/src/cpu/gp_functions.cpp:218-450):
        mean = K* alpha; var = diag(K**) - colsum((L^-1 K*^T)^2)."""
        m = m_tiles * m_tile_size
        _, L = self._factor()
        alpha = self._alpha(L)
        Kx = self._cross(x_test, m)
        V = sla.solve_triangular(L, Kx.T, lower=True)
        prior = np.full(m, self.hyper[1])  # k(x,x) = v (gen_tile_prior_covariance)
        return Kx @ alpha, prior - np.sum(V * V, axis=0)

    def predict_with_full_cov(self, x_test, m_tiles: int, m_tile_size: int):
        """cpu::predict_with_full_cov (core/src/cpu/gp_functions.cpp:452-698):
        forms K** - V^T V and returns its diagonal."""
        m = m_tiles * m_tile_size
        _, L = self._factor()
        alpha = self._alpha(L)
        Kx = self._cross(x_test, m)
        V = sla.solve_triangular(L, Kx.T, lower=True)
        Xs = feature_matrix(x_test, m, self.n_reg)
        Sigma = se_kernel(Xs, Xs, self.hyper[0], self.hyper[1]) - V.T @ V
        return Kx @ alpha, np.diag(Sigma).copy()

    def posterior_covariance(self, x_test, m: int) -> np.ndarray:
        """Full posterior covariance K** - K*^T K^-1 K* (m x m)."""
        _, L = self._factor()
        Kx = self._cross(x_test, m)
        V = sla.solve_triangular(L, Kx.T, lower=True)
        Xs = feature_matrix(x_test, m, self.n_reg)
        return se_kernel(Xs, Xs, self.hyper[0], self.hyper[1]) - V.T @ V

    def calculate_loss(self) -> float:
        """cpu::compute_loss (core/src/cpu/gp_functions.cpp:700-781) with
        compute_loss / add_losses (core/src/cpu/gp_optimizer.cpp:187-218):
        0.5 * (y^T alpha + sum log(L_ii^2) + N log 2pi) / N."""
        _, L = self._factor()
        alpha = self._alpha(L)
        return nlml(self.y[: self.n], alpha, np.diag(L))

    # -- optimisation -------------------------------------------------------
    def gradient(self) -> Tuple[float, np.ndarray]:
        """Loss and gradient w.r.t. the unconstrained hyper-parameters, as in
        update_hyperparameter_tiled (core/src/cpu/tiled_algorithms.cpp:296-426):
        g = s * 0.5/N * (tr(K^-1 dK) - alpha^T dK alpha), s = sigmoid(softplus^-1(theta))."""
        n = self.n
        l, v, noise = self.hyper
        X = feature_matrix(self.x, n, self.n_reg)
        dist = -0.5 / (l * l) * sq_dist(X, X)  # gen_tile_distance (gp_optimizer.cpp:59-82)
        E = np.exp(dist)
        K = v * E
        K[np.diag_indices(n)] += noise
        L = np.linalg.cholesky(K)
        Linv = sla.solve_triangular(L, np.eye(n), lower=True)
        Kinv = Linv.T @ Linv
        alpha = Kinv @ self.y[:n]
        loss = nlml(self.y[:n], alpha, np.diag(L))
        dK_l = (-2.0 * v / l) * dist * E * sigmoid(to_unconstrained(l, False))  # gen_tile_grad_l (:133-150)
        dK_v = E * sigmoid(to_unconstrained(v, False))  # gen_tile_grad_v (:115-131)
        g = np.zeros(3)
        g[0] = 0.5 / n * (np.sum(Kinv * dK_l) - alpha @ dK_l @ alpha)
        g[1] = 0.5 / n * (np.sum(Kinv * dK_v) - alpha @ dK_v @ alpha)
        g[2] = sigmoid(to_unconstrained(noise, True)) * 0.5 / n * (np.trace(Kinv) - alpha @ alpha)
        return loss, g

    def optimize_step(self, adam: "Adam", iter_: int) -> float:
        """cpu::optimize_step (core/src/cpu/gp_functions.cpp:1032-1269):
        gradients at the pre-step theta, then Adam per trainable parameter in
        the order l, v, noise (tiled_algorithms.cpp:428-447)."""
        loss, g = self.gradient()
        for p in range(3):
            if not self.trainable[p]:
                continue
            self.m_T[p] = adam.beta1 * self.m_T[p] + (1.0 - adam.beta1) * g[p]
            self.w_T[p] = adam.beta2 * self.w_T[p] + (1.0 - adam.beta2) * g[p] * g[p]
            jitter = p == 2
            u = to_unconstrained(self.hyper[p], jitter)
            u = adam_step(u, adam, self.m_T[p], self.w_T[p], iter_)
            self.hyper[p] = to_constrained(u, jitter)
        return loss

    def optimize(self, adam: "Adam") -> List[float]:
        """cpu::optimize (core/src/cpu/gp_functions.cpp:784-1029)."""
        return [self.optimize_step(adam, it) for it in range(adam.opt_iter)]


class Adam:
    """gprat_hyper::AdamParams (core/include/gp_hyperparameters.hpp:12-56)."""

    def __init__(self, learning_rate=0.001, beta1=0.9, beta2=0.999, epsilon=1e-8, opt_iter=0):
        self.learning_rate, self.beta1, self.beta2, self.epsilon, self.opt_iter = (
            learning_rate, beta1, beta2, epsilon, opt_iter)


def nlml(y, alpha, diagL) -> float:
    """compute_loss + add_losses (core/src/cpu/gp_optimizer.cpp:187-218)."""
    n = y.size
    s = float(y @ alpha) + float(np.sum(np.log(diagL * diagL)))
    return 0.5 * (s + n * LOG_2PI) / n


def to_constrained(p: float, noise: bool) -> float:
    """softplus (+1e-6 for the noise) (core/src/cpu/gp_optimizer.cpp:12-22)."""
    return math.log(1.0 + math.exp(p)) + (1e-6 if noise else 0.0)


def to_unconstrained(p: float, noise: bool) -> float:
    """inverse softplus (core/src/cpu/gp_optimizer.cpp:24-34)."""
    return math.log(math.exp(p - 1e-6) - 1.0) if noise else math.log(math.exp(p) - 1.0)


def sigmoid(p: float) -> float:
    """core/src/cpu/gp_optimizer.cpp:36."""
    return 1.0 / (1.0 + math.exp(-p))


def adam_step(u: float, adam: Adam, m: float, w: float, iter_: int) -> float:
    """Bias-corrected step (core/src/cpu/gp_optimizer.cpp:164-183)."""
    b1t = adam.beta1 ** float(iter_ + 1)
    b2t = adam.beta2 ** float(iter_ + 1)
    nu = adam.learning_rate * math.sqrt(1.0 - b2t) / (1.0 - b1t)
    return u - nu * m / (math.sqrt(w) + adam.epsilon)


# --------------------------------------------------------------------------
# Synthetic workload generator (the benchmark configurations' generator)
def synthetic(n_train: int, n_test: int, n_reg: int, seeds=(0, 1, 2)):
    """x ~ N(0,1) series of length n+d (train seed 0, test seed 1), targets
    y_i = sum_j sin(X_ij)/8 + N(0, 0.01^2) (noise seed 2)."""
    rng_tr, rng_te, rng_no = (np.random.default_rng(s) for s in seeds)
    x_train = rng_tr.standard_normal(n_train + n_reg)
    x_test = rng_te.standard_normal(n_test + n_reg)
    X = feature_matrix(x_train, n_train, n_reg)
    y = np.sin(X).sum(axis=1) / 8.0 + rng_no.normal(0.0, 0.01, n_train)
    return x_train, y, x_test
