"""A numpy stand-in for one rank's column shard (test infrastructure).

Same step interface as ``nmf_rs.shard.DeviceShard`` (step / status / result,
``reduce_buffer`` and ``objective`` tensors for the collective), so the gloo
tests drive ``nmf_rs.shard.run_shard`` -- the product's host logic -- on CPU
ranks.  The arithmetic restates the reference's updates (lib.rs:74-322,
582-635, 808-824, 1336-1470) with the W update's sums split by columns.
"""
from __future__ import annotations

import numpy as np
import torch

HALF_STEP, W_UPDATE, OBJECTIVE, STOP = 0, 1, 2, 3
DBL_EPS = float(np.finfo(np.float64).eps)


def _hals_h(H, wtv, wtw, lam, gam, reg, eps):
    r = H.shape[0]
    for k in range(r):
        s = wtv[k] - lam if reg else wtv[k].copy()
        for j in range(r):
            if j != k:
                s = s - wtw[k, j] * H[j]
        d = max(wtw[k, k] + gam, eps) if reg else max(wtw[k, k], eps)
        val = s / d
        H[k] = np.where(val > eps, val, eps)


def _hals_w(W, vht, hht, lam, gam, reg, eps):
    r = W.shape[1]
    for k in range(r):
        s = vht[:, k] - lam if reg else vht[:, k].copy()
        for j in range(r):
            if j != k:
                s = s - hht[k, j] * W[:, j]
        d = max(hht[k, k] + gam, eps) if reg else max(hht[k, k], eps)
        val = s / d
        W[:, k] = np.where(val > eps, val, eps)


class NumpyShard:
    def __init__(self, V_local, W0, H0_local, method, *, eps=1e-9, rescale=True, sparsity=0.01,
                 max_iter=100, stop="max_iter", stationary_th=DBL_EPS, check_interval=50,
                 check_niter=10):
        self.V = np.ascontiguousarray(V_local, dtype=np.float64)
        self.W = np.array(W0, dtype=np.float64)
        self.H = np.array(H0_local, dtype=np.float64)
        self.n, self.p = self.V.shape
        self.r = self.W.shape[1]
        self.method = method
        self.eps = eps
        self.rescale = rescale
        self.lam = sparsity if method == "dnmf" else 0.0
        self.max_iter = max_iter
        self.stat = stop == "stationary"
        self.th, self.ci, self.cn = stationary_th, check_interval, check_niter
        n, r = self.n, self.r
        self.reduce_buffer = torch.zeros(n * r + r * r + r, dtype=torch.float64)
        self.objective = torch.zeros(1, dtype=torch.float64)
        self.it = 0
        self.dev = []
        self.stopped = False
        self.n_iter_stop = None
        self.last_max, self.last_min, self.n_collected = -np.inf, np.inf, 0

    # -- the halves of an iteration ------------------------------------------
    def _unpack(self):
        n, r = self.n, self.r
        b = self.reduce_buffer.numpy()
        return b[: n * r].reshape(n, r), b[n * r: n * r + r * r].reshape(r, r), b[n * r + r * r:]

    def step(self, phase):
        if self.stopped:
            return
        V, W, H, eps = self.V, self.W, self.H, self.eps
        if phase == HALF_STEP:
            if self.method == "brunet":
                wh = W @ H
                q = np.where(wh != 0, V / np.where(wh != 0, wh, 1.0), 0.0)
                self.H = H = H * (W.T @ q) / W.sum(0)[:, None]
                wh = W @ H
                q = np.where(wh != 0, V / np.where(wh != 0, wh, 1.0), 0.0)
                num = q @ H.T
            elif self.method == "lee":
                temp = H * (W.T @ V)
                self.H = H = np.where(temp > eps, temp, eps) / ((W.T @ W) @ H + eps)
                num = V @ H.T
            else:
                reg = self.method == "dnmf"
                _hals_h(H, W.T @ V, W.T @ W, self.lam, 0.0, reg, eps)
                num = V @ H.T
            b = self.reduce_buffer.numpy()
            n, r = self.n, self.r
            b[: n * r] = num.ravel()
            b[n * r: n * r + r * r] = (H @ H.T).ravel()
            b[n * r + r * r:] = H.sum(1)
        elif phase == W_UPDATE:
            num, G, sums = self._unpack()
            itn = self.it + 1
            if self.method == "brunet":
                W *= num / sums[None, :]
                if itn % 10 == 0:
                    np.maximum(W, DBL_EPS, out=W)
                    np.maximum(H, DBL_EPS, out=H)
            elif self.method == "lee":
                temp = W * num
                self.W = W = np.where(temp < eps, eps, temp) / (W @ G + eps)
                if self.rescale:
                    s = W.sum(0)
                    W /= np.where(s > 0, s, 1.0)[None, :]
            else:
                reg = self.method == "dnmf"
                _hals_w(W, num, G, self.lam, 0.0, reg, eps)
                if reg:
                    nw = np.sqrt((W * W).sum(0))
                    nh = np.sqrt(np.diag(G))
                    d = nw * nh
                    W /= np.where(nw > 0, nw, 1.0)[None, :]
                    H /= np.where(nh > 0, nh, 1.0)[:, None]
                    H *= d[:, None]
            self.it = itn
        elif phase == OBJECTIVE:
            wh = self.W @ self.H
            if self.method == "brunet":
                pos = V > 0
                good = pos & (wh > 0)
                t = np.where(good, V * np.log(np.where(good, V / np.where(good, wh, 1), 1)) - V + wh, 0.0)
                t = np.where(pos, t, wh)
                self.objective[0] = float(t.sum())
            else:
                self.objective[0] = 0.5 * float(((V - wh) ** 2).sum())
        elif phase == STOP:
            self._stop(float(self.objective[0]))

    def _stop(self, d):
        # StationaryStop::should_stop, lib.rs:1378-1400
        i = self.it
        self.dev.append(d)
        stop = False
        if np.isnan(d):
            stop = True
        elif i == 0:
            self.last_max = self.last_min = d
            self.n_collected = 1
        else:
            sample = not (self.n_collected == 0 and i % self.ci != 0)
            if sample:
                self.last_max = max(self.last_max, d)
                self.last_min = min(self.last_min, d)
                self.n_collected += 1
                if self.n_collected == self.cn + 1:
                    if abs(self.last_max - self.last_min) / self.cn <= self.th:
                        stop = True
                    else:
                        self.last_max, self.last_min, self.n_collected = -np.inf, np.inf, 0
        if stop:
            self.stopped = True
            self.n_iter_stop = i

    def status(self):
        return (self.n_iter_stop if self.stopped else self.it), self.stopped

    def result(self):
        return self.W, self.H, np.array(self.dev)
