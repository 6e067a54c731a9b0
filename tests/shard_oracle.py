"""Exact CPU backend of paddi_b200.sharded (TEST INFRASTRUCTURE ONLY).

It stands in for the GPU backend in the CPU tests of the sharded driver: the
same three steps of an attempt (phase 1 on a row range, refine on a column
range, selection of the merged candidates), computed exactly in FP64 from the
full pairwise distance matrix of a short series.  Its selection checks that
the merged per-candidate values equal the ones of the whole column range, so
a wrong exchange shows up at once; the discords then follow the oracle's
selection rule (oracle.select).
"""
import numpy as np
import torch

from oracle import oracle as O


def f2ord(v):
    """Order-preserving uint32 image of float32 values (unsigned max = float max)."""
    u = np.asarray(v, np.float32).view(np.uint32).astype(np.int64)
    neg = u >= 2 ** 31
    return np.where(neg, (~u) & 0xFFFFFFFF, u | 0x80000000)


class OracleBackend:
    def __init__(self, series, seed=0):
        self.x = np.ascontiguousarray(series, np.float32)
        self.n = len(self.x)
        self.rng = np.random.default_rng(seed)
        self._m = None

    def _dist(self, m):
        if self._m != m:
            N = self.n - m + 1
            W = np.lib.stride_tricks.sliding_window_view(self.x.astype(np.float64), m)[:N]
            mu = W.mean(axis=1, keepdims=True)
            C0 = W - mu
            nrm = np.sqrt((C0 * C0).sum(axis=1))
            flat = (W == W[:, :1]).all(axis=1)
            Z = np.where(flat[:, None], 0.0, C0 / np.where(nrm > 0, nrm, 1.0)[:, None])
            P = Z @ Z.T
            P[np.ix_(flat, flat)] = 1.0  # two flat windows: distance 0
            D = np.maximum(2.0 * m * (1.0 - P), 0.0)
            i = np.arange(N)
            D[np.abs(i[:, None] - i[None, :]) < m - 1] = np.inf  # trivial matches
            self._m, self._D, self._P = m, D, np.where(np.isfinite(D), P, -np.inf)
        return self._D, self._P

    def phase1(self, m, r2, lo, hi):
        D, _ = self._dist(m)
        alive = np.ones(len(D), np.uint8)
        close = D[lo:hi] < r2
        alive[lo:hi][close.any(axis=1)] = 0   # rows with a neighbour inside r
        alive[close.any(axis=0)] = 0          # and those neighbours (columns)
        return torch.from_numpy(alive)

    def refine(self, m, r2, alive, lo, hi):
        D, P = self._dist(m)
        cand = np.flatnonzero(alive.numpy())
        cand = cand[self.rng.permutation(len(cand))]  # an order of this rank's own
        rho = P[cand][:, lo:hi].max(axis=1, initial=-np.inf)
        pruned = (D[cand][:, lo:hi] < r2).any(axis=1)
        return (torch.from_numpy(cand.astype(np.int32)), torch.from_numpy(f2ord(rho)),
                torch.from_numpy(pruned.astype(np.uint8)))

    def select(self, m, r2, ind, rho, pruned, top_k):
        D, P = self._dist(m)
        ind = ind.numpy().astype(np.int64)
        # the merged values must be those of the whole column range
        want_rho = f2ord(P[ind].max(axis=1, initial=-np.inf))
        want_pr = (D[ind] < r2).any(axis=1).astype(np.uint8)
        assert np.array_equal(rho.numpy(), want_rho), "merged correlation maxima differ"
        assert np.array_equal(pruned.numpy(), want_pr), "merged pruned flags differ"
        prof = np.full(len(D), -1.0)
        live = ind[want_pr == 0]
        prof[live] = D[live].min(axis=1)
        att, sel = O.select(prof, m, r2, top_k)
        return sel, {"m": m, "r2": r2, "n_cand": att["n_cand"], "n_disc": att["n_disc"],
                     "found": int(len(sel) >= top_k)}
