"""IVF-PQ index on seeded synthetic data, and the plaintext ADC search.

Restates, for data generation and result checking only (the offline training
is outside the accelerated path):
  * k-means (software_golden_model/ivf_quantizer.py:19-82): random-choice
    initialisation from a seed, Lloyd iterations, empty clusters reseeded;
  * residual product quantisation (product_quantizer.py:26-113): per-subspace
    k-means on x - centroid(x);
  * PQ encoding (encoder.py:20-76) and the candidate reconstruction the
    encrypted chain packs, centroid + codebook entry
    (integration_tools/generate_interactive_test_vectors.cpp:489-501);
  * plaintext ADC search (software_golden_model/fhe_core/plaintext_searcher.cpp:100-213):
    coarse distances, nprobe nearest lists, exact distances to reconstructions, top-k.
The synthetic set stands in for SIFT-small, which is absent.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np


def gaussian_mixture(n: int, d: int, components: int, sigma: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    centers = rng.normal(0.0, 1.0, (components, d))
    lab = rng.integers(0, components, n)
    return (centers[lab] + rng.normal(0.0, sigma, (n, d))).astype(np.float32)


def kmeans(X: np.ndarray, k: int, iters: int, seed: int, tol: float = 1e-5) -> np.ndarray:
    rng = np.random.default_rng(seed)
    X = X.astype(np.float64)
    C = X[rng.choice(len(X), size=k, replace=False)].copy()
    for _ in range(iters):
        d2 = (X * X).sum(1)[:, None] + (C * C).sum(1)[None, :] - 2 * X @ C.T
        lab = np.argmin(d2, axis=1)
        newC = np.zeros_like(C)
        for i in range(k):
            m = lab == i
            newC[i] = X[m].mean(0) if m.any() else X[rng.integers(len(X))]
        done = np.allclose(C, newC, atol=tol)
        C = newC
        if done:
            break
    return C.astype(np.float32)


def assign(X: np.ndarray, C: np.ndarray) -> np.ndarray:
    X = X.astype(np.float64)
    C = C.astype(np.float64)
    d2 = (X * X).sum(1)[:, None] + (C * C).sum(1)[None, :] - 2 * X @ C.T
    return np.argmin(d2, axis=1).astype(np.int32)


@dataclass
class IvfPqIndex:
    centroids: np.ndarray        # n_list x d
    codebooks: np.ndarray        # M x K x sub_dim
    assignments: np.ndarray      # n
    codes: np.ndarray            # n x M (uint8)
    lists: list                  # vector ids per list

    @property
    def d(self) -> int:
        return self.centroids.shape[1]

    @property
    def n_list(self) -> int:
        return self.centroids.shape[0]

    def reconstruct(self, vids) -> np.ndarray:
        vids = np.asarray(vids)
        M, K, sd = self.codebooks.shape
        rec = self.centroids[self.assignments[vids]].astype(np.float64).copy()
        for m in range(M):
            rec[:, m * sd:(m + 1) * sd] += self.codebooks[m][self.codes[vids, m]]
        return rec

    @classmethod
    def train(cls, X: np.ndarray, n_list: int, M: int, K: int, seed: int, iters: int = 25) -> "IvfPqIndex":
        C = kmeans(X, n_list, iters, seed)
        lab = assign(X, C)
        R = X - C[lab]
        d = X.shape[1]
        sd = d // M
        books = np.zeros((M, K, sd), dtype=np.float32)
        codes = np.zeros((len(X), M), dtype=np.uint8)
        for m in range(M):
            sub = R[:, m * sd:(m + 1) * sd]
            books[m] = kmeans(sub, K, iters, seed + 1 + m)
            codes[:, m] = assign(sub, books[m])
        lists = [np.nonzero(lab == c)[0].tolist() for c in range(n_list)]
        return cls(C, books, lab, codes, lists)


def plaintext_coarse(index: IvfPqIndex, q: np.ndarray) -> np.ndarray:
    c = index.centroids.astype(np.float64)
    return ((q[None, :].astype(np.float64) - c) ** 2).sum(1)


def plaintext_search(index: IvfPqIndex, q: np.ndarray, nprobe: int, top_k: int):
    """(probed lists, candidate ids, candidate distances, top-k ids)."""
    coarse = plaintext_coarse(index, q)
    probes = np.argsort(coarse, kind="stable")[:nprobe]
    cand = [v for c in probes for v in index.lists[c]]
    rec = index.reconstruct(cand)
    dist = ((q[None, :].astype(np.float64) - rec) ** 2).sum(1)
    order = np.argsort(dist, kind="stable")[:top_k]
    return probes, np.array(cand), dist, np.array(cand)[order]
