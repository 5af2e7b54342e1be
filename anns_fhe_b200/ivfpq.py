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


def _sqdist_argmin(X: np.ndarray, C: np.ndarray, chunk: int = 65536) -> np.ndarray:
    """argmin_j ||x_i - c_j||^2 in float64, in row chunks (bounded memory)."""
    X = np.asarray(X)
    C = C.astype(np.float64)
    cc = (C * C).sum(1)[None, :]
    out = np.empty(len(X), dtype=np.int64)
    for s in range(0, len(X), chunk):
        x = X[s:s + chunk].astype(np.float64)
        d2 = (x * x).sum(1)[:, None] + cc - 2 * x @ C.T
        out[s:s + chunk] = np.argmin(d2, axis=1)
    return out


def farthest_init(X: np.ndarray, k: int, rng) -> np.ndarray:
    """Farthest-point seeding: a random first centre, then each next centre is
    the point farthest from the centres chosen so far. On a well-separated
    mixture with k components it puts one centre in every component."""
    # float32 on a sample of at most 32 points per centre is plenty to seed
    if len(X) > 32 * k:
        X = X[np.sort(rng.choice(len(X), 32 * k, replace=False))]
    X = X.astype(np.float32)
    C = np.empty((k, X.shape[1]), dtype=np.float32)
    xx = (X * X).sum(1)
    C[0] = X[rng.integers(len(X))]
    d2 = xx + C[0] @ C[0] - 2 * X @ C[0]
    for i in range(1, k):
        C[i] = X[int(np.argmax(d2))]
        d2 = np.minimum(d2, xx + C[i] @ C[i] - 2 * X @ C[i])
    return C.astype(np.float64)


def kmeans(X: np.ndarray, k: int, iters: int, seed: int, tol: float = 1e-5, init: str = "random") -> np.ndarray:
    """Lloyd's k-means: seeded random-choice initialisation (the reference's,
    ivf_quantizer.py:19-82) or farthest-point seeding; empty clusters
    reseeded from a random point."""
    rng = np.random.default_rng(seed)
    X = X.astype(np.float64)
    if init == "farthest":
        C = farthest_init(X, k, rng)
    else:
        C = X[rng.choice(len(X), size=k, replace=False)].copy()
    for _ in range(iters):
        lab = _sqdist_argmin(X, C)
        cnt = np.bincount(lab, minlength=k)
        newC = np.zeros_like(C)
        np.add.at(newC, lab, X) if len(X) < 4096 else _scatter_sum(newC, lab, X)
        for i in np.nonzero(cnt == 0)[0]:
            newC[i] = X[rng.integers(len(X))]
        nz = cnt > 0
        newC[nz] /= cnt[nz, None]
        done = np.allclose(C, newC, atol=tol)
        C = newC
        if done:
            break
    return C.astype(np.float32)


def _scatter_sum(out: np.ndarray, lab: np.ndarray, X: np.ndarray) -> None:
    """out[lab[i]] += X[i], by sorting (faster than np.add.at for large inputs)."""
    order = np.argsort(lab, kind="stable")
    ls = lab[order]
    starts = np.concatenate([[0], np.nonzero(np.diff(ls))[0] + 1])
    sums = np.add.reduceat(X[order], starts, axis=0)
    out[ls[starts]] = sums


def assign(X: np.ndarray, C: np.ndarray) -> np.ndarray:
    return _sqdist_argmin(X, C).astype(np.int32)


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
    def train(cls, X: np.ndarray, n_list: int, M: int, K: int, seed: int, iters: int = 25,
              train_sample: int | None = None, pq_sample: int | None = None,
              init: str = "random") -> "IvfPqIndex":
        """IVF k-means, then residual PQ. With `train_sample` (`pq_sample`),
        the IVF (PQ) k-means run on a seeded sample of that many vectors;
        every vector is then assigned and encoded (training on a sample, as
        large IVF-PQ builds do)."""
        T = X
        if train_sample and train_sample < len(X):
            T = X[np.sort(np.random.default_rng(seed + 99).choice(len(X), train_sample, replace=False))]
        C = kmeans(T, n_list, iters, seed, init=init)
        lab = assign(X, C)
        tlab = lab if T is X else assign(T, C)
        R = X - C[lab]
        RT = R if T is X else T - C[tlab]
        if pq_sample and pq_sample < len(RT):
            RT = RT[np.sort(np.random.default_rng(seed + 98).choice(len(RT), pq_sample, replace=False))]
        d = X.shape[1]
        sd = d // M
        books = np.zeros((M, K, sd), dtype=np.float32)
        codes = np.zeros((len(X), M), dtype=np.uint8)
        for m in range(M):
            books[m] = kmeans(RT[:, m * sd:(m + 1) * sd], K, iters, seed + 1 + m)
            codes[:, m] = assign(R[:, m * sd:(m + 1) * sd], books[m])
        order = np.argsort(lab, kind="stable")
        bounds = np.searchsorted(lab[order], np.arange(n_list + 1))
        lists = [order[bounds[c]:bounds[c + 1]].tolist() for c in range(n_list)]
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
