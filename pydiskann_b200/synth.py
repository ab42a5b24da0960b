"""Seeded synthetic workloads with the shapes and value distributions of the
five benchmark configurations (no public dataset is used).

All generators use numpy PCG64 streams keyed by (seed, stream id), so the
same call gives the same bytes on every machine.
  plain:     100k x 128, 64-centre isotropic Gaussian mixture, sigma 20,
             centres U[0,255], rounded and clipped to [0, 255]
  pq:        1M x 128, same recipe with 256 centres
  cosine:    1M x 768, g * sigma_i with sigma_i = (i+1)^-0.25 (variance
             spectrum exponent -0.5), unit normalised, stored as BF16 values
  spfresh:   2M x 96, 1024 centres, Zipf(1.1) component weights, rounded,
             not clipped
  filtered:  1M x 256, 512 centres, clipped; 1-3 labels of 100 per vector
             drawn Zipf(1.0) without replacement, padded with u64::MAX
"""
from __future__ import annotations

import numpy as np

STREAM_CENTERS, STREAM_BASE, STREAM_QUERY, STREAM_LABELS, STREAM_MISC = 0, 1, 2, 3, 4
LABEL_PAD = np.uint64(0xFFFFFFFFFFFFFFFF)


def _rng(seed, stream):
    return np.random.default_rng([seed, stream])


def mixture(n, d, n_centers, seed=0, stream=STREAM_BASE, sigma=20.0, clip=True, zipf=None,
            chunk=131072):
    """Gaussian-mixture rows, rounded to integers (float32)."""
    centers = _rng(seed, STREAM_CENTERS).uniform(0.0, 255.0, size=(n_centers, d))
    rng = _rng(seed, stream)
    if zipf is None:
        w = None
    else:
        w = 1.0 / np.arange(1, n_centers + 1, dtype=np.float64) ** zipf
        w /= w.sum()
    out = np.empty((n, d), dtype=np.float32)
    for s in range(0, n, chunk):
        m = min(chunk, n - s)
        z = rng.integers(0, n_centers, size=m) if w is None else rng.choice(n_centers, size=m, p=w)
        x = centers[z] + rng.normal(0.0, sigma, size=(m, d))
        x = np.rint(x)
        if clip:
            np.clip(x, 0.0, 255.0, out=x)
        out[s:s + m] = x
    return out


def plain(n=100_000, nq=1_000, d=128, seed=0):
    return (mixture(n, d, 64, seed, STREAM_BASE), mixture(nq, d, 64, seed, STREAM_QUERY))


def pq_config(n=1_000_000, nq=10_000, d=128, seed=0):
    return (mixture(n, d, 256, seed, STREAM_BASE), mixture(nq, d, 256, seed, STREAM_QUERY))


def cosine(n=1_000_000, nq=20_000, d=768, seed=0, chunk=65536):
    """Anisotropic power-law embeddings, unit normalised, rounded to BF16."""
    sig = (np.arange(d, dtype=np.float64) + 1.0) ** -0.25

    def gen(m, stream):
        rng = _rng(seed, stream)
        out = np.empty((m, d), dtype=np.float32)
        for s in range(0, m, chunk):
            k = min(chunk, m - s)
            g = rng.standard_normal((k, d)) * sig
            g /= np.linalg.norm(g, axis=1, keepdims=True)
            out[s:s + k] = to_bf16_values(g.astype(np.float32))
        return out

    return gen(n, STREAM_BASE), gen(nq, STREAM_QUERY)


def to_bf16_values(x):
    """Round float32 values to the nearest BF16 (ties to even), kept as float32."""
    u = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).view(np.float32)


def spfresh(n=2_000_000, nq=10_000, d=96, seed=0):
    return (mixture(n, d, 1024, seed, STREAM_BASE, clip=False, zipf=1.1),
            mixture(nq, d, 1024, seed, STREAM_QUERY, clip=False, zipf=1.1))


def filtered(n=1_000_000, nq=10_000, d=256, seed=0, n_labels=100):
    X = mixture(n, d, 512, seed, STREAM_BASE)
    Q = mixture(nq, d, 512, seed, STREAM_QUERY)
    labels = label_sets(n, seed, n_labels)
    return X, Q, labels


def label_sets(n, seed=0, n_labels=100, max_per=3):
    """1..max_per distinct labels in [1, n_labels] per row, Zipf(1.0) weighted,
    stored as max_per u64 fields padded with u64::MAX."""
    rng = _rng(seed, STREAM_LABELS)
    w = 1.0 / np.arange(1, n_labels + 1, dtype=np.float64)
    w /= w.sum()
    cnt = rng.integers(1, max_per + 1, size=n)
    # Gumbel top-k gives weighted sampling without replacement
    keys = np.log(w)[None, :] + rng.gumbel(size=(n, n_labels)) if n * n_labels <= 50_000_000 else None
    out = np.full((n, max_per), LABEL_PAD, dtype=np.uint64)
    if keys is not None:
        top = np.argsort(-keys, axis=1)[:, :max_per] + 1
        for j in range(max_per):
            sel = cnt > j
            out[sel, j] = top[sel, j].astype(np.uint64)
        return out
    step = 200_000
    for s in range(0, n, step):
        m = min(step, n - s)
        k = np.log(w)[None, :] + rng.gumbel(size=(m, n_labels))
        top = np.argsort(-k, axis=1)[:, :max_per] + 1
        for j in range(max_per):
            sel = cnt[s:s + m] > j
            out[s:s + m][sel, j] = top[sel, j].astype(np.uint64)
    return out
