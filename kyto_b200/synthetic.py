"""Seeded synthetic single-cell inputs with the shapes of the benchmark workloads.

No dataset is downloaded: counts are drawn as kyto's benchmark describes them
(per-gene negative binomial with log-normal gene means, cell-type shifts planted on
some genes), on the device when torch has CUDA (fast at 1M cells) or on the CPU.

- ``counts_csr``: cells x genes u32 counts (CSR, genes ascending per cell).
- ``log1p_csr``: the same after normalize_total(1e4) + log1p, as f32 values.
- ``gaussian_mixture``: dense f32 points from an isotropic Gaussian mixture.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class Csr:
    indptr: np.ndarray  # u64, n_cells + 1
    indices: np.ndarray  # u32
    values: np.ndarray  # u32 counts or f32 values
    n_genes: int
    cell_type: np.ndarray | None = None

    @property
    def n_cells(self) -> int:
        return len(self.indptr) - 1

    @property
    def nnz(self) -> int:
        return int(self.indptr[-1])


def _nb_density(means: np.ndarray, dispersion: float) -> float:
    """Expected fraction of nonzero NB(mean, dispersion) draws over the given means."""
    r = 1.0 / dispersion
    return float(np.mean(1.0 - (1.0 + means * dispersion) ** (-r)))


def _calibrate_scale(means: np.ndarray, dispersion: float, density: float) -> float:
    lo, hi = 1e-6, 1e6
    for _ in range(80):
        mid = math.sqrt(lo * hi)
        if _nb_density(means * mid, dispersion) < density:
            lo = mid
        else:
            hi = mid
    return math.sqrt(lo * hi)


def counts_csr(n_cells: int, n_genes: int, nnz_per_cell: float, n_types: int,
               shifted_genes: int, mu: float = 0.0, sigma: float = 1.5,
               dispersion: float = 0.3, seed: int = 0, device: str | None = None,
               chunk_cells: int = 65536) -> Csr:
    """Cells x genes u32 counts: gene means LogNormal(mu, sigma) scaled so that about
    ``nnz_per_cell`` genes per cell are nonzero, ``n_types`` cell types each shifting
    ``shifted_genes`` genes by a factor in [2, 8], per-cell size LogNormal(0, 0.3),
    counts Gamma-Poisson (negative binomial with the given dispersion)."""
    dev = device or ("cuda" if torch.cuda.is_available() else "cpu")
    rng = np.random.default_rng(seed)
    gene_mean = np.exp(rng.normal(mu, sigma, n_genes))
    shift = np.ones((n_types, n_genes))
    for t in range(n_types):
        genes = rng.choice(n_genes, size=min(shifted_genes, n_genes), replace=False)
        shift[t, genes] = rng.uniform(2.0, 8.0, size=len(genes))
    cell_type = rng.integers(0, n_types, n_cells)
    size = np.exp(rng.normal(0.0, 0.3, n_cells))
    scale = _calibrate_scale(gene_mean, dispersion, nnz_per_cell / n_genes)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    g_mean = torch.tensor(gene_mean * scale, dtype=torch.float32, device=dev)
    g_shift = torch.tensor(shift, dtype=torch.float32, device=dev)
    shape = torch.tensor(1.0 / dispersion, dtype=torch.float32, device=dev)
    indptr = np.zeros(n_cells + 1, dtype=np.uint64)
    idx_parts, val_parts = [], []
    for a in range(0, n_cells, chunk_cells):
        b = min(n_cells, a + chunk_cells)
        ct = torch.tensor(cell_type[a:b], device=dev)
        sz = torch.tensor(size[a:b], dtype=torch.float32, device=dev)
        mean = g_mean[None, :] * g_shift[ct] * sz[:, None]
        # Gamma(shape r, scale mean / r) then Poisson: NB(mean, 1/r).
        lam = torch._standard_gamma(shape.expand_as(mean).contiguous(), generator=gen) * (
            mean / shape)
        counts = torch.poisson(lam, generator=gen).to(torch.int64)
        nz = counts.nonzero(as_tuple=False)
        per_row = torch.bincount(nz[:, 0], minlength=b - a).cpu().numpy().astype(np.uint64)
        indptr[a + 1:b + 1] = per_row
        idx_parts.append(nz[:, 1].to(torch.int32).cpu().numpy().view(np.uint32))
        val_parts.append(counts[nz[:, 0], nz[:, 1]].to(torch.int32).cpu().numpy().view(np.uint32))
        del counts, lam, mean, nz
    np.cumsum(indptr, out=indptr)
    return Csr(indptr, np.concatenate(idx_parts), np.concatenate(val_parts), n_genes,
               cell_type)


def log1p_values(x: Csr, target_sum: float = 1e4) -> np.ndarray:
    """normalize_total(target_sum) + log1p of the counts, f32, as kyto computes them
    (f64 row totals; f32 divisor and division; log1p in f64 rounded to f32)."""
    counts = x.values.astype(np.float64)
    rows = np.repeat(np.arange(x.n_cells), np.diff(x.indptr).astype(np.int64))
    totals = np.bincount(rows, weights=counts, minlength=x.n_cells)
    div = (totals.astype(np.float32) / np.float32(target_sum)).astype(np.float32)
    div[div == 0] = 1.0
    v = x.values.astype(np.float32) / div[rows]
    return np.log1p(v.astype(np.float64)).astype(np.float32)


def log1p_csr(n_cells: int, n_genes: int, nnz_per_cell: float, n_types: int,
              shifted_genes: int, seed: int = 0, **kw) -> Csr:
    x = counts_csr(n_cells, n_genes, nnz_per_cell, n_types, shifted_genes, seed=seed, **kw)
    return Csr(x.indptr, x.indices, log1p_values(x), n_genes, x.cell_type)


def gaussian_mixture(n: int, dim: int = 50, n_components: int = 200, spread: float = 3.0,
                     seed: int = 0, device: str | None = None) -> tuple[np.ndarray, np.ndarray]:
    """n x dim f32 points: component weights Dirichlet(1), means N(0, spread^2) per
    dimension, isotropic sigma log-uniform in [0.2, 2]. Returns (points, labels)."""
    dev = device or ("cuda" if torch.cuda.is_available() else "cpu")
    rng = np.random.default_rng(seed)
    w = rng.dirichlet(np.ones(n_components))
    means = rng.normal(0.0, spread, (n_components, dim)).astype(np.float32)
    sig = np.exp(rng.uniform(math.log(0.2), math.log(2.0), n_components)).astype(np.float32)
    labels = rng.choice(n_components, size=n, p=w)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    lab = torch.tensor(labels, device=dev)
    pts = torch.randn((n, dim), generator=gen, device=dev) * torch.tensor(sig, device=dev)[lab, None]
    pts += torch.tensor(means, device=dev)[lab]
    return pts.float().cpu().numpy(), labels
