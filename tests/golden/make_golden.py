"""Write the golden fixtures the parity tests read (run once, in a container that has
the kyto source tree; the outputs are committed so the tests never read that tree).

What it writes (all small ``.npz`` files beside this script):

- ``synthetic_counts.npz``: kyto's ``synthetic`` test input (500 cells x 400 genes,
  30,277 stored counts), rebuilt by importing kyto's own generator
  ``tests/fixtures/synthetic.py`` (``make_synthetic``; its digest is checked against
  ``tests/fixtures/registry.py``'s expected digest).
- ``synthetic_{normalize_log1p,hvg,pca,neighbors}.npz``: the arrays of kyto's checked-in
  scanpy references ``tests/fixtures/reference/synthetic/*.npz`` that pin this path
  (normalize_total(1e4) + log1p values, seurat HVG statistics for n_top_genes=100, PCA
  with 20 components on those HVGs, exact 15-NN distance graph on that PCA embedding).
- ``pbmc3k_neighbors.npz``: scanpy's pbmc3k ``X_pca`` (2,700 x 50) and its exact 15-NN
  distance graph (``tests/fixtures/reference/pbmc3k/{pca,neighbors}.npz``); pbmc3k's
  raw counts are a download and are not needed for the kNN fixture.
- ``{synthetic,pbmc3k}_connectivities.npz``: scanpy's distance graph and its UMAP
  ``connectivities`` (the same ``neighbors.npz`` files).

Usage: ``python tests/golden/make_golden.py /path/to/kyto``
"""

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def main(kyto: Path) -> None:
    fixtures = kyto / "tests"
    sys.path.insert(0, str(fixtures))
    from fixtures.registry import EXPECTED_DIGESTS  # noqa: PLC0415
    from fixtures.synthetic import make_synthetic  # noqa: PLC0415

    data = make_synthetic()
    assert data.digest() == EXPECTED_DIGESTS["synthetic"], "synthetic digest changed"
    counts = np.asarray(data.data)
    assert np.all(counts == np.round(counts)) and counts.min() > 0
    np.savez_compressed(
        HERE / "synthetic_counts.npz",
        indptr=np.asarray(data.indptr, dtype=np.uint64),
        indices=np.asarray(data.indices, dtype=np.uint32),
        counts=counts.astype(np.uint32),
        n_genes=np.array([data.n_genes], dtype=np.uint64),
        gene_id=np.asarray(data.genes["gene_id"]),
    )

    ref = kyto / "tests" / "fixtures" / "reference"

    def load(name: str) -> dict:
        with np.load(ref / f"{name}.npz", allow_pickle=False) as z:
            return {key: z[key] for key in z.files}

    norm = load("synthetic/normalize_log1p")
    np.savez_compressed(
        HERE / "synthetic_normalize_log1p.npz",
        indptr=norm["target/normalized/indptr"],
        indices=norm["target/normalized/indices"],
        normalized=norm["target/normalized/data"],
        log1p=norm["target/log1p/data"],
    )
    hvg = load("synthetic/hvg")
    np.savez_compressed(
        HERE / "synthetic_hvg.npz",
        gene_id=hvg["genes/gene_id"],
        means=hvg["seurat/means"],
        dispersions=hvg["seurat/dispersions"],
        dispersions_norm=hvg["seurat/dispersions_norm"],
        highly_variable=hvg["seurat/highly_variable"],
    )
    pca = load("synthetic/pca")
    np.savez_compressed(
        HERE / "synthetic_pca.npz",
        gene_id=pca["genes/gene_id"],
        embedding=pca["embedding"],
        components=pca["components"],
        variance=pca["variance"],
        variance_ratio=pca["variance_ratio"],
    )
    nn = load("synthetic/neighbors")
    np.savez_compressed(
        HERE / "synthetic_neighbors.npz",
        indptr=nn["distances/indptr"],
        indices=nn["distances/indices"],
        distances=nn["distances/data"],
    )
    ppca = load("pbmc3k/pca")
    pnn = load("pbmc3k/neighbors")
    np.savez_compressed(
        HERE / "pbmc3k_neighbors.npz",
        embedding=ppca["embedding"],
        indptr=pnn["distances/indptr"],
        indices=pnn["distances/indices"],
        distances=pnn["distances/data"],
    )
    # scanpy's UMAP connectivities of those distance graphs (float64 distances in, the
    # float32 fuzzy-union weights out).
    for name, graph in (("synthetic", nn), ("pbmc3k", pnn)):
        np.savez_compressed(
            HERE / f"{name}_connectivities.npz",
            dist_indptr=graph["distances/indptr"],
            dist_indices=graph["distances/indices"],
            dist_data=graph["distances/data"],
            indptr=graph["connectivities/indptr"],
            indices=graph["connectivities/indices"],
            weights=graph["connectivities/data"],
        )


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/kyto")
    main(Path(sys.argv[1]))
