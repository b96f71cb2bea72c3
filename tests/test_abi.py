"""The C ABI library loads and exports every entry point include/kyto_gpu.h declares
(no compute call: this runs without a GPU)."""

import ctypes
import re
from pathlib import Path

import pytest

import kyto_b200 as K

ROOT = Path(__file__).resolve().parents[1]


def declared_symbols() -> set[str]:
    text = (ROOT / "include" / "kyto_gpu.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return set(re.findall(r"\b(kg_[a-z0-9_]+)\s*\(", text))


def test_header_declares_the_mirror_exports():
    assert declared_symbols() == set(K.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = K.library()
    for name in declared_symbols():
        assert hasattr(lib, name), name
        assert ctypes.cast(getattr(lib, name), ctypes.c_void_p).value


def test_library_exports_nothing_but_the_abi():
    import subprocess

    out = subprocess.run(["nm", "-D", "--defined-only", str(K.LIB_PATH)],
                         capture_output=True, text=True, check=True).stdout
    exported = {line.split()[-1] for line in out.splitlines() if " T " in line}
    assert {s for s in exported if s.startswith("kg_")} == declared_symbols()


def test_status_codes_map_to_kyto_codes():
    assert K.KYTO_CODE[K.KG_ERR_INVALID] == "KY-E215"
    assert K.KYTO_CODE[K.KG_CANCELLED] == "KY-E503"
    assert K.KYTO_CODE[K.KG_ERR_DEVICE] == "KY-E505"


def test_seurat_flags_on_host_match_the_oracle():
    # kg_hvg_seurat is host arithmetic: check it against the oracle on kyto's golden
    # moments without a GPU.
    import numpy as np

    from oracle import oracle as O
    from tests.conftest import load_golden

    g = load_golden("synthetic_counts")
    x = O.normalize_log1p(O.Csr(g["indptr"], g["indices"], g["counts"], int(g["n_genes"][0])))
    sums, squares, positives = O.hvg_moments(x)
    n_genes = x.n_genes
    means, disp, norm = np.empty(n_genes), np.empty(n_genes), np.empty(n_genes)
    flags = np.empty(n_genes, dtype=np.uint8)
    P = K._ptr
    assert K.library().kg_hvg_seurat(P(sums), P(squares), P(positives), x.n_rows, n_genes, 100,
                                     P(means), P(disp), P(norm), P(flags)) == 0
    om, od, on, of = O.hvg_seurat(sums, squares, positives, x.n_rows, 100)
    assert np.array_equal(flags.astype(bool), of)
    assert np.array_equal(flags.astype(bool), load_golden("synthetic_hvg")["highly_variable"])
    np.testing.assert_allclose(means, om, rtol=1e-15)
    fin = np.isfinite(on)
    np.testing.assert_allclose(norm[fin], on[fin], rtol=1e-12)
