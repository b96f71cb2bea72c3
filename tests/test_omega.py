"""Omega, the PCA's random sketch (kyto's omega_row, crates/kyto-exec/src/pca.rs:936-950):
the oracle's C restatement against the same SplitMix64 steps in Python integers (CPU),
and the device generator (kg_diag_omega, the generator every PCA kernel draws from)
against the oracle, bit for bit."""

import numpy as np
import pytest

from oracle import oracle as O

CELLS = np.array([0, 1, 2, 17, 4095, 65_536, 999_999, 2**32 + 5, 2**40 + 12345, 2**63 - 1],
                 dtype=np.uint64)


@pytest.mark.parametrize("seed", [0, 1, 42, 2**63 + 7])
def test_oracle_omega_is_kytos_stream(seed):
    got = O.omega_rows(seed, CELLS, 60)
    for i, cell in enumerate(CELLS):
        want = np.array(O.omega_row_reference(seed, int(cell), 60))
        assert np.array_equal(got[i].view(np.uint64), want.view(np.uint64))
    assert np.all(got >= -1.0) and np.all(got < 1.0)


@pytest.mark.gpu
@pytest.mark.parametrize("seed", [0, 1, 42, 2**63 + 7])
def test_device_omega_bits_equal_the_oracle(seed):
    import kyto_b200 as K

    rng = np.random.default_rng(seed % 1000)
    cells = np.concatenate([CELLS, rng.integers(0, 2**62, 5000, dtype=np.uint64),
                            np.arange(3000, dtype=np.uint64)])
    for width in (1, 7, 60, 64):
        dev = K.omega(seed, cells, width)
        ref = O.omega_rows(seed, cells, width)
        assert np.array_equal(dev.view(np.uint64), ref.view(np.uint64)), width
