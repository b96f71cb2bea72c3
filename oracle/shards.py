"""Oracle (test infrastructure only): the shards of kyto's tiled layers, restated.

The checker for the library's shard decoder (``kg_shard_read`` / ``kg_chunk_read``);
nothing on the product path imports this file.

kyto stores a layer's ``indptr``, ``indices`` and ``data`` with Zarr v3's
``sharding_indexed`` codec (docs/format.md §4.4): a shard is its inner chunks, each the
chunk's elements little-endian compressed by zstd, back to back, followed by the shard
index. The index holds one (offset, nbytes) pair of little-endian u64 per inner chunk (in
chunk order; 2^64 - 1 twice for a chunk that is not stored, which reads as the fill value
0), then the CRC-32C of those index bytes (little-endian u32). A writer stores no chunk
whose elements all equal the fill value (format.md §4.4). ``tile_offsets`` is not sharded:
each of its chunks is one zstd frame ([bytes(little), zstd]). kyto reads these through a
third-party Zarr crate (zarrs, not vendored); this file restates the published layout,
and zstd comes from pyarrow's codec.

CRC-32C is the Castagnoli CRC (reflected polynomial 0x82F63B78, initial and final XOR
0xFFFFFFFF; check value 0xE3069283 for b"123456789").
"""

from __future__ import annotations

import numpy as np

MISSING = 0xFFFFFFFFFFFFFFFF


def _crc32c_table() -> list[int]:
    table = []
    for i in range(256):
        c = i
        for _ in range(8):
            c = (c >> 1) ^ 0x82F63B78 if c & 1 else c >> 1
        table.append(c)
    return table


_TABLE = _crc32c_table()


def crc32c(data: bytes) -> int:
    c = 0xFFFFFFFF
    for byte in data:
        c = _TABLE[(c ^ byte) & 0xFF] ^ (c >> 8)
    return c ^ 0xFFFFFFFF


def _zstd(raw: bytes) -> bytes:
    import pyarrow as pa

    return pa.compress(raw, codec="zstd", asbytes=True)


def write_shards(values: np.ndarray, chunk_elems: int, shard_elems: int) -> list[bytes]:
    """A 1-D array as Zarr v3 shards of ``shard_elems`` elements in inner chunks of
    ``chunk_elems`` (the last shard and chunk padded with the fill value 0, as Zarr's
    regular grid has them)."""
    assert shard_elems % chunk_elems == 0
    values = np.ascontiguousarray(values)
    n = len(values)
    per_shard = shard_elems // chunk_elems
    shards = []
    for s0 in range(0, max(n, 1), shard_elems):
        body, index = bytearray(), []
        for c in range(per_shard):
            a = s0 + c * chunk_elems
            chunk = np.zeros(chunk_elems, dtype=values.dtype)
            part = values[a:min(a + chunk_elems, n)] if a < n else values[:0]
            chunk[:len(part)] = part
            if not chunk.any():
                index.append((MISSING, MISSING))
                continue
            frame = _zstd(chunk.astype(chunk.dtype.newbyteorder("<")).tobytes())
            index.append((len(body), len(frame)))
            body += frame
        ib = np.array(index, dtype="<u8").tobytes()
        shards.append(bytes(body) + ib + crc32c(ib).to_bytes(4, "little"))
    return shards


def write_chunk(values: np.ndarray) -> bytes:
    """One unsharded chunk ([bytes(little), zstd]): tile_offsets' encoding."""
    v = np.ascontiguousarray(values)
    return _zstd(v.astype(v.dtype.newbyteorder("<")).tobytes())


def read_range(shards: list[bytes], chunk_elems: int, shard_elems: int, first: int,
               count: int, dtype) -> np.ndarray:
    """Elements [first, first + count) of the array ``write_shards`` wrote."""
    import pyarrow as pa

    dtype = np.dtype(dtype)
    per_shard = shard_elems // chunk_elems
    out = np.zeros(count, dtype=dtype)
    for i in range(count):
        e = first + i
        s, r = divmod(e, shard_elems)
        c, k = divmod(r, chunk_elems)
        shard = shards[s]
        ib = shard[len(shard) - 16 * per_shard - 4:len(shard) - 4]
        off, nb = np.frombuffer(ib, dtype="<u8")[2 * c:2 * c + 2]
        if off == MISSING:
            continue
        raw = pa.decompress(shard[off:off + nb], decompressed_size=chunk_elems * dtype.itemsize,
                            codec="zstd", asbytes=True)
        out[i] = np.frombuffer(raw, dtype=dtype.newbyteorder("<"))[k]
    return out
