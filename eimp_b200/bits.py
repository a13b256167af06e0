"""Bit-packing helpers for the EagleImp data layouts.

EagleImp stores every bit vector in 64-bit words, least significant bit first,
padded to whole 512-bit units (``UNITWORDS = 8`` words, Datatypes.h:70).  The
genotype vectors interleave two words per 64 sites: ``is0`` then ``is2``; a
missing genotype sets both bits (Datatypes.cpp:27-95).
"""
from __future__ import annotations

import numpy as np

UNITWORDS = 8


def W(nbits: int) -> int:
    """Number of uint64 words of a bit vector of ``nbits`` padded to 512 bits."""
    return ((int(nbits) + 511) // 512) * UNITWORDS


def pack_rows(bits: np.ndarray, nwords: int | None = None) -> np.ndarray:
    """Pack a (rows, n) array of 0/1 into (rows, nwords) uint64, LSB first."""
    bits = np.ascontiguousarray(bits, dtype=np.uint8)
    if bits.ndim == 1:
        return pack_rows(bits[None, :], nwords)[0]
    rows, n = bits.shape
    if nwords is None:
        nwords = W(n)
    nbytes = nwords * 8
    packed = np.packbits(bits, axis=1, bitorder="little")
    out = np.zeros((rows, nbytes), dtype=np.uint8)
    out[:, : packed.shape[1]] = packed
    return out.view("<u8").reshape(rows, nwords)


def unpack_rows(words: np.ndarray, n: int) -> np.ndarray:
    """Inverse of :func:`pack_rows`: (rows, nwords) uint64 -> (rows, n) uint8."""
    words = np.ascontiguousarray(words, dtype="<u8")
    if words.ndim == 1:
        return unpack_rows(words[None, :], n)[0]
    b = words.view(np.uint8)
    return np.unpackbits(b, axis=1, bitorder="little", count=n)


_T64_MASKS = {j: np.uint64(sum(1 << b for b in range(64) if not b & j)) for j in (32, 16, 8, 4, 2, 1)}


def _transpose64_inplace(a: np.ndarray) -> None:
    """Transpose the 64 x 64 bit blocks along the last axis of ``a`` (uint64,
    last axis 64 rows, bit c of row r is element (r, c)) in place: row c of
    the result holds bit r of every input row r.  Six butterfly stages; at
    stage j the bits (k, c + j) and (k + j, c) with k & j == c & j == 0 trade
    places."""
    lead = a.shape[:-1]
    for j in (32, 16, 8, 4, 2, 1):
        v = a.reshape(*lead, 64 // (2 * j), 2, j)
        lo, hi = v[..., 0, :], v[..., 1, :]
        t = ((lo >> np.uint64(j)) ^ hi) & _T64_MASKS[j]
        lo ^= t << np.uint64(j)
        hi ^= t


def transpose_bits(words: np.ndarray, nrows: int, ncols: int, out_words: int | None = None,
                   chunk_words: int = 256) -> np.ndarray:
    """Transpose a packed (nrows x ncols bits) matrix into (ncols x nrows bits).

    ``words`` is (>= nrows, >= ceil(ncols/64)) uint64, LSB first; the result is
    (ncols, out_words) uint64 with ``out_words`` defaulting to W(nrows).  Works
    on 64 x 64 bit blocks, ``chunk_words`` source words at a time."""
    words = np.asarray(words, dtype=np.uint64)
    if out_words is None:
        out_words = W(nrows)
    rb = (nrows + 63) // 64
    cw_total = (ncols + 63) // 64
    assert out_words >= rb
    src = words[:nrows]
    out = np.zeros((cw_total * 64, out_words), dtype=np.uint64)
    for c0 in range(0, cw_total, chunk_words):
        c1 = min(cw_total, c0 + chunk_words)
        blk = np.zeros((rb * 64, c1 - c0), dtype=np.uint64)
        blk[:nrows] = src[:, c0:c1]
        b = np.ascontiguousarray(blk.reshape(rb, 64, c1 - c0).transpose(0, 2, 1))   # (rb, cw, 64 rows)
        _transpose64_inplace(b)                                                     # (rb, cw, 64 cols)
        out[c0 * 64:c1 * 64, :rb] = b.transpose(1, 2, 0).reshape((c1 - c0) * 64, rb)
    return np.ascontiguousarray(out[:ncols])


def gather_bits(words: np.ndarray, cols: np.ndarray) -> np.ndarray:
    """Bits of every row of packed ``words`` at the bit positions ``cols``:
    (rows, len(cols)) uint8."""
    cols = np.asarray(cols, dtype=np.int64)
    w = np.asarray(words, dtype=np.uint64)[:, cols >> 6]
    return ((w >> (cols & 63).astype(np.uint64)) & np.uint64(1)).astype(np.uint8)


def pack_genotypes(gt: np.ndarray) -> np.ndarray:
    """Encode genotypes 0/1/2/3(missing) of shape (ntargets, M) into the
    interleaved ``[is0, is2]`` word layout: (ntargets, 2*W(M)) uint64.

    Follows GenotypeVector::push_back (Datatypes.cpp:27-59): is0 is set for
    HomRef or Miss, is2 for HomAlt or Miss.
    """
    gt = np.asarray(gt, dtype=np.uint8)
    if gt.ndim == 1:
        return pack_genotypes(gt[None, :])[0]
    nt, m = gt.shape
    nw = W(m)
    is0 = pack_rows((gt == 0) | (gt == 3), nw)
    is2 = pack_rows((gt == 2) | (gt == 3), nw)
    out = np.empty((nt, 2 * nw), dtype=np.uint64)
    out[:, 0::2] = is0
    out[:, 1::2] = is2
    return out
