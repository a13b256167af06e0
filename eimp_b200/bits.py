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


def transpose_bits(words: np.ndarray, nrows: int, ncols: int, out_words: int | None = None) -> np.ndarray:
    """Transpose a packed (nrows x ncols bits) matrix into (ncols x nrows bits)."""
    dense = unpack_rows(words, ncols)[:nrows]
    return pack_rows(np.ascontiguousarray(dense.T), out_words)


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
