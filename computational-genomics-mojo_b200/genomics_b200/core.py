"""2-bit DNA packing and SequenceBatch, mirroring genomics/core/dna.mojo and
genomics/core/sequence.mojo of the reference.

Encoding (dna.mojo:12-22): A=0 C=1 G=2 T=3, 32 bases per uint64, MSB-first
(base i of a word sits at bits 62-2i .. 63-2i).  Any other character is
stored as A and flagged in a parallel NMask word, bit i = position i,
LSB-first (dna.mojo:107-141; sequence.mojo:53-57).

SequenceBatch is a structure of arrays (sequence.mojo:23-36): packed words,
NMask words, per-sequence word offsets (int64, like Mojo's Int) and lengths.
Arrays are numpy; `pinned=True` places them in page-locked host memory so the
end-to-end entry points copy them by DMA.
"""
from __future__ import annotations

import ctypes

import numpy as np

BASE_BITS = 2
BASES_PER_WORD = 32


class Base:
    """2-bit codes (dna.mojo:12-22)."""
    A = 0
    C = 1
    G = 2
    T = 3
    N = 0xFF


_LUT = np.full(256, 4, np.uint8)
for _c, _v in ((b"A", 0), (b"C", 1), (b"G", 2), (b"T", 3), (b"a", 0), (b"c", 1), (b"g", 2),
               (b"t", 3)):
    _LUT[_c[0]] = _v


def ascii_to_2bit(c: int) -> int:
    """dna.mojo:25-40: ACGT/acgt -> 0..3, anything else Base.N."""
    v = int(_LUT[c & 0xFF])
    return Base.N if v == 4 else v


def base_to_ascii(b: int) -> int:
    """dna.mojo:43-52."""
    return (65, 67, 71, 84)[b] if 0 <= b <= 2 else 84


def get_base_from_word(word: int, pos: int) -> int:
    """dna.mojo:96-100: base at position pos (0 = leftmost)."""
    return (int(word) >> (62 - pos * BASE_BITS)) & 3


class NMask:
    """One N bit per position of a packed word (dna.mojo:107-141)."""

    def __init__(self, data: int = 0):
        self.data = int(data)

    def is_n(self, pos: int) -> bool:
        return (self.data >> pos) & 1 == 1

    def set_n(self, pos: int):
        self.data |= 1 << pos

    def any_n_in_range(self, start: int, end: int) -> bool:
        bits = end - start
        mask = (1 << 64) - 1 if bits >= 64 else (1 << bits) - 1
        return ((self.data >> start) & mask) != 0

    def has_any_n(self) -> bool:
        return self.data != 0

    @staticmethod
    def empty() -> "NMask":
        return NMask(0)


def pack_ascii(seqs):
    """Packs a list of ASCII sequences (str/bytes) in add_sequence order.

    Returns (packed u64[words], nmask u64[words], offsets i64[n], lengths
    i64[n]).  Vectorised restatement of sequence.mojo:38-66."""
    bs = [s.encode() if isinstance(s, str) else bytes(s) for s in seqs]
    n = len(bs)
    lengths = np.fromiter((len(b) for b in bs), np.int64, n)
    words = (lengths + 31) // 32
    offsets = np.zeros(n, np.int64)
    if n:
        np.cumsum(words[:-1], out=offsets[1:])
    total_words = int(words.sum()) if n else 0
    packed = np.zeros(total_words, np.uint64)
    nmask = np.zeros(total_words, np.uint64)
    if total_words:
        buf = np.frombuffer(b"".join(bs), np.uint8)
        codes = _LUT[buf]
        # position of every base inside the padded 32-per-word layout
        starts = np.repeat(offsets * 32 - np.concatenate(([0], np.cumsum(lengths)[:-1])), lengths)
        pos = np.arange(buf.size, dtype=np.int64) + starts
        padded = np.zeros(total_words * 32, np.uint8)
        padded[pos] = codes
        isn = np.zeros(total_words * 32, np.uint8)
        isn[pos] = codes == 4
        padded[isn.astype(bool)] = 0
        grid = padded.reshape(total_words, 32).astype(np.uint64)
        shifts = (62 - 2 * np.arange(32, dtype=np.uint64)).astype(np.uint64)
        packed = np.bitwise_or.reduce(grid << shifts, axis=1).astype(np.uint64)
        ngrid = isn.reshape(total_words, 32).astype(np.uint64)
        nshifts = np.arange(32, dtype=np.uint64)
        nmask = np.bitwise_or.reduce(ngrid << nshifts, axis=1).astype(np.uint64)
    return packed, nmask, offsets, lengths


class SequenceBatch:
    """SoA batch of 2-bit packed sequences (sequence.mojo:23-75)."""

    def __init__(self, capacity: int = 256):
        self.packed = np.zeros(0, np.uint64)
        self.n_masks = np.zeros(0, np.uint64)
        self.offsets = np.zeros(0, np.int64)
        self.lengths = np.zeros(0, np.int64)
        self._pending = []
        self._pinned_blocks = []

    # -- construction -------------------------------------------------------
    def add_sequence(self, src, length: int | None = None):
        """Encode and append one ASCII sequence (sequence.mojo:38-66)."""
        b = src.encode() if isinstance(src, str) else bytes(src)
        if length is not None:
            b = b[:length]
        self._pending.append(b)

    def add_sequences(self, seqs):
        for s in seqs:
            self.add_sequence(s)

    def _flush(self):
        if not self._pending:
            return
        p, m, o, l = pack_ascii(self._pending)
        self._pending = []
        base = self.packed.size
        self.packed = np.concatenate((self.packed, p))
        self.n_masks = np.concatenate((self.n_masks, m))
        self.offsets = np.concatenate((self.offsets, o + base))
        self.lengths = np.concatenate((self.lengths, l))

    @classmethod
    def from_arrays(cls, packed, n_masks, offsets, lengths, pinned: bool = False):
        b = cls()
        if pinned:
            b.packed = pinned_empty(len(packed), np.uint64, b)
            b.packed[:] = packed
            b.n_masks = pinned_empty(len(n_masks), np.uint64, b)
            b.n_masks[:] = n_masks
            b.offsets = pinned_empty(len(offsets), np.int64, b)
            b.offsets[:] = offsets
            b.lengths = pinned_empty(len(lengths), np.int64, b)
            b.lengths[:] = lengths
        else:
            b.packed = np.ascontiguousarray(packed, np.uint64)
            b.n_masks = np.ascontiguousarray(n_masks, np.uint64)
            b.offsets = np.ascontiguousarray(offsets, np.int64)
            b.lengths = np.ascontiguousarray(lengths, np.int64)
        return b

    @classmethod
    def from_strings(cls, seqs):
        b = cls()
        b.add_sequences(seqs)
        b._flush()
        return b

    # -- reference API --------------------------------------------------------
    @property
    def count(self) -> int:
        self._flush()
        return int(self.lengths.size)

    def total_bases(self) -> int:
        self._flush()
        return int(self.lengths.sum())

    def words_for(self, idx: int) -> int:
        self._flush()
        return (int(self.lengths[idx]) + 31) // 32

    def arrays(self):
        """(packed, n_masks, offsets, lengths) as contiguous numpy arrays."""
        self._flush()
        return self.packed, self.n_masks, self.offsets, self.lengths

    def __del__(self):
        for blk in getattr(self, "_pinned_blocks", []):
            blk.free()


class SequenceView:
    """Owned copy of one sequence's words (sequence.mojo:78-120)."""

    def __init__(self, packed, n_masks, length: int, word_count: int):
        self.packed = np.ascontiguousarray(packed, np.uint64)
        self.n_masks = np.ascontiguousarray(n_masks, np.uint64)
        self.length = int(length)
        self.word_count = int(word_count)

    def get_base(self, pos: int) -> int:
        return get_base_from_word(self.packed[pos // BASES_PER_WORD], pos % BASES_PER_WORD)

    def is_n(self, pos: int) -> bool:
        return NMask(int(self.n_masks[pos // BASES_PER_WORD])).is_n(pos % BASES_PER_WORD)

    def has_n_in_window(self, start: int, end: int) -> bool:
        first, last = start // BASES_PER_WORD, (end - 1) // BASES_PER_WORD
        for w in range(first, last + 1):
            lo = max(0, start - w * BASES_PER_WORD)
            hi = min(BASES_PER_WORD, end - w * BASES_PER_WORD)
            if NMask(int(self.n_masks[w])).any_n_in_range(lo, hi):
                return True
        return False


def get_view(batch: SequenceBatch, idx: int) -> SequenceView:
    """sequence.mojo:123-137: copy sequence idx into a SequenceView."""
    packed, nm, off, ln = batch.arrays()
    o, L = int(off[idx]), int(ln[idx])
    nw = (L + 31) // 32
    return SequenceView(packed[o:o + nw].copy(), nm[o:o + nw].copy(), L, nw)


# -- pinned host memory ------------------------------------------------------------

class _PinnedBlock:
    def __init__(self, nbytes: int):
        from . import _lib
        self._L = _lib.lib()
        ptr = ctypes.c_void_p()
        _lib.check(self._L.gb2_host_alloc(max(int(nbytes), 8), ctypes.byref(ptr)))
        self.ptr = ptr.value
        self.nbytes = int(nbytes)

    def free(self):
        if self.ptr:
            self._L.gb2_host_free(self.ptr)
            self.ptr = None


def pinned_empty(n: int, dtype, owner) -> np.ndarray:
    """A numpy array in page-locked memory, freed with `owner`."""
    dtype = np.dtype(dtype)
    blk = _PinnedBlock(max(int(n), 1) * dtype.itemsize)
    owner._pinned_blocks.append(blk)
    buf = (ctypes.c_char * blk.nbytes).from_address(blk.ptr)
    return np.frombuffer(buf, dtype, count=int(n))
