"""FASTA ingest for the alignment path.

The first three functions mirror the reference's fixture loader
(tests/fasta_loader.mojo:11-49): `load_fasta_seq` joins every line that is
not a header ('>' after leading blanks), stripped and upper-cased;
`make_batch_from_seq` / `make_batch_substr` encode a string (or a slice of
it) into a one-sequence SequenceBatch through add_sequence
(genomics/core/sequence.mojo:38-66).

`load_fasta_records` and `fasta_to_device` serve batch workloads: every record
of a multi-record file becomes one sequence; `fasta_to_device` packs them on
the GPU (gb2_batch_from_ascii) straight from the file's bytes, so a genome
never goes through a per-base host loop.
"""
from __future__ import annotations

from .core import SequenceBatch


def load_fasta_seq(path: str) -> str:
    """Single-sequence FASTA -> upper-case nucleotide string (fasta_loader.mojo:11-23)."""
    with open(path, "r") as f:
        lines = f.read().splitlines()
    return "".join(line.strip().upper() for line in lines if not line.lstrip().startswith(">"))


def make_batch_from_seq(seq: str) -> SequenceBatch:
    """One-entry SequenceBatch of seq (fasta_loader.mojo:26-33)."""
    return SequenceBatch.from_strings([seq])


def make_batch_substr(seq: str, start: int, end: int) -> SequenceBatch:
    """One-entry SequenceBatch of seq[start:end] (fasta_loader.mojo:36-49)."""
    return SequenceBatch.from_strings([seq[start:end]])


def _records(data: bytes):
    """(name, sequence bytes with line breaks and surrounding blanks removed) per record.
    Lines before the first header form an unnamed record, as load_fasta_seq keeps them."""
    recs = []
    name, parts = None, []
    for line in data.splitlines():
        s = line.strip()
        if line.lstrip().startswith(b">"):
            if parts or name is not None:
                recs.append((name, b"".join(parts)))
            name, parts = s[1:].decode(errors="replace"), []
        else:
            parts.append(s)
    if parts or name is not None:
        recs.append((name, b"".join(parts)))
    return recs


def load_fasta_records(path: str):
    """Multi-record FASTA -> [(name, upper-case sequence)] in file order."""
    with open(path, "rb") as f:
        data = f.read()
    return [(n, s.upper().decode()) for n, s in _records(data)]


def fasta_to_device(path: str, device):
    """Every record of a FASTA file as one sequence of a device-resident batch, packed on
    the GPU from the raw bytes (case does not matter to the 2-bit code or the N mask).
    Returns (DeviceBatch, names)."""
    with open(path, "rb") as f:
        data = f.read()
    recs = _records(data)
    return device.batch_from_ascii([s for _, s in recs]), [n for n, _ in recs]
