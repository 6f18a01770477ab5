"""FASTA ingest (tests/fasta_loader.mojo:11-49) on generated FASTA text: the
reference loader's join/strip/upper rules, packing through add_sequence, and
multi-record files packed on the GPU equal to the host packing."""
import random

import numpy as np
import pytest

from genomics_b200 import fasta


def _write(path, records, width, newline="\n", lower=False, blank_lines=False):
    out = []
    for name, seq in records:
        if name is not None:
            out.append(">" + name)
        s = seq.lower() if lower else seq
        for i in range(0, len(s), width):
            out.append(s[i:i + width])
            if blank_lines and i % (3 * width) == 0:
                out.append("   ")
    path.write_bytes(newline.join(out).encode() + newline.encode())


def _random_records(rng, n, maxlen):
    recs = []
    for i in range(n):
        L = rng.randint(0, maxlen)
        seq = "".join(rng.choice("ACGT") for _ in range(L))
        if L > 20 and rng.random() < 0.5:  # an N run
            a = rng.randint(0, L - 10)
            seq = seq[:a] + "N" * rng.randint(1, 10) + seq[a + 10:]
        recs.append((f"seq{i} synthetic", seq))
    return recs


@pytest.mark.parametrize("width,newline,lower,blank", [(60, "\n", False, False),
                                                       (80, "\r\n", True, True),
                                                       (7, "\n", True, False)])
def test_single_sequence_loader(tmp_path, oracle, width, newline, lower, blank):
    rng = random.Random(width)
    seq = "".join(rng.choice("ACGTN") for _ in range(rng.randint(1, 3000)))
    p = tmp_path / "one.fa"
    _write(p, [("chrT test", seq)], width, newline, lower, blank)
    got = fasta.load_fasta_seq(str(p))
    assert got == seq
    b = fasta.make_batch_from_seq(got)
    pk, nm = oracle.pack(seq)
    bp, bm, bo, bl = b.arrays()
    assert (bp == pk).all() and (bm == nm).all() and bl[0] == len(seq)
    sub = fasta.make_batch_substr(got, 5, min(len(got), 205))
    sp, _, _, sl = sub.arrays()
    assert sl[0] == len(got[5:205]) and (sp == oracle.pack(got[5:205])[0]).all()


def test_multi_record_loader(tmp_path):
    rng = random.Random(4)
    recs = _random_records(rng, 50, 700)
    p = tmp_path / "many.fa"
    _write(p, recs, 61, lower=True, blank_lines=True)
    got = fasta.load_fasta_records(str(p))
    assert [n for n, _ in got] == [n for n, _ in recs]
    assert [s for _, s in got] == [s for _, s in recs]
    # the reference's single-sequence loader joins every record
    assert fasta.load_fasta_seq(str(p)) == "".join(s for _, s in recs)


@pytest.mark.gpu
def test_fasta_packed_on_device(tmp_path, device):
    rng = random.Random(8)
    recs = _random_records(rng, 300, 5000)
    p = tmp_path / "dev.fa"
    _write(p, recs, 70, newline="\r\n", lower=True)
    db, names = fasta.fasta_to_device(str(p), device)
    assert names == [n for n, _ in recs]
    host = fasta.SequenceBatch.from_strings([s for _, s in recs])
    back = device.download_batch(db)
    for a, b in zip(back.arrays(), host.arrays()):
        assert np.array_equal(a, b)
    db.close()
