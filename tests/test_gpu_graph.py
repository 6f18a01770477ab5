"""CUDA-graph replay of the resident entry points (gb2_sw_banded,
gb2_wfa_affine) under GB2_FLAG_GRAPH: the first call with a shape runs
eagerly, the second is captured and launched as a graph, later ones replay
it.  Every call must give the results of the eager launches (the default),
also when the caller's result array moves, after the context's buffers are
reallocated by a larger call, and after a batch is freed and uploaded again."""
import numpy as np
import pytest

from genomics_b200 import AlignConfig, SequenceBatch, WFAConfig, synth
from genomics_b200._lib import FLAG_GRAPH
from genomics_b200.core import pinned_empty
from genomics_b200.device import SW_RESULT_DTYPE

pytestmark = pytest.mark.gpu

CFG = AlignConfig(2, -4, -4, -2, 32)


class _Owner:
    _pinned_blocks = []


def _pinned_results(n):
    return pinned_empty(n * SW_RESULT_DTYPE.itemsize, np.uint8, _Owner).view(SW_RESULT_DTYPE)


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.int32), np.asarray(b).view(np.int32))


@pytest.mark.parametrize("n", [5000, 300_000])  # one launch; four parts on two executors
def test_sw_replay_matches_eager(device, n):
    q, r, _, _ = synth.generate(1, n, seed=77)
    dq, dr = device.upload_batch(q, with_nmask=False), device.upload_batch(r, with_nmask=False)
    ref = device.sw_banded(dq, dr, CFG, flags=0).copy()
    outs = [np.zeros(n, SW_RESULT_DTYPE), _pinned_results(n), _pinned_results(n),
            np.zeros(n, SW_RESULT_DTYPE)]
    device.stats_reset()
    for i in range(6):  # eager, capture, replays; the result array changes between calls
        out = outs[i % len(outs)]
        out[:] = np.zeros(1, SW_RESULT_DTYPE)
        device.sw_banded(dq, dr, CFG, out=out, flags=FLAG_GRAPH)
        assert _same(out, ref), f"call {i}"
    assert device.stats()["launches"] >= 6  # replays count the graph's kernels
    # a larger call reallocates the context's buffers; the graph must not replay
    # stale addresses
    q2, r2, _, _ = synth.generate(1, 2 * n, seed=78)
    dq2, dr2 = device.upload_batch(q2, with_nmask=False), device.upload_batch(r2, with_nmask=False)
    big = device.sw_banded(dq2, dr2, CFG, flags=FLAG_GRAPH)
    assert _same(big, device.sw_banded(dq2, dr2, CFG, flags=0))
    for _ in range(3):
        assert _same(device.sw_banded(dq, dr, CFG, flags=FLAG_GRAPH), ref)
    for b in (dq, dr, dq2, dr2):
        b.close()


def test_sw_replay_after_batch_reupload(device):
    """A batch freed and uploaded again (other sequences, maybe the same device
    addresses) gives the new batch's results."""
    n = 3000
    res = []
    for seed in (5, 6):
        q, r, _, _ = synth.generate(1, n, seed=seed)
        dq = device.upload_batch(q, with_nmask=False)
        dr = device.upload_batch(r, with_nmask=False)
        for _ in range(3):
            got = device.sw_banded(dq, dr, CFG, flags=FLAG_GRAPH)
        assert _same(got, device.sw_banded(dq, dr, CFG, flags=0))
        res.append(got.copy())
        dq.close()
        dr.close()
    assert not _same(res[0], res[1])


def test_sw_replay_with_bands(device):
    """Per-pair bands are copied before every launch: changing their values between
    replays changes the results accordingly."""
    rng = np.random.default_rng(9)
    strs = lambda k: ["".join(rng.choice(list("ACGT"), int(rng.integers(50, 400)))) for _ in range(k)]
    q, r = SequenceBatch.from_strings(strs(800)), SequenceBatch.from_strings(strs(800))
    dq, dr = device.upload_batch(q, with_nmask=False), device.upload_batch(r, with_nmask=False)
    for trial in range(3):
        bands = rng.choice([16, 32, 64, 128], 800).astype(np.int32)
        bands[0] = 128  # the same widest band, so the shape (and the graph) is kept
        ref = device.sw_banded(dq, dr, CFG, bands=bands, flags=0).copy()
        for _ in range(3):
            assert _same(device.sw_banded(dq, dr, CFG, bands=bands, flags=FLAG_GRAPH), ref), trial
    dq.close()
    dr.close()


def test_wfa_replay_matches_eager_and_oracle(device, oracle):
    q, r, _, _ = synth.generate(2, 400, seed=12)
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    cfg = WFAConfig(4, 6, 2, me)
    dq, dr = device.upload_batch(q, with_nmask=False), device.upload_batch(r, with_nmask=False)
    ref = device.wfa_affine(dq, dr, cfg, flags=0).copy()
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    want, _ = oracle.wfa_batch(qp, qo[:40], ql[:40], rp, ro[:40], rl[:40], 4, 6, 2, me,
                               envelope=True)
    assert np.array_equal(ref[:40], want)
    for i in range(4):
        assert np.array_equal(device.wfa_affine(dq, dr, cfg, flags=FLAG_GRAPH), ref), f"call {i}"
    dq.close()
    dr.close()
