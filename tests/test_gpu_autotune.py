"""The autotuner (gb2_autotune): every candidate variant of a kernel gives the
same results, the fastest is installed in the context, later calls with the
variant field at 0 use it and still equal the oracle, and a saved table
restores the same choices."""
import ctypes
import os

import numpy as np
import pytest

from genomics_b200 import AlignConfig, WFAConfig, autotune, synth
from genomics_b200._lib import FLAG_INT32, GB2_EINVAL

from test_gpu_sw import assert_same, oracle_sw

pytestmark = pytest.mark.gpu

SW_VARIANTS = {16: {0, 1}, 32: {0, 1, 2}, 64: {0, 1}, 128: {0, 1}}
WFA_VARIANTS = {0x00, 0x04, 0x03, 0x10, 0x20}


@pytest.fixture(scope="module")
def mixed(device):
    """2,000 pairs of the mixed-length workload (100-2,000 bp, N runs)."""
    q, r, bands, _ = synth.generate(3, 2000, seed=41)
    dq, dr = device.upload_batch(q, with_nmask=False), device.upload_batch(r, with_nmask=False)
    yield q, r, dq, dr, bands
    dq.close()
    dr.close()
    for b in SW_VARIANTS:
        device.tune_set("sw", 0, b)


@pytest.mark.parametrize("band", [16, 32, 64, 128])
def test_sw_tuning_installs_an_equal_variant(device, oracle, mixed, band):
    q, r, dq, dr, _ = mixed
    cfg = AlignConfig(2, -4, -4, -2, band)
    res = device.autotune("sw", dq, dr, cfg, reps=2)
    assert res["band_class"] == band
    assert {v for v, _ in res["candidates"]} == SW_VARIANTS[band]
    assert all(ms > 0 for _, ms in res["candidates"])
    assert res["chosen"] == min(res["candidates"], key=lambda c: c[1])[0]
    assert device.tune_get("sw", band) == res["chosen"]
    got = device.sw_banded(dq, dr, cfg, flags=FLAG_INT32)  # uses the installed variant
    assert_same(got[:300], oracle_sw(oracle, q, r, cfg, n=300), f"band {band}")
    for v in SW_VARIANTS[band]:  # every variant, explicitly
        other = device.sw_banded(dq, dr, cfg, flags=FLAG_INT32 | (v << 8))
        assert np.array_equal(got.view(np.int32), other.view(np.int32)), v


def test_sw_tuning_inside_the_mixed_call(device, oracle, mixed):
    """Per-pair bands: each class is tuned inside the whole mixed call, one after
    another; the mixed results then equal the oracle's."""
    q, r, dq, dr, bands = mixed
    cfg = AlignConfig(2, -4, -4, -2, 32)
    table = autotune.tune(device, dq, dr, sw_cfg=cfg, reps=1, pair_bands=bands)
    assert set(table["sw"]) == {"16", "32", "64", "128"}
    for b, v in table["sw"].items():
        assert device.tune_get("sw", int(b)) == v
    got = device.sw_banded(dq, dr, cfg, bands=bands, flags=FLAG_INT32)
    assert_same(got[:400], oracle_sw(oracle, q, r, cfg, bands=bands, n=400), "mixed tuned")
    for b in SW_VARIANTS:
        device.tune_set("sw", 0, b)


def test_wfa_tuning_installs_an_equal_variant(device, oracle):
    q, r, _, _ = synth.generate(2, 600, seed=43)
    me = synth.wfa_max_error_cover(q, r, 4, 6, 2)
    cfg = WFAConfig(4, 6, 2, me)
    dq, dr = device.upload_batch(q, with_nmask=False), device.upload_batch(r, with_nmask=False)
    base = device.wfa_affine(dq, dr, cfg).copy()
    res = device.autotune("wfa", dq, dr, cfg, reps=2)
    assert {v for v, _ in res["candidates"]} == WFA_VARIANTS
    assert device.tune_get("wfa") == res["chosen"]
    assert np.array_equal(device.wfa_affine(dq, dr, cfg), base)
    qp, _, qo, ql = q.arrays()
    rp, _, ro, rl = r.arrays()
    want, _ = oracle.wfa_batch(qp, qo[:30], ql[:30], rp, ro[:30], rl[:30], 4, 6, 2, me,
                               envelope=True)
    assert np.array_equal(base[:30], want)
    device.tune_set("wfa", 0)
    dq.close()
    dr.close()


def test_table_save_and_load(device, mixed, tmp_path):
    _, _, dq, dr, _ = mixed
    table = autotune.tune(device, dq, dr, sw_cfg=AlignConfig(2, -4, -4, -2, 32), bands=(32, 64),
                          reps=1)
    path = os.path.join(tmp_path, "tune.json")
    autotune.save(table, path)
    device.tune_set("sw", 0, 32)
    device.tune_set("sw", 0, 64)
    autotune.load(device, path)
    assert device.tune_get("sw", 32) == table["sw"]["32"]
    assert device.tune_get("sw", 64) == table["sw"]["64"]


def test_tuner_argument_errors(device, mixed):
    _, _, dq, dr, _ = mixed
    from genomics_b200._lib import GenomicsError
    with pytest.raises(GenomicsError):
        device.autotune("sw", dq, dr, AlignConfig(2, -4, -4, -2, 48))  # no variants for band 48
    with pytest.raises(GenomicsError):
        device.tune_set("sw", 1, 48)
    assert device.L.gb2_tune_set(device.ctx, 7, 32, 1) == GB2_EINVAL
