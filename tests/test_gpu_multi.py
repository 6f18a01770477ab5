"""One pair list over several contexts (gb2_*_multi): the slices, each aligned
by its own context from the caller's host arrays, give exactly one call's
results in input order.  Two contexts on the one GPU stand in for two GPUs."""
import numpy as np
import pytest

from genomics_b200 import AlignConfig, GenomicsDevice, WFAConfig, multi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def two():
    devs = [GenomicsDevice(0), GenomicsDevice(0)]
    yield devs
    for d in devs:
        d.close()


def test_sw_split_over_two_contexts_equals_one_call(device, two):
    q, r, bands, _ = synth.generate(3, 20_000)
    cfg = AlignConfig(2, -4, -4, -2, 32)
    want = device.sw_banded(q, r, cfg, bands=bands)
    got = multi.sw_banded_multi(two, q, r, cfg, bands=bands)
    assert (got == want).all()
    q1, r1, _, _ = synth.generate(1, 100_000)
    assert (multi.sw_banded_multi(two, q1, r1, cfg) == device.sw_banded(q1, r1, cfg)).all()


def test_wfa_split_over_two_contexts_equals_one_call(device, two):
    q, r, _, _ = synth.generate(2, 3000)
    cfg = WFAConfig(4, 6, 2, synth.wfa_max_error_cover(q, r, 4, 6, 2))
    want = np.asarray(device.wfa_affine(q, r, cfg))
    assert (multi.wfa_affine_multi(two, q, r, cfg) == want).all()
    assert (multi.wfa_affine_multi(two[:1], q, r, cfg) == want).all()
