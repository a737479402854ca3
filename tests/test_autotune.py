"""Autotuner logic that needs no GPU: FFT plans and candidate ranges."""
import pytest

from afid_b200 import BouIn
from afid_b200.autotune import candidates, fft_plan, TuneCache


@pytest.mark.parametrize("n,plan", [(768, [3, 16, 16]), (1280, [5, 16, 16]), (384, [3, 8, 16]),
                                    (96, [2, 3, 16]), (48, [3, 16]), (32, [2, 16]), (64, [4, 16]),
                                    (128, [8, 16]), (16, [16]), (12, [3, 4]), (14, [2, 7])])
def test_fft_plan(n, plan):
    assert fft_plan(n) == plan
    prod = 1
    for r in plan:
        prod *= r
    assert prod == n


def test_fft_plan_rejects_large_primes():
    with pytest.raises(ValueError):
        fft_plan(22)


@pytest.mark.parametrize("nyz", [32, 48, 96, 128, 384, 768, 1280])
def test_candidates_fit_shared_memory(nyz):
    c = candidates(BouIn(nxm=64, nym=nyz, nzm=nyz))
    for v in c["fft_y_lines"]:
        assert (2 * v + 1) * nyz * 16 <= 200 * 1024
    for v in c["fft_z_lines"]:
        assert (2 * v + 1) * nyz * 16 <= 200 * 1024 and v <= nyz // 2 + 1
    assert c["k1_minb"] == [2, 3, 4]


def test_cache_roundtrip(tmp_path):
    path = str(tmp_path / "t.json")
    c = TuneCache(path)
    cfg = BouIn(nxm=32, nym=48, nzm=48)
    assert c.get(cfg) is None
    c.put(cfg, {"fft_y_lines": 4, "fft_z_lines": 8, "k1_minb": 2})
    c.save()
    assert TuneCache(path).get(cfg)["fft_z_lines"] == 8
