"""Autotuner logic that needs no GPU: FFT plans and candidate ranges."""
import pytest

from afid_b200 import BouIn
from afid_b200.autotune import candidates, fft_plan, TuneCache


@pytest.mark.parametrize("n,plan", [(768, [16, 16, 3]), (1280, [16, 16, 5]), (384, [16, 8, 3]),
                                    (96, [16, 2, 3]), (48, [16, 3]), (32, [16, 2]), (64, [16, 4]),
                                    (128, [16, 8]), (16, [16]), (12, [4, 3]), (14, [2, 7])])
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
        assert (4 * v * (nyz // 2 + 1) + nyz) * 16 <= 200 * 1024 and v * nyz <= 14 * 256
        assert v & (v - 1) == 0
    for v in c["fft_z_lines"]:
        assert (2 * v * nyz + nyz) * 16 <= 200 * 1024 and v * nyz <= 14 * 256
        assert v & (v - 1) == 0
    assert c["fft_y_lines"] and c["fft_z_lines"]
    assert c["k1_minb"] == [2, 3, 4, 5, 6, 7, 8]


def test_cache_roundtrip(tmp_path):
    path = str(tmp_path / "t.json")
    c = TuneCache(path)
    cfg = BouIn(nxm=32, nym=48, nzm=48)
    assert c.get(cfg) is None
    c.put(cfg, {"fft_y_lines": 4, "fft_z_lines": 8, "k1_minb": 2})
    c.save()
    assert TuneCache(path).get(cfg)["fft_z_lines"] == 8
