"""Host-side pieces of bench.py's JSON contract, without a GPU: the workload record, the
roofline inputs read from the committed profile summaries and the measured peaks, and the
engine statistics keys matching the library's hook."""
import re
from pathlib import Path

import bench

ROOT = Path(__file__).resolve().parent.parent


def test_config_names_the_workload_and_no_model():
    cfg = bench.config_dict("block even-odd BiCGStab on S")
    assert cfg["workload"].startswith("su3-clover-24^3x48")
    assert cfg["rhs"] == 44 and cfg["tolerance"] == 1e-10
    assert not {"model", "global_batch", "seq_len"} & set(cfg)


def test_traffic_comes_from_the_profile_summary():
    text = (ROOT / "profiles" / "batched_stencil_schur_clover_24c48_nb16.md").read_text()
    Vh = 24 * 24 * 24 * 48 // 2
    for reals in (12, 18):
        m = re.search(rf"traffic_bytes_per_launch\[prec=1,kernel=xpay,batch=16,links={reals}\]:\s*(\d+)", text)
        assert m, f"the profile summary lost its traffic line ({reals}-real links)"
        assert bench.traffic_from_profiles(1, 16, reals) == float(m.group(1))
        # algorithmic bytes of one 16-RHS FP32 launch against the measured traffic: re-read
        # neighbour spinors and the links' padding keep it within 20 % above them
        alg = (bench.STENCIL_SITE_BYTES[reals] + 16 * bench.STENCIL_RHS_BYTES[1]) * Vh
        assert 1.0 <= float(m.group(1)) / alg <= 1.2, reals


def test_peaks_are_measured_or_the_stated_fallback():
    pk = bench.peaks()
    assert pk["which"] in ("measured", "fallback")
    assert pk["hbm_gbs"] > 1000


def test_engine_keys_match_the_library_hook():
    header = (ROOT / "include" / "lym_b200.h").read_text()
    m = re.search(r"out\[8\][^;]*; n = (\d+)", header, re.S)
    assert m and int(m.group(1)) == len(bench.ENGINE_KEYS) == 9
