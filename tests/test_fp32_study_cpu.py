"""The FP32 parity study (oracle/fp32_study.py) on a small sample: the
reference algorithm with REAL_T = float keeps the FP64 discrete outcome on
the large majority of traces, and where it does the IMFs agree to float
precision (median error a few 1e-7 of the trace's range)."""
from oracle import fp32_study


def test_fp32_study_small_sample():
    res = fp32_study.study(16, processes=2)
    for name, r in res.items():
        assert r["traces"] > 0, name
        assert r["same_n_imfs"] >= 0.75, (name, r)
        assert r["median_rel_err_same_n"] is not None and r["median_rel_err_same_n"] < 1e-5, (name, r)
