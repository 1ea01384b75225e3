"""The accuracy bench (oz2.bench_accuracy): its input distributions on CPU, and one small run on
the device with the reference's CSV columns."""
import numpy as np
import pytest

from oz2 import bench_accuracy as ba


def test_distributions_have_their_structure():
    A = ba.generate(40, 64, "spike", 3, True)
    base = ba.generate(40, 64, "urand", 3, True)
    r = np.arange(40)
    assert np.array_equal(A[r, (r * 7919) % 64], base[r, (r * 7919) % 64] * 2.0 ** 40)
    C = ba.generate(40, 64, "cancel", 4, True)
    assert np.array_equal(C[:, 32:], C[:, :32])
    Bc = ba.generate(64, 40, "cancel", 5, False)
    Bu = ba.generate(64, 40, "urand", 5, False)
    assert np.array_equal(Bc[32:], -Bu[:32] + np.ldexp(Bu[32:], -30))
    S = ba.generate(5, 7, "sincos", 0, True)
    assert S[2, 3] == np.sin(5.0)
    P = ba.generate(100, 100, "phi4", 1, True)
    assert np.isfinite(P).all() and P.flags["F_CONTIGUOUS"]
    assert ba.parse_ints("4-6,9") == [4, 5, 6, 9]


@pytest.mark.gpu
def test_small_run_reports_every_row():
    lines = ba.main(["--k", "256", "--s", "8,20", "--L", "4,8", "--dist", "urand,phi2,sincos,spike,cancel",
                     "--mn", "96"])
    rows = [dict(zip(ba.CSV_HEADER.split(","), l.split(","))) for l in lines]
    assert len(rows) == 5 * 5
    for r in rows:
        assert r["method"] in ("dgemm_gpu", "ozaki2", "ozaki1")
        assert float(r["ulp_max"]) >= 0 and 0 <= float(r["cr_frac"]) <= 1
    # s = 20 carries about 70 bits per element at k = 256: nearly every entry correctly rounded
    u20 = next(r for r in rows if r["dist"] == "urand" and r["method"] == "ozaki2" and r["s"] == "20")
    gpu = next(r for r in rows if r["dist"] == "urand" and r["method"] == "dgemm_gpu")
    assert float(u20["cr_frac"]) >= max(0.99, float(gpu["cr_frac"])) and float(u20["fro_rel"]) <= 1e-15
    # Ozaki-I with L = 8: 36 GEMMs, 54 bits per element; L = 4: 10 GEMMs, 26 bits
    o8 = next(r for r in rows if r["dist"] == "urand" and r["method"] == "ozaki1" and r["s"] == "36")
    o4 = next(r for r in rows if r["dist"] == "urand" and r["method"] == "ozaki1" and r["s"] == "10")
    assert o8["tk"] == "54" and o4["tk"] == "26"
    assert float(o8["fro_rel"]) <= 1e-14 and float(o4["fro_rel"]) > 1e-9
    zl = ba.main(["--k", "256", "--s", "20", "--dist", "urand", "--mn", "64", "--complex"])
    z = [dict(zip(ba.CSV_HEADER.split(","), l.split(","))) for l in zl]
    assert [r["method"] for r in z] == ["zgemm_gpu", "ozaki2_3m"] and z[0]["dist"] == "zurand"
    assert float(z[1]["cr_frac"]) >= 0.99 and float(z[1]["fro_rel"]) <= 1e-15
