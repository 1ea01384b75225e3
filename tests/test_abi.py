"""The C ABI library on the CPU: it loads, exports every entry point the header declares, and
its host-only planning entry points agree with the oracle. No kernel is launched here."""
import ctypes as C
import os
import re
import subprocess

import pytest

from common import ROOT

HEADER = os.path.join(ROOT, "include", "oz2", "oz2.h")
LIB = os.path.join(ROOT, "os2-xe_b200", "oz2", "liboz2.so")


def declared():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(oz2_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "liboz2.so is not built (python os2-xe_b200/build.py)"
    lib = C.CDLL(LIB)
    names = declared()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_planning_entry_points_match_oracle(oracle):
    import oz2
    for s in range(2, 25):
        for k in [1, 7, 1024, 8192, 131071, 262144]:
            try:
                want = oracle.precision_bits(k, s)
            except ValueError:
                with pytest.raises(ValueError, match="too small"):
                    oz2.Ozaki2.precision_bits(k, s)
                continue
            assert oz2.Ozaki2.precision_bits(k, s) == want
            assert oz2.Ozaki2.precision_bits_complex(k, s) == oracle.precision_bits(2 * k, s)
    for k in [1, 16, 1024, 2000, 8192, 131071, 300000]:
        for b in [1, 20, 40, 53, 60, 80, 90, 101]:
            assert oz2.Ozaki2.moduli_for_bits(k, b) == oracle.moduli_for_bits(k, b)
    with pytest.raises(ValueError, match=r"num_moduli must be in \[2, 24\]"):
        oz2.Ozaki2.precision_bits(100, 1)


def test_precision_bits_at_the_edges_of_k(oracle):
    """tk changes where k 2^(2 tk + 2) crosses M: k on both sides of every power of two up to 2^40
    and of M / 2^(2 t + 2) for each plan, against the oracle's plan"""
    import oz2
    ks = {2 ** e + d for e in range(41) for d in (-2, -1, 0, 1, 2) if 2 ** e + d >= 1}
    for s in range(2, 25):
        M = oracle.plan(s, 1).Mint
        for t in range(20, 101, 7):
            edge = M >> (2 * t + 2)
            ks.update(x for x in (edge - 1, edge, edge + 1) if 1 <= x < 2 ** 62)
    for s in range(2, 25):
        for k in sorted(ks):
            try:
                want = oracle.precision_bits(k, s)
            except ValueError:
                with pytest.raises(ValueError, match="too small"):
                    oz2.Ozaki2.precision_bits(k, s)
                continue
            assert oz2.Ozaki2.precision_bits(k, s) == want, (s, k)


def test_null_handle_is_rejected():
    import oz2
    lib = oz2.lib()
    assert lib.oz2_dgemm(None, b"N", b"N", 1, 1, 1, 1.0, None, 1, None, 1, 0.0, None, 1, 8, None, 0, None) == 1
    assert b"null handle" in lib.oz2_last_error(None)
    assert lib.oz2_status_string(4) == b"device-side wait timed out"


def test_cpp_header_compiles():
    """include/oz2/ozaki2.hpp (the reference's class over the C ABI) compiles and links"""
    src = os.path.join(ROOT, "include", "oz2", "ozaki2.hpp")
    # the grouped / adaptive members are instantiated (not run: no device here)
    prog = ('#include "oz2/ozaki2.hpp"\n'
            "void use(oz2::Ozaki2& oz) { std::vector<oz2::Problem> ps(1); oz.gemm_grouped(ps);\n"
            "  oz2::AdaptiveStats st = oz.gemm_adaptive(ps, 53, oz2::Adaptive::Mlp); (void)st;\n"
            "  oz.set_mlp_weights({}); oz.set_adaptive_options(512, 0.99f); oz.autotune_grouped(ps); }\n"
            "void use1(oz1::Ozaki1& o) { o.gemm(1, 1, 1, nullptr, 1, nullptr, 1, nullptr, 1, 4); }\n"
            "int main(int argc, char**) { if (argc > 5) { oz2::Ozaki2 oz; use(oz); oz1::Ozaki1 o; use1(o); }\n"
            "  return oz2::Ozaki2::moduli_for_bits(1024, 53) == 15 && oz1::Ozaki1::num_gemms(9) == 45 &&\n"
            "    oz1::Ozaki1::precision_bits(9) == 61 ? 0 : 1; }\n")
    exe = os.path.join(ROOT, "os2-xe_b200", "_build", "hdr_check")
    os.makedirs(os.path.dirname(exe), exist_ok=True)
    r = subprocess.run(["/usr/bin/g++", "-std=c++17", "-x", "c++", "-", "-I" + os.path.join(ROOT, "include"),
                        "-I/usr/local/cuda/include", "-o", exe, "-x", "none", LIB,
                        "-Wl,-rpath," + os.path.dirname(LIB)],
                       input=prog, capture_output=True, text=True, timeout=120)
    assert os.path.exists(src)
    assert r.returncode == 0, r.stderr
    assert subprocess.run([exe], timeout=60).returncode == 0


def test_split_kernel_selector():
    """process-wide choice of the real split's kernel: host-only, checked values"""
    import oz2
    oz2.set_split_kernel(oz2.SPLIT_DP4A)
    oz2.set_split_kernel(oz2.SPLIT_TENSOR_CORE)
    with pytest.raises(ValueError, match="split kernel"):
        oz2.set_split_kernel(7)


def test_crt_kernel_selector():
    import oz2
    for kind in (oz2.CRT_DP2A, oz2.CRT_TENSOR_CORE, oz2.CRT_AUTO):
        oz2.set_crt_kernel(kind)
    with pytest.raises(ValueError, match="CRT kernel"):
        oz2.set_crt_kernel(3)
