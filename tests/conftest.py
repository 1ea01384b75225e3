import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for sub in ("tests", "tests/golden", "oracle", "os2-xe_b200"):
    sys.path.insert(0, os.path.join(ROOT, sub))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device of compute capability 10.0 (B200)")
    # the oracle is plain C: build it when missing (here and on a GPU box alike)
    so = os.path.join(ROOT, "oracle", "liboz2_oracle.so")
    if not os.path.exists(so):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "liboz2_oracle.so"], check=True,
                       capture_output=True)


@pytest.fixture(scope="session")
def oracle():
    from common import oracle as make
    return make()


@pytest.fixture(scope="session")
def ref():
    from pyoracle import Ref, ref_available
    if not ref_available():
        pytest.skip("oracle/_ref (the reference built for the host) is not present")
    r = Ref()
    r.set_threads(os.cpu_count() or 1)
    return r


@pytest.fixture(scope="session")
def oz():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    import oz2
    h = oz2.Ozaki2(torch.cuda.current_stream())
    yield h
    h.close()
