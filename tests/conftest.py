import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
for p in (ROOT, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libtomgpu.so")
    # the oracle's own C restatement needs no reference sources: build it if absent
    lib = os.path.join(ORACLE, "_ref", "liboracle.so")
    if not os.path.exists(lib):
        subprocess.run(["make", "-C", ORACLE, "oracle"], check=False, capture_output=True)


# host-side tests of the library's C++ (no GPU needed) skip, like the ABI
# tests, where libtomgpu.so has not been built
needs_library = pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "tom_b200", "libtomgpu.so")),
                                   reason="libtomgpu.so not built (python -m tom_b200.build_ext)")


@pytest.fixture(scope="session")
def oracle():
    import tm_oracle
    return tm_oracle


@pytest.fixture(scope="session")
def ref_libs(oracle):
    if not oracle.ref_available():
        pytest.skip("reference libraries (oracle/_ref) not built")
    return oracle


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import tom_b200
    return tom_b200
