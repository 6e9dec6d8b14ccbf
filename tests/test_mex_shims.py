"""The MEX gateways compile (against a declaration-only mex.h; MATLAB is not
installed) and call only entry points the C ABI declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MEX = os.path.join(ROOT, "tom_b200", "mex")


@pytest.mark.parametrize("src", sorted(f for f in os.listdir(MEX) if f.endswith(".c")))
def test_gateway_compiles(src, tmp_path):
    r = subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-c", "-I" + os.path.join(MEX, "stub"),
                        "-I" + os.path.join(ROOT, "include"), "-I" + MEX, os.path.join(MEX, src), "-o",
                        str(tmp_path / (src + ".o"))], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    txt = open(os.path.join(MEX, src)).read()
    from tom_b200._lib import declared_symbols
    used = set(re.findall(r"\b(tomgpu_[a-z0-9_]+)\s*\(", txt)) - {"tomgpu_mex_ctx", "tomgpu_mex_check",
                                                                    "tomgpu_mex_dims3"}
    assert used <= set(declared_symbols())
